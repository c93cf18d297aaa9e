// Generated by gen_instances.py: class kernels (5,0|3,3), (5,0|4,0), (5,0|5,0).
#include "../eri_launch_d1.cuh"

namespace lible_b200
{
    cudaError_t launch_d1_11_09(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<5,0,3,3>(a, s, n);
    }
    cudaError_t launch_d1_11_10(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<5,0,4,0>(a, s, n);
    }
    cudaError_t launch_d1_11_11(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<5,0,5,0>(a, s, n);
    }
}
