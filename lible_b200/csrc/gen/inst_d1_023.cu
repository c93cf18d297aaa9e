// Generated by gen_instances.py: class kernels (5,0|2,0), (5,0|2,1), (5,0|2,2).
#include "../eri_launch_d1.cuh"

namespace lible_b200
{
    cudaError_t launch_d1_11_03(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<5,0,2,0>(a, s, n);
    }
    cudaError_t launch_d1_11_04(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<5,0,2,1>(a, s, n);
    }
    cudaError_t launch_d1_11_05(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<5,0,2,2>(a, s, n);
    }
}
