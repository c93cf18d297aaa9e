// Generated by gen_instances.py: class kernels (4,0|3,2), (4,0|3,3), (4,0|4,0).
#include "../eri_launch_d1.cuh"

namespace lible_b200
{
    cudaError_t launch_d1_10_08(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<4,0,3,2>(a, s, n);
    }
    cudaError_t launch_d1_10_09(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<4,0,3,3>(a, s, n);
    }
    cudaError_t launch_d1_10_10(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<4,0,4,0>(a, s, n);
    }
}
