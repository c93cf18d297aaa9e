// Generated by gen_instances.py: class kernels (4,0|2,2), (4,0|3,0), (4,0|3,1).
#include "../eri_launch_d1.cuh"

namespace lible_b200
{
    cudaError_t launch_d1_10_05(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<4,0,2,2>(a, s, n);
    }
    cudaError_t launch_d1_10_06(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<4,0,3,0>(a, s, n);
    }
    cudaError_t launch_d1_10_07(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<4,0,3,1>(a, s, n);
    }
}
