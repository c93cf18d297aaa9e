// Generated by gen_instances.py: class kernels (4,0|1,1), (4,0|2,0), (4,0|2,1).
#include "../eri_launch_d1.cuh"

namespace lible_b200
{
    cudaError_t launch_d1_10_02(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<4,0,1,1>(a, s, n);
    }
    cudaError_t launch_d1_10_03(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<4,0,2,0>(a, s, n);
    }
    cudaError_t launch_d1_10_04(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<4,0,2,1>(a, s, n);
    }
}
