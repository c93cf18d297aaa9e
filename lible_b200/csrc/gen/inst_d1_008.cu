// Generated by gen_instances.py: class kernels (3,0|2,0), (3,0|2,1), (3,0|2,2).
#include "../eri_launch_d1.cuh"

namespace lible_b200
{
    cudaError_t launch_d1_06_03(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<3,0,2,0>(a, s, n);
    }
    cudaError_t launch_d1_06_04(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<3,0,2,1>(a, s, n);
    }
    cudaError_t launch_d1_06_05(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<3,0,2,2>(a, s, n);
    }
}
