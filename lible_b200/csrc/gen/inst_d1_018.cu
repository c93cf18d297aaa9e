// Generated by gen_instances.py: class kernels (3,3|3,3), (4,0|0,0), (4,0|1,0).
#include "../eri_launch_d1.cuh"

namespace lible_b200
{
    cudaError_t launch_d1_09_09(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<3,3,3,3>(a, s, n);
    }
    cudaError_t launch_d1_10_00(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<4,0,0,0>(a, s, n);
    }
    cudaError_t launch_d1_10_01(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<4,0,1,0>(a, s, n);
    }
}
