// Generated by gen_instances.py: class kernels (3,0|3,0), (3,1|0,0), (3,1|1,0).
#include "../eri_launch_d1.cuh"

namespace lible_b200
{
    cudaError_t launch_d1_06_06(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<3,0,3,0>(a, s, n);
    }
    cudaError_t launch_d1_07_00(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<3,1,0,0>(a, s, n);
    }
    cudaError_t launch_d1_07_01(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<3,1,1,0>(a, s, n);
    }
}
