// Generated by gen_instances.py: class kernels (3,0|0,0), (3,0|1,0), (3,0|1,1).
#include "../eri_launch_d1.cuh"

namespace lible_b200
{
    cudaError_t launch_d1_06_00(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<3,0,0,0>(a, s, n);
    }
    cudaError_t launch_d1_06_01(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<3,0,1,0>(a, s, n);
    }
    cudaError_t launch_d1_06_02(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<3,0,1,1>(a, s, n);
    }
}
