// Generated by gen_instances.py: class kernels (0,0|0,0), (1,0|0,0), (1,0|1,0).
#include "../eri_launch_d1.cuh"

namespace lible_b200
{
    cudaError_t launch_d1_00_00(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<0,0,0,0>(a, s, n);
    }
    cudaError_t launch_d1_01_00(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<1,0,0,0>(a, s, n);
    }
    cudaError_t launch_d1_01_01(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<1,0,1,0>(a, s, n);
    }
}
