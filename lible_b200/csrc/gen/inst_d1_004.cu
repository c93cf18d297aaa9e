// Generated by gen_instances.py: class kernels (2,1|1,1), (2,1|2,0), (2,1|2,1).
#include "../eri_launch_d1.cuh"

namespace lible_b200
{
    cudaError_t launch_d1_04_02(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<2,1,1,1>(a, s, n);
    }
    cudaError_t launch_d1_04_03(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<2,1,2,0>(a, s, n);
    }
    cudaError_t launch_d1_04_04(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<2,1,2,1>(a, s, n);
    }
}
