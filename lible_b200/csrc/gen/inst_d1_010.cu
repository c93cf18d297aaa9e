// Generated by gen_instances.py: class kernels (3,1|1,1), (3,1|2,0), (3,1|2,1).
#include "../eri_launch_d1.cuh"

namespace lible_b200
{
    cudaError_t launch_d1_07_02(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<3,1,1,1>(a, s, n);
    }
    cudaError_t launch_d1_07_03(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<3,1,2,0>(a, s, n);
    }
    cudaError_t launch_d1_07_04(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<3,1,2,1>(a, s, n);
    }
}
