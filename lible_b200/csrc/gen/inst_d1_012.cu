// Generated by gen_instances.py: class kernels (3,2|0,0), (3,2|1,0), (3,2|1,1).
#include "../eri_launch_d1.cuh"

namespace lible_b200
{
    cudaError_t launch_d1_08_00(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<3,2,0,0>(a, s, n);
    }
    cudaError_t launch_d1_08_01(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<3,2,1,0>(a, s, n);
    }
    cudaError_t launch_d1_08_02(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<3,2,1,1>(a, s, n);
    }
}
