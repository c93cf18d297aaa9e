// Generated by gen_instances.py: class kernels (3,3|2,0), (3,3|2,1), (3,3|2,2).
#include "../eri_launch_d1.cuh"

namespace lible_b200
{
    cudaError_t launch_d1_09_03(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<3,3,2,0>(a, s, n);
    }
    cudaError_t launch_d1_09_04(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<3,3,2,1>(a, s, n);
    }
    cudaError_t launch_d1_09_05(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<3,3,2,2>(a, s, n);
    }
}
