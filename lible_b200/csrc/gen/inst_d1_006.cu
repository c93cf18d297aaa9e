// Generated by gen_instances.py: class kernels (2,2|2,0), (2,2|2,1), (2,2|2,2).
#include "../eri_launch_d1.cuh"

namespace lible_b200
{
    cudaError_t launch_d1_05_03(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<2,2,2,0>(a, s, n);
    }
    cudaError_t launch_d1_05_04(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<2,2,2,1>(a, s, n);
    }
    cudaError_t launch_d1_05_05(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<2,2,2,2>(a, s, n);
    }
}
