// Generated by gen_instances.py: class kernels (3,3|3,0), (3,3|3,1), (3,3|3,2).
#include "../eri_launch_d1.cuh"

namespace lible_b200
{
    cudaError_t launch_d1_09_06(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<3,3,3,0>(a, s, n);
    }
    cudaError_t launch_d1_09_07(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<3,3,3,1>(a, s, n);
    }
    cudaError_t launch_d1_09_08(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchD1<3,3,3,2>(a, s, n);
    }
}
