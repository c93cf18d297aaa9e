// Generated by gen_instances.py: class kernels (2,0|1,1), (2,0|2,0).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    cudaError_t launch_fwd64_03_02(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<2,0,1,1,double>(a, s, n);
    }
    cudaError_t launch_fwd64_03_03(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<2,0,2,0,double>(a, s, n);
    }
}
