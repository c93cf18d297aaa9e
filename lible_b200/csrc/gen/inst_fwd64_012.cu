// Generated by gen_instances.py: class kernels (3,0|2,0), (3,0|2,1).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    cudaError_t launch_fwd64_06_03(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<3,0,2,0,double>(a, s, n);
    }
    cudaError_t launch_fwd64_06_04(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<3,0,2,1,double>(a, s, n);
    }
}
