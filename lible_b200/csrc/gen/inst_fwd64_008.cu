// Generated by gen_instances.py: class kernels (2,2|1,0), (2,2|1,1).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    cudaError_t launch_fwd64_05_01(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<2,2,1,0,double>(a, s, n);
    }
    cudaError_t launch_fwd64_05_02(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<2,2,1,1,double>(a, s, n);
    }
}
