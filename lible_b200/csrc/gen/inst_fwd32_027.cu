// Generated by gen_instances.py: class kernels (3,3|3,3).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    cudaError_t launch_fwd32_09_09(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<3,3,3,3,float>(a, s, n);
    }
    cudaError_t launch_fwd32_09_09_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<3,3,3,3,float>())
            return launchFwd<3,3,3,3,float,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd32_09_09_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<3,3,3,3,float>())
            return launchFwd<3,3,3,3,float>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
}
