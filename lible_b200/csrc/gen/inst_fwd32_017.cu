// Generated by gen_instances.py: class kernels (3,1|3,0), (3,1|3,1).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    cudaError_t launch_fwd32_07_06(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<3,1,3,0,float>(a, s, n);
    }
    cudaError_t launch_fwd32_07_06_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<3,1,3,0,float>())
            return launchFwd<3,1,3,0,float,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd32_07_06_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<3,1,3,0,float>())
            return launchFwd<3,0,3,1,float>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd32_07_07(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<3,1,3,1,float>(a, s, n);
    }
    cudaError_t launch_fwd32_07_07_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<3,1,3,1,float>())
            return launchFwd<3,1,3,1,float,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd32_07_07_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<3,1,3,1,float>())
            return launchFwd<3,1,3,1,float>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
}
