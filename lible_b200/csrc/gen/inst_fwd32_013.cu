// Generated by gen_instances.py: class kernels (3,0|2,2), (3,0|3,0).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    cudaError_t launch_fwd32_06_05(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<3,0,2,2,float>(a, s, n);
    }
    cudaError_t launch_fwd32_06_05_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<3,0,2,2,float>())
            return launchFwd<3,0,2,2,float,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd32_06_05_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<3,0,2,2,float>())
            return launchFwd<2,2,3,0,float>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd32_06_06(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<3,0,3,0,float>(a, s, n);
    }
    cudaError_t launch_fwd32_06_06_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<3,0,3,0,float>())
            return launchFwd<3,0,3,0,float,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd32_06_06_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<3,0,3,0,float>())
            return launchFwd<3,0,3,0,float>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
}
