// Generated by gen_instances.py: class kernels (2,1|2,1), (2,2|0,0).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    cudaError_t launch_fwd32_04_04(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<2,1,2,1,float>(a, s, n);
    }
    cudaError_t launch_fwd32_04_04_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<2,1,2,1,float>())
            return launchFwd<2,1,2,1,float,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd32_04_04_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<2,1,2,1,float>())
            return launchFwd<2,1,2,1,float>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd32_05_00(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<2,2,0,0,float>(a, s, n);
    }
    cudaError_t launch_fwd32_05_00_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<2,2,0,0,float>())
            return launchFwd<2,2,0,0,float,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd32_05_00_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<2,2,0,0,float>())
            return launchFwd<0,0,2,2,float>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
}
