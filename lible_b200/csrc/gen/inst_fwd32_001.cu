// Generated by gen_instances.py: class kernels (1,0|1,0), (1,1|0,0).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    cudaError_t launch_fwd32_01_01(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<1,0,1,0,float>(a, s, n);
    }
    cudaError_t launch_fwd32_01_01_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<1,0,1,0,float>())
            return launchFwd<1,0,1,0,float,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd32_01_01_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<1,0,1,0,float>())
            return launchFwd<1,0,1,0,float>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd32_02_00(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<1,1,0,0,float>(a, s, n);
    }
    cudaError_t launch_fwd32_02_00_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<1,1,0,0,float>())
            return launchFwd<1,1,0,0,float,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd32_02_00_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<1,1,0,0,float>())
            return launchFwd<0,0,1,1,float>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
}
