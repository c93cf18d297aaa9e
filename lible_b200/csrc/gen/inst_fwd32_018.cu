// Generated by gen_instances.py: class kernels (3,2|0,0), (3,2|1,0).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    cudaError_t launch_fwd32_08_00(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<3,2,0,0,float>(a, s, n);
    }
    cudaError_t launch_fwd32_08_00_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<3,2,0,0,float>())
            return launchFwd<3,2,0,0,float,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd32_08_00_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<3,2,0,0,float>())
            return launchFwd<0,0,3,2,float>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd32_08_01(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<3,2,1,0,float>(a, s, n);
    }
    cudaError_t launch_fwd32_08_01_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<3,2,1,0,float>())
            return launchFwd<3,2,1,0,float,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd32_08_01_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<3,2,1,0,float>())
            return launchFwd<1,0,3,2,float>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
}
