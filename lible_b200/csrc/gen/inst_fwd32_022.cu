// Generated by gen_instances.py: class kernels (3,2|3,2), (3,3|0,0).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    cudaError_t launch_fwd32_08_08(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<3,2,3,2,float>(a, s, n);
    }
    cudaError_t launch_fwd32_08_08_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<3,2,3,2,float>())
            return launchFwd<3,2,3,2,float,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd32_08_08_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<3,2,3,2,float>())
            return launchFwd<3,2,3,2,float>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd32_09_00(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<3,3,0,0,float>(a, s, n);
    }
    cudaError_t launch_fwd32_09_00_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<3,3,0,0,float>())
            return launchFwd<3,3,0,0,float,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd32_09_00_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<3,3,0,0,float>())
            return launchFwd<0,0,3,3,float>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
}
