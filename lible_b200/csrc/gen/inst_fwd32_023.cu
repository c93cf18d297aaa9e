// Generated by gen_instances.py: class kernels (3,3|1,0), (3,3|1,1).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    cudaError_t launch_fwd32_09_01(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<3,3,1,0,float>(a, s, n);
    }
    cudaError_t launch_fwd32_09_01_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<3,3,1,0,float>())
            return launchFwd<3,3,1,0,float,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd32_09_01_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<3,3,1,0,float>())
            return launchFwd<1,0,3,3,float>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd32_09_02(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<3,3,1,1,float>(a, s, n);
    }
    cudaError_t launch_fwd32_09_02_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<3,3,1,1,float>())
            return launchFwd<3,3,1,1,float,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd32_09_02_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<3,3,1,1,float>())
            return launchFwd<1,1,3,3,float>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
}
