// Generated by gen_instances.py: class kernels (4,0|3,3), (4,0|4,0).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    cudaError_t launch_fwd64_10_09(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<4,0,3,3,double>(a, s, n);
    }
    cudaError_t launch_fwd64_10_09_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<4,0,3,3,double>())
            return launchFwd<4,0,3,3,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_10_09_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<4,0,3,3,double>())
            return launchFwd<3,3,4,0,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_10_10(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<4,0,4,0,double>(a, s, n);
    }
    cudaError_t launch_fwd64_10_10_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<4,0,4,0,double>())
            return launchFwd<4,0,4,0,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_10_10_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<4,0,4,0,double>())
            return launchFwd<4,0,4,0,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
}
