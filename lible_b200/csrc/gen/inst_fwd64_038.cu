// Generated by gen_instances.py: class kernels (5,0|4,0), (5,0|5,0).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    cudaError_t launch_fwd64_11_10(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<5,0,4,0,double>(a, s, n);
    }
    cudaError_t launch_fwd64_11_10_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<5,0,4,0,double>())
            return launchFwd<5,0,4,0,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_11_10_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<5,0,4,0,double>())
            return launchFwd<4,0,5,0,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_11_11(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<5,0,5,0,double>(a, s, n);
    }
    cudaError_t launch_fwd64_11_11_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<5,0,5,0,double>())
            return launchFwd<5,0,5,0,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_11_11_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<5,0,5,0,double>())
            return launchFwd<5,0,5,0,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
}
