// Generated by gen_instances.py: class kernels (5,0|3,2), (5,0|3,3).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    cudaError_t launch_fwd64_11_08(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<5,0,3,2,double>(a, s, n);
    }
    cudaError_t launch_fwd64_11_08_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<5,0,3,2,double>())
            return launchFwd<5,0,3,2,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_11_08_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<5,0,3,2,double>())
            return launchFwd<3,2,5,0,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_11_09(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<5,0,3,3,double>(a, s, n);
    }
    cudaError_t launch_fwd64_11_09_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<5,0,3,3,double>())
            return launchFwd<5,0,3,3,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_11_09_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<5,0,3,3,double>())
            return launchFwd<3,3,5,0,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
}
