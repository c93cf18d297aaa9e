// Generated by gen_instances.py: class kernels (4,0|3,1), (4,0|3,2).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    cudaError_t launch_fwd64_10_07(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<4,0,3,1,double>(a, s, n);
    }
    cudaError_t launch_fwd64_10_07_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<4,0,3,1,double>())
            return launchFwd<4,0,3,1,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_10_07_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<4,0,3,1,double>())
            return launchFwd<3,1,4,0,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_10_08(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<4,0,3,2,double>(a, s, n);
    }
    cudaError_t launch_fwd64_10_08_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<4,0,3,2,double>())
            return launchFwd<4,0,3,2,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_10_08_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<4,0,3,2,double>())
            return launchFwd<3,2,4,0,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
}
