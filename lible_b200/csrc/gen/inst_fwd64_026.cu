// Generated by gen_instances.py: class kernels (3,3|3,1), (3,3|3,2).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    cudaError_t launch_fwd64_09_07(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<3,3,3,1,double>(a, s, n);
    }
    cudaError_t launch_fwd64_09_07_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<3,3,3,1,double>())
            return launchFwd<3,3,3,1,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_09_07_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<3,3,3,1,double>())
            return launchFwd<3,1,3,3,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_09_08(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<3,3,3,2,double>(a, s, n);
    }
    cudaError_t launch_fwd64_09_08_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<3,3,3,2,double>())
            return launchFwd<3,3,3,2,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_09_08_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<3,3,3,2,double>())
            return launchFwd<3,2,3,3,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
}
