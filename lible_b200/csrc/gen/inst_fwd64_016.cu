// Generated by gen_instances.py: class kernels (3,1|2,1), (3,1|2,2).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    cudaError_t launch_fwd64_07_04(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<3,1,2,1,double>(a, s, n);
    }
    cudaError_t launch_fwd64_07_04_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<3,1,2,1,double>())
            return launchFwd<3,1,2,1,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_07_04_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<3,1,2,1,double>())
            return launchFwd<2,1,3,1,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_07_05(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<3,1,2,2,double>(a, s, n);
    }
    cudaError_t launch_fwd64_07_05_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<3,1,2,2,double>())
            return launchFwd<3,1,2,2,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_07_05_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<3,1,2,2,double>())
            return launchFwd<2,2,3,1,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
}
