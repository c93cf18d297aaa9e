// Generated by gen_instances.py: class kernels (2,2|2,2), (3,0|0,0).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    cudaError_t launch_fwd64_05_05(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<2,2,2,2,double>(a, s, n);
    }
    cudaError_t launch_fwd64_05_05_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<2,2,2,2,double>())
            return launchFwd<2,2,2,2,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_05_05_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<2,2,2,2,double>())
            return launchFwd<2,2,2,2,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_06_00(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<3,0,0,0,double>(a, s, n);
    }
    cudaError_t launch_fwd64_06_00_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<3,0,0,0,double>())
            return launchFwd<3,0,0,0,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_06_00_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<3,0,0,0,double>())
            return launchFwd<0,0,3,0,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
}
