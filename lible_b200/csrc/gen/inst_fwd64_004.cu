// Generated by gen_instances.py: class kernels (2,0|1,1), (2,0|2,0).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    cudaError_t launch_fwd64_03_02(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<2,0,1,1,double>(a, s, n);
    }
    cudaError_t launch_fwd64_03_02_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<2,0,1,1,double>())
            return launchFwd<2,0,1,1,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_03_02_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<2,0,1,1,double>())
            return launchFwd<1,1,2,0,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_03_03(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<2,0,2,0,double>(a, s, n);
    }
    cudaError_t launch_fwd64_03_03_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<2,0,2,0,double>())
            return launchFwd<2,0,2,0,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_03_03_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<2,0,2,0,double>())
            return launchFwd<2,0,2,0,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
}
