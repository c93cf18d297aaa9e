// Generated by gen_instances.py: class kernels (2,2|1,0), (2,2|1,1).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    cudaError_t launch_fwd64_05_01(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<2,2,1,0,double>(a, s, n);
    }
    cudaError_t launch_fwd64_05_01_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<2,2,1,0,double>())
            return launchFwd<2,2,1,0,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_05_01_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<2,2,1,0,double>())
            return launchFwd<1,0,2,2,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_05_02(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<2,2,1,1,double>(a, s, n);
    }
    cudaError_t launch_fwd64_05_02_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<2,2,1,1,double>())
            return launchFwd<2,2,1,1,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_05_02_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<2,2,1,1,double>())
            return launchFwd<1,1,2,2,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
}
