// Generated by gen_instances.py: class kernels (1,1|1,0), (1,1|1,1).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    cudaError_t launch_fwd64_02_01(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<1,1,1,0,double>(a, s, n);
    }
    cudaError_t launch_fwd64_02_01_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<1,1,1,0,double>())
            return launchFwd<1,1,1,0,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_02_01_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<1,1,1,0,double>())
            return launchFwd<1,0,1,1,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_02_02(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<1,1,1,1,double>(a, s, n);
    }
    cudaError_t launch_fwd64_02_02_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<1,1,1,1,double>())
            return launchFwd<1,1,1,1,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_02_02_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<1,1,1,1,double>())
            return launchFwd<1,1,1,1,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
}
