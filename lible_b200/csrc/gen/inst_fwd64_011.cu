// Generated by gen_instances.py: class kernels (3,0|1,0), (3,0|1,1).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    cudaError_t launch_fwd64_06_01(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<3,0,1,0,double>(a, s, n);
    }
    cudaError_t launch_fwd64_06_01_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<3,0,1,0,double>())
            return launchFwd<3,0,1,0,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_06_01_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<3,0,1,0,double>())
            return launchFwd<1,0,3,0,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_06_02(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<3,0,1,1,double>(a, s, n);
    }
    cudaError_t launch_fwd64_06_02_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<3,0,1,1,double>())
            return launchFwd<3,0,1,1,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_06_02_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<3,0,1,1,double>())
            return launchFwd<1,1,3,0,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
}
