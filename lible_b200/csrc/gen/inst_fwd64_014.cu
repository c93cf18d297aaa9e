// Generated by gen_instances.py: class kernels (3,1|0,0), (3,1|1,0).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    cudaError_t launch_fwd64_07_00(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<3,1,0,0,double>(a, s, n);
    }
    cudaError_t launch_fwd64_07_00_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<3,1,0,0,double>())
            return launchFwd<3,1,0,0,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_07_00_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<3,1,0,0,double>())
            return launchFwd<0,0,3,1,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_07_01(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<3,1,1,0,double>(a, s, n);
    }
    cudaError_t launch_fwd64_07_01_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<3,1,1,0,double>())
            return launchFwd<3,1,1,0,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_07_01_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<3,1,1,0,double>())
            return launchFwd<1,0,3,1,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
}
