// Generated by gen_instances.py: class kernels (3,3|2,0), (3,3|2,1).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    cudaError_t launch_fwd64_09_03(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<3,3,2,0,double>(a, s, n);
    }
    cudaError_t launch_fwd64_09_03_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<3,3,2,0,double>())
            return launchFwd<3,3,2,0,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_09_03_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<3,3,2,0,double>())
            return launchFwd<2,0,3,3,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_09_04(const QuartetArgs &a, cudaStream_t s, int n)
    {
        return launchFwd<3,3,2,1,double>(a, s, n);
    }
    cudaError_t launch_fwd64_09_04_v1(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasShapeVariant<3,3,2,1,double>())
            return launchFwd<3,3,2,1,double,1>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t launch_fwd64_09_04_f(const QuartetArgs &a, cudaStream_t s, int n)
    {
        if constexpr (hasFlippedShape<3,3,2,1,double>())
            return launchFwd<2,1,3,3,double>(a, s, n);
        else
            return cudaErrorNotSupported;
    }
}
