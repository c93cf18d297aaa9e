// Generated by gen_instances.py: class kernels with bra pair type (0,0).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    extern const LaunchFn k_fwd32_00[1] = {
        &launchFwd<0,0,0,0,float>,
    };
    extern const int u_fwd32_00[1] = {
        workUnit<0,0,0,0,float>(),
    };
}
