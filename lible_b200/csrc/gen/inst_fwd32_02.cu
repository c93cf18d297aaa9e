// Generated by gen_instances.py: class kernels with bra pair type (1,1).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    extern const LaunchFn k_fwd32_02[3] = {
        &launchFwd<1,1,0,0,float>,
        &launchFwd<1,1,1,0,float>,
        &launchFwd<1,1,1,1,float>,
    };
    extern const int u_fwd32_02[3] = {
        workUnit<1,1,0,0,float>(),
        workUnit<1,1,1,0,float>(),
        workUnit<1,1,1,1,float>(),
    };
}
