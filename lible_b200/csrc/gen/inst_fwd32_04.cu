// Generated by gen_instances.py: class kernels with bra pair type (2,1).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    extern const LaunchFn k_fwd32_04[5] = {
        &launchFwd<2,1,0,0,float>,
        &launchFwd<2,1,1,0,float>,
        &launchFwd<2,1,1,1,float>,
        &launchFwd<2,1,2,0,float>,
        &launchFwd<2,1,2,1,float>,
    };
    extern const int u_fwd32_04[5] = {
        workUnit<2,1,0,0,float>(),
        workUnit<2,1,1,0,float>(),
        workUnit<2,1,1,1,float>(),
        workUnit<2,1,2,0,float>(),
        workUnit<2,1,2,1,float>(),
    };
}
