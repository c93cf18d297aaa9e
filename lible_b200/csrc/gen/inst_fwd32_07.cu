// Generated by gen_instances.py: class kernels with bra pair type (3,1).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    extern const LaunchFn k_fwd32_07[8] = {
        &launchFwd<3,1,0,0,float>,
        &launchFwd<3,1,1,0,float>,
        &launchFwd<3,1,1,1,float>,
        &launchFwd<3,1,2,0,float>,
        &launchFwd<3,1,2,1,float>,
        &launchFwd<3,1,2,2,float>,
        &launchFwd<3,1,3,0,float>,
        &launchFwd<3,1,3,1,float>,
    };
    extern const int u_fwd32_07[8] = {
        workUnit<3,1,0,0,float>(),
        workUnit<3,1,1,0,float>(),
        workUnit<3,1,1,1,float>(),
        workUnit<3,1,2,0,float>(),
        workUnit<3,1,2,1,float>(),
        workUnit<3,1,2,2,float>(),
        workUnit<3,1,3,0,float>(),
        workUnit<3,1,3,1,float>(),
    };
}
