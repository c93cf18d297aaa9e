// Generated by gen_instances.py: class kernels with bra pair type (3,3).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    extern const LaunchFn k_fwd32_09[10] = {
        &launchFwd<3,3,0,0,float>,
        &launchFwd<3,3,1,0,float>,
        &launchFwd<3,3,1,1,float>,
        &launchFwd<3,3,2,0,float>,
        &launchFwd<3,3,2,1,float>,
        &launchFwd<3,3,2,2,float>,
        &launchFwd<3,3,3,0,float>,
        &launchFwd<3,3,3,1,float>,
        &launchFwd<3,3,3,2,float>,
        &launchFwd<3,3,3,3,float>,
    };
    extern const int u_fwd32_09[10] = {
        workUnit<3,3,0,0,float>(),
        workUnit<3,3,1,0,float>(),
        workUnit<3,3,1,1,float>(),
        workUnit<3,3,2,0,float>(),
        workUnit<3,3,2,1,float>(),
        workUnit<3,3,2,2,float>(),
        workUnit<3,3,3,0,float>(),
        workUnit<3,3,3,1,float>(),
        workUnit<3,3,3,2,float>(),
        workUnit<3,3,3,3,float>(),
    };
}
