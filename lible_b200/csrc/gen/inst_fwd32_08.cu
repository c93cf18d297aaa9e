// Generated by gen_instances.py: class kernels with bra pair type (3,2).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    extern const LaunchFn k_fwd32_08[9] = {
        &launchFwd<3,2,0,0,float>,
        &launchFwd<3,2,1,0,float>,
        &launchFwd<3,2,1,1,float>,
        &launchFwd<3,2,2,0,float>,
        &launchFwd<3,2,2,1,float>,
        &launchFwd<3,2,2,2,float>,
        &launchFwd<3,2,3,0,float>,
        &launchFwd<3,2,3,1,float>,
        &launchFwd<3,2,3,2,float>,
    };
    extern const int u_fwd32_08[9] = {
        workUnit<3,2,0,0,float>(),
        workUnit<3,2,1,0,float>(),
        workUnit<3,2,1,1,float>(),
        workUnit<3,2,2,0,float>(),
        workUnit<3,2,2,1,float>(),
        workUnit<3,2,2,2,float>(),
        workUnit<3,2,3,0,float>(),
        workUnit<3,2,3,1,float>(),
        workUnit<3,2,3,2,float>(),
    };
}
