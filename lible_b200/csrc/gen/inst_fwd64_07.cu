// Generated by gen_instances.py: class kernels with bra pair type (3,1).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    extern const LaunchFn k_fwd64_07[8] = {
        &launchFwd<3,1,0,0,double>,
        &launchFwd<3,1,1,0,double>,
        &launchFwd<3,1,1,1,double>,
        &launchFwd<3,1,2,0,double>,
        &launchFwd<3,1,2,1,double>,
        &launchFwd<3,1,2,2,double>,
        &launchFwd<3,1,3,0,double>,
        &launchFwd<3,1,3,1,double>,
    };
    extern const int u_fwd64_07[8] = {
        workUnit<3,1,0,0,double>(),
        workUnit<3,1,1,0,double>(),
        workUnit<3,1,1,1,double>(),
        workUnit<3,1,2,0,double>(),
        workUnit<3,1,2,1,double>(),
        workUnit<3,1,2,2,double>(),
        workUnit<3,1,3,0,double>(),
        workUnit<3,1,3,1,double>(),
    };
}
