// Generated by gen_instances.py: class kernels with bra pair type (4,0).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    extern const LaunchFn k_fwd64_10[11] = {
        &launchFwd<4,0,0,0,double>,
        &launchFwd<4,0,1,0,double>,
        &launchFwd<4,0,1,1,double>,
        &launchFwd<4,0,2,0,double>,
        &launchFwd<4,0,2,1,double>,
        &launchFwd<4,0,2,2,double>,
        &launchFwd<4,0,3,0,double>,
        &launchFwd<4,0,3,1,double>,
        &launchFwd<4,0,3,2,double>,
        &launchFwd<4,0,3,3,double>,
        &launchFwd<4,0,4,0,double>,
    };
    extern const int u_fwd64_10[11] = {
        workUnit<4,0,0,0,double>(),
        workUnit<4,0,1,0,double>(),
        workUnit<4,0,1,1,double>(),
        workUnit<4,0,2,0,double>(),
        workUnit<4,0,2,1,double>(),
        workUnit<4,0,2,2,double>(),
        workUnit<4,0,3,0,double>(),
        workUnit<4,0,3,1,double>(),
        workUnit<4,0,3,2,double>(),
        workUnit<4,0,3,3,double>(),
        workUnit<4,0,4,0,double>(),
    };
}
