// Generated by gen_instances.py: class kernels with bra pair type (3,3).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    extern const LaunchFn k_fwd64_09[10] = {
        &launchFwd<3,3,0,0,double>,
        &launchFwd<3,3,1,0,double>,
        &launchFwd<3,3,1,1,double>,
        &launchFwd<3,3,2,0,double>,
        &launchFwd<3,3,2,1,double>,
        &launchFwd<3,3,2,2,double>,
        &launchFwd<3,3,3,0,double>,
        &launchFwd<3,3,3,1,double>,
        &launchFwd<3,3,3,2,double>,
        &launchFwd<3,3,3,3,double>,
    };
    extern const int u_fwd64_09[10] = {
        workUnit<3,3,0,0,double>(),
        workUnit<3,3,1,0,double>(),
        workUnit<3,3,1,1,double>(),
        workUnit<3,3,2,0,double>(),
        workUnit<3,3,2,1,double>(),
        workUnit<3,3,2,2,double>(),
        workUnit<3,3,3,0,double>(),
        workUnit<3,3,3,1,double>(),
        workUnit<3,3,3,2,double>(),
        workUnit<3,3,3,3,double>(),
    };
}
