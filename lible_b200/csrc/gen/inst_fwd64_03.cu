// Generated by gen_instances.py: class kernels with bra pair type (2,0).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    extern const LaunchFn k_fwd64_03[4] = {
        &launchFwd<2,0,0,0,double>,
        &launchFwd<2,0,1,0,double>,
        &launchFwd<2,0,1,1,double>,
        &launchFwd<2,0,2,0,double>,
    };
    extern const int u_fwd64_03[4] = {
        workUnit<2,0,0,0,double>(),
        workUnit<2,0,1,0,double>(),
        workUnit<2,0,1,1,double>(),
        workUnit<2,0,2,0,double>(),
    };
}
