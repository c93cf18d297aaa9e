// Generated by gen_instances.py: class kernels with bra pair type (1,0).
#include "../eri_launch_fwd.cuh"

namespace lible_b200
{
    extern const LaunchFn k_fwd64_01[2] = {
        &launchFwd<1,0,0,0,double>,
        &launchFwd<1,0,1,0,double>,
    };
    extern const int u_fwd64_01[2] = {
        workUnit<1,0,0,0,double>(),
        workUnit<1,0,1,0,double>(),
    };
}
