// Generated by gen_instances.py: class kernels with bra pair type (4,0).
#include "../eri_launch_d1.cuh"

namespace lible_b200
{
    extern const LaunchFn k_d1_10[11] = {
        &launchD1<4,0,0,0>,
        &launchD1<4,0,1,0>,
        &launchD1<4,0,1,1>,
        &launchD1<4,0,2,0>,
        &launchD1<4,0,2,1>,
        &launchD1<4,0,2,2>,
        &launchD1<4,0,3,0>,
        &launchD1<4,0,3,1>,
        &launchD1<4,0,3,2>,
        &launchD1<4,0,3,3>,
        &launchD1<4,0,4,0>,
    };
}
