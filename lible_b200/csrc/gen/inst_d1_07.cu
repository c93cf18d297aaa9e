// Generated by gen_instances.py: class kernels with bra pair type (3,1).
#include "../eri_launch_d1.cuh"

namespace lible_b200
{
    extern const LaunchFn k_d1_07[8] = {
        &launchD1<3,1,0,0>,
        &launchD1<3,1,1,0>,
        &launchD1<3,1,1,1>,
        &launchD1<3,1,2,0>,
        &launchD1<3,1,2,1>,
        &launchD1<3,1,2,2>,
        &launchD1<3,1,3,0>,
        &launchD1<3,1,3,1>,
    };
}
