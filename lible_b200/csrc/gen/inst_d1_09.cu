// Generated by gen_instances.py: class kernels with bra pair type (3,3).
#include "../eri_launch_d1.cuh"

namespace lible_b200
{
    extern const LaunchFn k_d1_09[10] = {
        &launchD1<3,3,0,0>,
        &launchD1<3,3,1,0>,
        &launchD1<3,3,1,1>,
        &launchD1<3,3,2,0>,
        &launchD1<3,3,2,1>,
        &launchD1<3,3,2,2>,
        &launchD1<3,3,3,0>,
        &launchD1<3,3,3,1>,
        &launchD1<3,3,3,2>,
        &launchD1<3,3,3,3>,
    };
}
