// Generated by gen_instances.py: class kernels with bra pair type (3,0).
#include "../eri_launch_d1.cuh"

namespace lible_b200
{
    extern const LaunchFn k_d1_06[7] = {
        &launchD1<3,0,0,0>,
        &launchD1<3,0,1,0>,
        &launchD1<3,0,1,1>,
        &launchD1<3,0,2,0>,
        &launchD1<3,0,2,1>,
        &launchD1<3,0,2,2>,
        &launchD1<3,0,3,0>,
    };
}
