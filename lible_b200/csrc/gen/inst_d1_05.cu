// Generated by gen_instances.py: class kernels with bra pair type (2,2).
#include "../eri_launch_d1.cuh"

namespace lible_b200
{
    extern const LaunchFn k_d1_05[6] = {
        &launchD1<2,2,0,0>,
        &launchD1<2,2,1,0>,
        &launchD1<2,2,1,1>,
        &launchD1<2,2,2,0>,
        &launchD1<2,2,2,1>,
        &launchD1<2,2,2,2>,
    };
}
