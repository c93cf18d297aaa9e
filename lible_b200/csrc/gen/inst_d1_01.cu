// Generated by gen_instances.py: class kernels with bra pair type (1,0).
#include "../eri_launch_d1.cuh"

namespace lible_b200
{
    extern const LaunchFn k_d1_01[2] = {
        &launchD1<1,0,0,0>,
        &launchD1<1,0,1,0>,
    };
}
