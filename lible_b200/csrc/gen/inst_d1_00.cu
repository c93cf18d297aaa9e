// Generated by gen_instances.py: class kernels with bra pair type (0,0).
#include "../eri_launch_d1.cuh"

namespace lible_b200
{
    extern const LaunchFn k_d1_00[1] = {
        &launchD1<0,0,0,0>,
    };
}
