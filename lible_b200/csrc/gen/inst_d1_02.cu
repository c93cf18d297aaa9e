// Generated by gen_instances.py: class kernels with bra pair type (1,1).
#include "../eri_launch_d1.cuh"

namespace lible_b200
{
    extern const LaunchFn k_d1_02[3] = {
        &launchD1<1,1,0,0>,
        &launchD1<1,1,1,0>,
        &launchD1<1,1,1,1>,
    };
}
