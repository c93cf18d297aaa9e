// The dispatch table that maps a quartet class to its kernel instantiation (launch wrappers:
// eri_launch_fwd.cuh and eri_launch_d1.cuh, included by the generated instantiation files only).
#pragma once

#include "device_common.cuh"

namespace lible_b200
{
    using LaunchFn = cudaError_t (*)(const QuartetArgs &, cudaStream_t, int num_sms);

    // Pair types in canonical order; a quartet class is instantiated with the larger type in the
    // bra.  Index: la*(la+1)/2 + lb for la <= 3, then (4,0) -> 10, (5,0) -> 11.
    constexpr int kNumPairTypes = 12;
    inline int pairType(int la, int lb)
    {
        if (la <= 3)
            return la * (la + 1) / 2 + lb;
        return la == 4 ? 10 : 11;
    }

    // Implemented by the generated instantiation files.
    // `shape` selects the tile-shape variant of the forward class kernels (0 default, 1 the
    // alternative of Shape<..., 1>); variant 1 is null where it equals the default.
    LaunchFn lookupFwd64(int bra_type, int ket_type, int shape = 0);
    LaunchFn lookupFwd32(int bra_type, int ket_type, int shape = 0);
    LaunchFn lookupD1(int bra_type, int ket_type);
    int unitFwd(int bra_type, int ket_type, bool fp32, int shape = 0);
    bool hasFwdVariant(int bra_type, int ket_type, bool fp32, int shape = 1);
}
