// The quartet-class kernel family: one instantiation per angular-momentum class
// (la lb | lc ld), computing contracted shell-quartet batches in the SHARK form
//     (ab|cd) = sum_p sum_q E_ab[p] . R_pq . E_cd[q]^T
// (src/lible/ints/twoel/eri_kernel_funs.hpp:104-193) and consuming them in a fused epilogue
// (store, J/K digestion, RI-J).  Three- and two-centre integrals use the same kernels: an
// auxiliary shell is a "pair" whose second member is a unit s function of exponent 0.
//
// Two execution shapes, chosen per class at compile time:
//  * G = 1  (small classes): one thread owns a whole contracted quartet; R, R.E and the batch live
//    in registers and every index is a compile-time constant.
//  * G = 32*W (larger classes): a group of W warps owns one quartet; the R recursion, the signed
//    R matrix and the staged E tiles live in shared memory and the two contractions are split
//    over the group's threads.
#pragma once

#include "device_common.cuh"

namespace lible_b200
{
    // Register-path group size: the smallest g dividing S_cd (g <= 32) for which one thread's share
    // of the batch (S_ab x S_cd/g), of R.E (H_ab x S_cd/g) and the R vector fit `budget` values; 0
    // when none does.
    constexpr int pickRegGroupWithin(int sab, int scd, int hab, int nr, int budget)
    {
        for (int g = 1; g <= 32; g++)
            if (scd % g == 0 && sab * (scd / g) + hab * (scd / g) + nr <= budget)
                return g;
        return 0;
    }
    // Two tiers per arithmetic type: a share that fits the register file without spilling (104
    // doubles / 200 floats) is preferred; failing that, a moderate overflow (144 / 288 values, a few
    // hundred bytes of spills) still beats one quartet per warp on the group path; a third budget
    // (170 / 340) is open to whole quartets per thread only; beyond that the class uses the group
    // path (0).
    template <typename T>
    constexpr int pickRegGroup(int sab, int scd, int hab, int nr)
    {
        constexpr int tier1 = sizeof(T) == 8 ? 104 : 200, tier2 = sizeof(T) == 8 ? 144 : 288;
        const int g = pickRegGroupWithin(sab, scd, hab, nr, tier1);
        const int g2 = g ? g : pickRegGroupWithin(sab, scd, hab, nr, tier2);
        return g2 ? g2 : (sab * scd + hab * scd + nr <= (sizeof(T) == 8 ? 170 : 340) ? 1 : 0);
    }

    // Shared-memory pitches (in doubles) of the DMMA operand tiles.  Fragments read either 4 rows x 8
    // consecutive elements (k-major: R, E_ket, R.E) or 8 rows x 4 (m-major: E_bra); a pitch of 8
    // (resp. 4) modulo 16 spreads those rows over all 32 banks.
    constexpr int kPitch(int x)
    {
        const int p = (x + 7) / 8 * 8;
        return p % 16 == 0 ? p + 8 : p;
    }
    constexpr int mPitch(int x)
    {
        int p = (x + 3) / 4 * 4;
        while (p % 16 != 4)
            p += 4;
        return p;
    }

    // The alternative register-path group of shape variant 1: the next divisor of S_cd above g0 (more
    // threads per quartet, fewer values per thread); g0 itself when there is none.
    constexpr int altRegGroup(int scd, int g0)
    {
        if (g0 == 0)
            return 0;
        for (int g = g0 + 1; g <= 32 && g <= scd; g++)
            if (scd % g == 0)
                return g;
        return g0;
    }

    // Tile shape of a class kernel.  Shape variant SV = 0 is the default; SV = 1 is the alternative
    // the launch autotuner times against it: twice the warps per quartet on the group paths (each
    // warp owning fewer output tiles), the next larger thread group on the register path, and the
    // default register bound for the classes compiled with a raised occupancy bound.
    template <int LA, int LB, int LC, int LD, typename T, int SV = 0>
    struct Shape
    {
        using C = Cls<LA, LB, LC, LD>;
        // register path: GT threads per quartet, each owning CW consecutive ket columns
        static constexpr int GT0 = pickRegGroup<T>(C::SAB, C::SCD, C::HAB, C::NR);
        static constexpr int GT = SV == 0 ? GT0 : altRegGroup(C::SCD, GT0);
        static constexpr int CW = GT ? C::SCD / GT : 0;
        static constexpr int QPW = GT ? 32 / GT : 0;           // quartets per warp
        // group path in FP64: both contractions on the DMMA pipe (mma.m8n8k4.f64) in 8x8 tiles of
        // R.E_ket^T [H_ab x S_cd] (K = H_cd) and of the batch [S_ab x S_cd] (K = H_ab)
        static constexpr bool MMA = GT == 0 && sizeof(T) == 8;
        static constexpr int MT = (C::HAB + 7) / 8, NT = (C::SCD + 7) / 8, KT = (C::HCD + 3) / 4;
        static constexpr int MT2 = (C::SAB + 7) / 8, KT2 = (C::HAB + 3) / 4;
        static constexpr int TILES = MT * NT, TILES2 = MT2 * NT;
        static constexpr int WM0 = (TILES + 5) / 6 < 1 ? 1 : ((TILES + 5) / 6 > 8 ? 8 : (TILES + 5) / 6);
        static constexpr int WM1 = 2 * WM0 > 8 ? 8 : (2 * WM0 > TILES ? (TILES > WM0 ? TILES : WM0) : 2 * WM0);
        static constexpr int WM = SV == 0 ? WM0 : WM1;
        static constexpr int TPW = (TILES + WM - 1) / WM, TPW2 = (TILES2 + WM - 1) / WM;
        static constexpr int P_RM = kPitch(C::HAB), P_EC = kPitch(C::SCD), P_EA = mPitch(C::HAB);
        static constexpr size_t a16(size_t x) { return (x + 15) / 16 * 16; }
        static constexpr size_t m_off_rb = 0;                                            // 2 x NR
        static constexpr size_t m_off_rm = a16(m_off_rb + 8 * 2 * C::NR);                // KT*4 x P_RM
        static constexpr size_t m_off_ec = a16(m_off_rm + 8 * (size_t)KT * 4 * P_RM);    // KT*4 x P_EC
        static constexpr size_t m_off_ea = a16(m_off_ec + 8 * (size_t)KT * 4 * P_EC);    // MT2*8 x P_EA
        static constexpr size_t m_off_rx = a16(m_off_ea + 8 * (size_t)MT2 * 8 * P_EA);   // MT*8 x P_EC
        static constexpr size_t m_off_ix = a16(m_off_rx + 8 * (size_t)MT * 8 * P_EC);    // HCD x HAB int16
        static constexpr size_t m_off_ht = a16(m_off_ix + 2 * C::HCD * C::HAB);          // NR char4
        static constexpr size_t m_off_mb = a16(m_off_ht + 4 * C::NR);                    // mbarrier
        static constexpr size_t m_off_tb = m_off_mb + 16;                                // decoded tasks
        static constexpr size_t m_smem = m_off_tb + sizeof(GroupTask) * kGroupTaskBatch;
        // bytes of one padded ket E tile (KT*4 rows of P_EC doubles), the unit of the bulk copy
        static constexpr unsigned ec_tile_bytes = 8u * KT * 4 * P_EC;
        static constexpr int W0 = ((C::HAB * C::SCD + C::SAB * C::SCD) <= 64 * 32)    ? 1
                                  : ((C::HAB * C::SCD + C::SAB * C::SCD) <= 64 * 64)  ? 2
                                  : ((C::HAB * C::SCD + C::SAB * C::SCD) <= 64 * 128) ? 4
                                                                                       : 8;
        static constexpr int W = GT ? 0 : MMA ? WM : (SV == 0 ? W0 : (2 * W0 > 8 ? 8 : 2 * W0));
        static constexpr int G = W == 0 ? 1 : 32 * W;
        static constexpr int block = W == 0 ? 128 : G;
        // register path: per-warp staging of finished batches for the digestion epilogue
        static constexpr size_t reg_smem = (GT > 1) ? sizeof(double) * (block / 32) * QPW * C::SAB * C::SCD : 0;
        // register path: the order-L Boys table, staged once per block
        static constexpr size_t off_boys = (reg_smem + 15) / 16 * 16;
        static constexpr size_t boys_bytes = sizeof(T) == 8 ? sizeof(double) * kBoysTerms * kBoysPitch
                                                            : sizeof(float) * (C::L + kBoysTermsF) * kBoysPitch;
        static constexpr int IK = W == 0 ? 0 : (C::HAB * C::SCD + G - 1) / G;
        static constexpr int IB = W == 0 ? 0 : (C::SAB * C::SCD + G - 1) / G;
        // shared-memory carve-up (bytes) for the group shape
        static constexpr size_t off_rb = 0;                                          // 2 x NR of T
        static constexpr size_t off_rm = off_rb + sizeof(T) * 2 * C::NR;            // HCD x HAB
        static constexpr size_t off_ec = off_rm + sizeof(T) * C::HCD * C::HAB;      // HCD x SCD
        static constexpr size_t off_ea = off_ec + sizeof(T) * C::HCD * C::SCD;      // SAB x HAB
        static constexpr size_t off_rx = off_ea + sizeof(T) * C::SAB * C::HAB;      // HAB x SCD
        static constexpr size_t off_ix = off_rx + sizeof(T) * C::HAB * C::SCD;      // HCD x HAB int16
        static constexpr size_t off_ht = (off_ix + 2 * C::HCD * C::HAB + 15) / 16 * 16; // NR char4
        static constexpr size_t smem = W == 0 ? off_boys + boys_bytes : MMA ? m_smem : off_ht + 4 * C::NR;
        static_assert(!MMA || m_smem <= 227 * 1024, "DMMA shared-memory layout exceeds 227 KB");
    };

    // ---------------------------------------------------------------------------------------
    // Bulk asynchronous copies (the TMA engine's 1-D form, cp.async.bulk) into shared memory,
    // completed on an mbarrier.  Addresses and sizes are multiples of 16 bytes.
    __device__ __forceinline__ void mbarInit(uint64_t *mbar)
    {
        const unsigned a = (unsigned)__cvta_generic_to_shared(mbar);
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }

    // One thread: announce `bytes` on the barrier and start the copy global -> shared.
    __device__ __forceinline__ void bulkLoad(void *dst_smem, const void *src_gmem, unsigned bytes, uint64_t *mbar)
    {
        const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
        const unsigned m = (unsigned)__cvta_generic_to_shared(mbar);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(m), "r"(bytes) : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(d),
                     "l"(src_gmem), "r"(bytes), "r"(m)
                     : "memory");
    }

    // Waits for the barrier phase with parity `phase`; gives up after `polls` polls, records
    // kStatusTimeout-style failure in *status and returns false.
    // Asynchronous 8-byte global -> shared copy (no register staging); completed by cpAsyncWaitAll
    // in the issuing thread, then published to the block by a barrier.
    __device__ __forceinline__ void cpAsync8(void *dst_smem, const void *src_gmem)
    {
        const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src_gmem) : "memory");
    }
    __device__ __forceinline__ void cpAsync4(void *dst_smem, const void *src_gmem)
    {
        const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src_gmem) : "memory");
    }
    template <typename T>
    __device__ __forceinline__ void cpAsyncElem(T *dst_smem, const T *src_gmem)
    {
        static_assert(sizeof(T) == 4 || sizeof(T) == 8, "4- or 8-byte elements");
        if constexpr (sizeof(T) == 8)
            cpAsync8(dst_smem, src_gmem);
        else
            cpAsync4(dst_smem, src_gmem);
    }
    __device__ __forceinline__ void cpAsyncWaitAll() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

    __device__ __forceinline__ bool mbarWait(uint64_t *mbar, unsigned phase, int *status, int polls = kWaitPolls)
    {
        const unsigned m = (unsigned)__cvta_generic_to_shared(mbar);
        for (int it = 0; it < polls; it++)
        {
            unsigned done;
            asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                         "selp.u32 %0, 1, 0, p;\n\t}"
                         : "=r"(done)
                         : "r"(m), "r"(phase)
                         : "memory");
            if (done)
                return true;
        }
        if (status)
            atomicExch(status, 6);
        return false;
    }

    // D += A B for one 8x8x4 FP64 tile (PTX mma.sync.aligned.m8n8k4.row.col.f64): lane l holds
    // A[l/4][l%4], B[l%4][l/4] and D[l/4][2(l%4) + {0,1}].
    __device__ __forceinline__ void dmma8x8x4(double &d0, double &d1, double a, double b)
    {
        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                     : "+d"(d0), "+d"(d1)
                     : "d"(a), "d"(b));
    }

    __device__ __forceinline__ void groupSync(int G)
    {
        if (G == 32)
            __syncwarp();
        else
            __syncthreads();
    }

    static __device__ HermAxisTable kHermAxis = makeHermAxisTable();

    // Group paths of total angular momentum L build R from its closed form (groupHermiteR) when the
    // staging fits the second R buffer and the expansion's extra terms stay few (it sums about 1.5x
    // the recursion's terms at L = 8 and 2x at L = 12, but needs two group barriers instead of L + 1).
    template <int L>
    constexpr bool closedFormR()
    {
        return L >= 4 && L <= 10 && 3 * hermAxisOffset(L + 1) + L + 1 <= nherm(L);
    }

    // R_tuv (t + u + v <= L) of one primitive quartet into out[0 .. nherm(L)) by the G threads of a
    // group, without the level-by-level recursion.  With g_n = fac (-2 alpha)^n F_n,
    //   R_tuv = sum_{a <= t/2} sum_{b <= u/2} sum_{c <= v/2} A_x[t][a] A_y[u][b] A_z[v][c] g_{t+u+v-a-b-c},
    //   A_x[t][a] = h(t, a) X^{t-2a}   (and A_y, A_z from Y, Z; h in HermAxisTable),
    // which is the McMurchie-Davidson recursion R^{(n)}_{t+1,u,v} = t R^{(n+1)}_{t-1,u,v} +
    // X R^{(n+1)}_{tuv} (Helgaker, Jorgensen, Olsen 9.9.18-9.9.20; src/lible/ints/rints.hpp:112-175)
    // unrolled to its closed form.  Step 1 writes the three axis tables and g (3 NH + L + 1 values)
    // to `stage`; step 2 sums every entry's terms.  Every thread of the group holds the same F, fac,
    // alpha and X, Y, Z; `ht` is the block's (t, u, v, t + u + v) table of the entries.
    template <int L, typename T>
    __device__ __forceinline__ void groupHermiteR(const double (&F)[L + 1], double fac, double m2a, double X, double Y,
                                                  double Z, T *stage, T *out, const char4 *ht, int tid, int G)
    {
        constexpr int NH = hermAxisOffset(L + 1);
        constexpr int NS = 3 * NH + L + 1;
        for (int j = tid; j < NS; j += G)
        {
            double base, pw;
            int p;
            if (j < 3 * NH)
            {
                const int axis = j >= 2 * NH ? 2 : (j >= NH ? 1 : 0);
                const int idx = j - axis * NH;
                base = axis == 0 ? X : (axis == 1 ? Y : Z);
                pw = __ldg(&kHermAxis.c[idx]);
                p = __ldg(&kHermAxis.p[idx]);
            }
            else
            {
                p = j - 3 * NH;
                double fn = F[0];
#pragma unroll
                for (int k = 1; k <= L; k++)
                    if (p == k)
                        fn = F[k];
                base = m2a;
                pw = fn * fac;
            }
            while (p)
            {
                if (p & 1)
                    pw *= base;
                base *= base;
                p >>= 1;
            }
            stage[j] = T(pw);
        }
        groupSync(G);
        const T *Ax = stage, *Ay = stage + NH, *Az = stage + 2 * NH, *g = stage + 3 * NH;
        for (int e = tid; e < nherm(L); e += G)
        {
            const char4 tv = ht[e];
            const int t = tv.x, u = tv.y, v = tv.z;
            const T *ax = Ax + hermAxisOffset(t), *ay = Ay + hermAxisOffset(u), *az = Az + hermAxisOffset(v);
            const T *gt = g + tv.w;
            T r = T(0);
            for (int a = 0; 2 * a <= t; a++)
                for (int b = 0; 2 * b <= u; b++)
                {
                    const T xy = ax[a] * ay[b];
                    const T *gn = gt - a - b;
                    for (int c = 0; 2 * c <= v; c++)
                        r += xy * az[c] * gn[-c];
                }
            out[e] = r;
        }
        groupSync(G);
    }

    template <typename T>
    __device__ __forceinline__ const T *braE(const PairView &v);
    template <>
    __device__ __forceinline__ const double *braE<double>(const PairView &v) { return v.E; }
    template <>
    __device__ __forceinline__ const float *braE<float>(const PairView &v) { return v.Ef; }
    template <typename T>
    __device__ __forceinline__ const T *ketE(const PairView &v);
    template <>
    __device__ __forceinline__ const double *ketE<double>(const PairView &v) { return v.Et; }
    template <>
    __device__ __forceinline__ const float *ketE<float>(const PairView &v) { return v.Etf; }

    // Destination offset of element (m, n, k, t) of a batch for kStore with the caller's
    // orientation flags.
    template <int SA, int SB, int SC, int SD>
    __device__ __forceinline__ size_t storeIndex(int flags, int m, int n, int k, int t)
    {
        int b0 = m, b1 = n, k0 = k, k1 = t;
        int db0 = SA, db1 = SB, dk0 = SC, dk1 = SD;
        if (flags & 1)
        {
            b0 = n; b1 = m; db0 = SB; db1 = SA;
        }
        if (flags & 2)
        {
            k0 = t; k1 = k; dk0 = SD; dk1 = SC;
        }
        if (flags & 4)
            return (((size_t)k0 * dk1 + k1) * db0 + b0) * db1 + b1;
        return (((size_t)b0 * db1 + b1) * dk0 + k0) * dk1 + k1;
    }

    // The bra pair's fields the digestion needs: first AOs of its shells, its molecule's block of
    // the packed D, J, K (first element, dimension; the ket shares it) and, optionally, the D_ab
    // block gathered in Schwarz order (dab[mn * dab_stride]) for coalesced reads.
    struct BraFields
    {
        int oa, ob, n;
        uint32_t base;
        const double *dab;
        int dab_stride;
    };

    __device__ __forceinline__ BraFields braFields(const int32_t *bi)
    {
        return BraFields{bi[0], bi[1], bi[7], (uint32_t)bi[6], nullptr, 0};
    }

    // Generic digestion of one batch V[SAB][SCD] (values read through `val(e)`), with the
    // thread subset [tid, tid + stride, ...] producing outputs.  Implements
    //   J_ab += 2 f V D_cd,  J_cd += 2 f V D_ab,
    //   K_ac += f V D_bd, K_ad += f V D_bc, K_bc += f V D_ad, K_bd += f V D_ac
    // into the unsymmetrised accumulators (J = A + A^T, K = B + B^T afterwards).  The K blocks are
    // written transposed (rows of the ket's AOs) and their D factors read through the symmetry of D,
    // so a ket-uniform warp whose bras are sorted by AO touches neighbouring columns of one row.
    // `collective` (serial form only): all 32 lanes of the warp call together, lane i holding the
    // quartet of ket pair `ket` (consecutive lanes hold consecutive tasks, so equal kets form runs).
    // The J_cd sums of each run of lanes with one ket pair, and the K_ac / K_ad sums of each run
    // with one ket pair and one shell a, are reduced by shuffles and added once by the run's first
    // lane.  `active` = false (collective form only): the lane holds no quartet; it forms a run of
    // its own with zeros and writes nothing.
    template <int SA, int SB, int SC, int SD, bool SERIAL, typename F>
    __device__ __forceinline__ void digestJK(const QuartetArgs &a, double f, const BraFields &bf,
                                             const int32_t *ki, F val, int tid, int stride,
                                             bool collective = false, bool active = true, uint32_t ket = 0)
    {
        if constexpr (SERIAL)
        {
            tid = 0;
            stride = 1;
        }
        const int n = bf.n;
        const size_t base = bf.base;
        const int oa = bf.oa, ob = bf.ob, oc = ki[0], od = ki[1];
        const double *D = a.D + base;
        double *const Jm = a.J + base;
        double *const Km = a.K + base;
        constexpr int n0 = SA * SB, n1 = n0 + SC * SD, n2 = n1 + SA * SC, n3 = n2 + SA * SD,
                      n4 = n3 + SB * SC, n5 = n4 + SB * SD;
        // runs of neighbouring lanes (a run starts where the key differs from the left neighbour's):
        // one ket pair for J_cd; one ket pair and one shell a for K_ac / K_ad (AO-sorted bras put
        // equal a next to each other).  Each run is summed with a shuffle tree and added once by its
        // first lane.
        int run_last_j = 0, run_last_k = 0;
        bool head_j = true, head_k = true;
        if constexpr (SERIAL)
            if (collective)
            {
                const int lane = threadIdx.x & 31;
                const long long kj = active ? (long long)ket : -1 - lane;
                const long long kleft = __shfl_up_sync(0xffffffffu, kj, 1);
                const int oleft = __shfl_up_sync(0xffffffffu, oa, 1);
                head_j = lane == 0 || kleft != kj;
                head_k = head_j || oleft != oa;
                const unsigned hj = __ballot_sync(0xffffffffu, head_j), hk = __ballot_sync(0xffffffffu, head_k);
                const unsigned above = lane == 31 ? 0u : (0xffffffffu << (lane + 1));
                run_last_j = (hj & above) ? __ffs(hj & above) - 2 : 31;
                run_last_k = (hk & above) ? __ffs(hk & above) - 2 : 31;
            }
#pragma unroll
        for (int o = tid; o < n5; o += stride)
        {
            double s = 0.0;
            double *dst;
            double w;
            if (o < n0)
            {
                int m = o / SB, nn = o % SB;
#pragma unroll
                for (int k = 0; k < SC; k++)
#pragma unroll
                    for (int t = 0; t < SD; t++)
                        s += val(((m * SB + nn) * SC + k) * SD + t) * __ldg(D + (size_t)(oc + k) * n + od + t);
                dst = Jm + (size_t)(oa + m) * n + ob + nn;
                w = 2.0 * f;
            }
            else if (o < n1)
            {
                int k = (o - n0) / SD, t = (o - n0) % SD;
#pragma unroll
                for (int m = 0; m < SA; m++)
#pragma unroll
                    for (int nn = 0; nn < SB; nn++)
                        s += val(((m * SB + nn) * SC + k) * SD + t) *
                             (bf.dab ? __ldg(bf.dab + (size_t)(m * SB + nn) * bf.dab_stride)
                                     : __ldg(D + (size_t)(oa + m) * n + ob + nn));
                dst = Jm + (size_t)(oc + k) * n + od + t;
                w = 2.0 * f;
            }
            else if (o < n2)
            {
                int m = (o - n1) / SC, k = (o - n1) % SC;
#pragma unroll
                for (int nn = 0; nn < SB; nn++)
#pragma unroll
                    for (int t = 0; t < SD; t++)
                        s += val(((m * SB + nn) * SC + k) * SD + t) * __ldg(D + (size_t)(od + t) * n + ob + nn);
                dst = Km + (size_t)(oc + k) * n + oa + m;
                w = f;
            }
            else if (o < n3)
            {
                int m = (o - n2) / SD, t = (o - n2) % SD;
#pragma unroll
                for (int nn = 0; nn < SB; nn++)
#pragma unroll
                    for (int k = 0; k < SC; k++)
                        s += val(((m * SB + nn) * SC + k) * SD + t) * __ldg(D + (size_t)(oc + k) * n + ob + nn);
                dst = Km + (size_t)(od + t) * n + oa + m;
                w = f;
            }
            else if (o < n4)
            {
                int nn = (o - n3) / SC, k = (o - n3) % SC;
#pragma unroll
                for (int m = 0; m < SA; m++)
#pragma unroll
                    for (int t = 0; t < SD; t++)
                        s += val(((m * SB + nn) * SC + k) * SD + t) * __ldg(D + (size_t)(od + t) * n + oa + m);
                dst = Km + (size_t)(oc + k) * n + ob + nn;
                w = f;
            }
            else
            {
                int nn = (o - n4) / SD, t = (o - n4) % SD;
#pragma unroll
                for (int m = 0; m < SA; m++)
#pragma unroll
                    for (int k = 0; k < SC; k++)
                        s += val(((m * SB + nn) * SC + k) * SD + t) * __ldg(D + (size_t)(oc + k) * n + oa + m);
                dst = Km + (size_t)(od + t) * n + ob + nn;
                w = f;
            }
            double v = active ? w * s : 0.0;
            if constexpr (SERIAL)
            {
                if (collective && o >= n0 && o < n3)
                {
                    // J_cd over the run of lanes with this lane's ket pair; K_ac, K_ad over the run
                    // with this lane's ket pair and shell a
                    const int lane = threadIdx.x & 31;
                    const int last = o < n1 ? run_last_j : run_last_k;
#pragma unroll
                    for (int off = 1; off < 32; off <<= 1)
                    {
                        const double u = __shfl_down_sync(0xffffffffu, v, off);
                        if (lane + off <= last)
                            v += u;
                    }
                    if (!(o < n1 ? head_j : head_k) || v == 0.0)
                        continue;
                }
                else if (!active)
                    continue;
            }
            atomicAdd(dst, v);
        }
    }

    // RI-J digestion of a three-centre batch (main pair | aux shell) or (aux | main).
    template <int SA, int SB, int SC, int SD, bool SERIAL, typename F>
    __device__ __forceinline__ void digestRI(const QuartetArgs &a, const int32_t *bi, const int32_t *ki,
                                             F val, int tid, int stride)
    {
        if constexpr (SERIAL)
        {
            tid = 0;
            stride = 1;
        }
        const int n = a.nao;
        // main pair (m0, m1) with sizes (S0, S1); aux shell with size SX
        const bool auxket = a.aux_side == 0;
        const int32_t *mi = auxket ? bi : ki;
        const int32_t *xi = auxket ? ki : bi;
        const int S0 = auxket ? SA : SC, S1 = auxket ? SB : SD, SX = auxket ? SC : SA;
        const int o0 = mi[0], o1 = mi[1], ox = xi[0];
        const double fb = (mi[4] == mi[5]) ? 0.5 : 1.0;
        auto V = [&](int m, int nn, int x) {
            return auxket ? val((m * SB + nn) * SC * SD + x) : val(x * SC * SD + m * SD + nn);
        };
        if (a.mode == kRIStore)
        {
            // both orientations of the main pair, or its packed lower-triangle element; consecutive
            // threads write consecutive n
            const bool packed = a.flags & kRIPacked;
            const size_t row = packed ? (size_t)n * (n + 1) / 2 : (size_t)n * n;
            for (int o = tid; o < SX * S0 * S1; o += stride)
            {
                const int nn = o % S1, m = (o / S1) % S0, x = o / (S0 * S1);
                const double v = V(m, nn, x);
                double *blk = a.out + (size_t)(ox + x - a.ri_lo) * row;
                const size_t i = (size_t)(o0 + m), j = (size_t)(o1 + nn);
                if (packed)
                    blk[i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i] = v;
                else
                {
                    blk[i * n + j] = v;
                    blk[j * n + i] = v;
                }
            }
        }
        else if (a.mode == kRIGamma)
        {
            for (int x = tid; x < SX; x += stride)
            {
                double s = 0.0;
                for (int m = 0; m < S0; m++)
                    for (int nn = 0; nn < S1; nn++)
                        s += V(m, nn, x) * __ldg(a.D + (size_t)(o0 + m) * n + o1 + nn);
                atomicAdd(a.gamma + ox + x, 2.0 * fb * s);
            }
        }
        else
        {
            for (int o = tid; o < S0 * S1; o += stride)
            {
                int m = o / S1, nn = o % S1;
                double s = 0.0;
                for (int x = 0; x < SX; x++)
                    s += V(m, nn, x) * __ldg(a.dcoef + ox + x);
                atomicAdd(a.J + (size_t)(o0 + m) * n + o1 + nn, fb * s);
            }
        }
    }

    // ---------------------------------------------------------------------------------------
    // Register path: a group of GT threads per contracted quartet, thread `member` owning the ket
    // columns [c0, c0 + CW) of the batch (c0 = member * CW).  Each thread evaluates the Boys
    // function and the R vector itself, so the group never synchronises; every index into R, the
    // R.E accumulator and the batch is a compile-time constant.
    template <typename T>
    __device__ __forceinline__ const T *braEs(const QuartetArgs &a);
    template <>
    __device__ __forceinline__ const double *braEs<double>(const QuartetArgs &a) { return a.bra_Es; }
    template <>
    __device__ __forceinline__ const float *braEs<float>(const QuartetArgs &a) { return a.bra_Efs; }

    // `sv` is the bra's structure-of-arrays entry (sv.z = 0: read the per-pair records instead).
    // `nk` >= 0 is the bra's primitive-pair count from the per-position fields (the bra records are
    // then read from the structure-of-arrays copies only); -1 reads the pair's primitive range.
    template <int LA, int LB, int LC, int LD, typename T, int SV = 0>
    __device__ __forceinline__ void quartetThread(const QuartetArgs &a, uint32_t ib, uint32_t ik, int c0, T *V,
                                                  const T *btab, uint4 sv, int nk)
    {
        using C = Cls<LA, LB, LC, LD>;
        constexpr int CW = Shape<LA, LB, LC, LD, T, SV>::CW;
#pragma unroll
        for (int x = 0; x < C::SAB * CW; x++)
            V[x] = T(0);
        uint32_t p0 = 0, p1 = (uint32_t)nk;
        if (nk < 0)
        {
            p0 = a.bra.pofs[ib];
            p1 = a.bra.pofs[ib + 1];
        }
        const uint32_t q0 = a.ket.pofs[ik], q1 = a.ket.pofs[ik + 1];
        const T *Eb = braE<T>(a.bra);
        const T *Ek = ketE<T>(a.ket) + c0;
        const size_t sn = sv.z;
        for (uint32_t p = p0; p < p1; p++)
        {
            PQ4 P;          // FP64 record
            float Pf[8];    // FP32 record: p, 1/p, P hi, P lo
            if constexpr (sizeof(T) == 8)
            {
                if (sn)
                {
                    const double *pp = a.bra_pPs + sv.x + (size_t)(p - p0) * 5 * sn;
                    P = {__ldg(pp), __ldg(pp + sn), __ldg(pp + 2 * sn), __ldg(pp + 3 * sn), __ldg(pp + 4 * sn)};
                }
                else
                    P = loadPQ(a.bra.pP, p);
            }
            else
            {
                if (sn)
                {
                    const float *pp = a.bra_pPfs + sv.w + (size_t)(p - p0) * 8 * sn;
#pragma unroll
                    for (int f = 0; f < 8; f++)
                        Pf[f] = __ldg(pp + f * sn);
                }
                else
                {
                    const float4 u = __ldg(reinterpret_cast<const float4 *>(a.bra.pPf) + 2 * (size_t)p);
                    const float4 w = __ldg(reinterpret_cast<const float4 *>(a.bra.pPf) + 2 * (size_t)p + 1);
                    Pf[0] = u.x; Pf[1] = u.y; Pf[2] = u.z; Pf[3] = u.w;
                    Pf[4] = w.x; Pf[5] = w.y; Pf[6] = w.z; Pf[7] = w.w;
                }
            }
            T RxE[C::HAB * CW];
#pragma unroll
            for (int x = 0; x < C::HAB * CW; x++)
                RxE[x] = T(0);
            for (uint32_t q = q0; q < q1; q++)
            {
                T R[C::NR];
                if constexpr (sizeof(T) == 8)
                {
                    const PQ4 Q = loadPQ(a.ket.pP, q);
                    // alpha = pq/(p+q) and the prefactor 2 pi^{5/2} / (p q sqrt(p+q)) from one rsqrt
                    const double rs = rsqrt(P.x + Q.x);
                    const double alpha = P.x * Q.x * (rs * rs);
                    const double X = P.y - Q.y, Y = P.z - Q.z, Z = P.w - Q.w;
                    const double fac = 34.986836655249725 * rs * P.ip * Q.ip;
                    double F[C::L + 1];
                    boysF<C::L, true>(alpha * (X * X + Y * Y + Z * Z), reinterpret_cast<const double *>(btab), F);
                    double Ft[C::L + 1];
#pragma unroll
                    for (int k = 0; k <= C::L; k++)
                        Ft[k] = F[k] * fac;
                    hermiteR<C::L, double>(-2.0 * alpha, Ft, X, Y, Z, reinterpret_cast<double *>(R));
                }
                else
                {
                    // FP32 geometry: P - Q from the hi/lo parts keeps float relative accuracy
                    const float4 u = __ldg(reinterpret_cast<const float4 *>(a.ket.pPf) + 2 * (size_t)q);
                    const float4 w = __ldg(reinterpret_cast<const float4 *>(a.ket.pPf) + 2 * (size_t)q + 1);
                    const float rs = rsqrtf(Pf[0] + u.x);
                    const float alpha = Pf[0] * u.x * (rs * rs);
                    const float X = (Pf[2] - u.z) + (Pf[5] - w.y);
                    const float Y = (Pf[3] - u.w) + (Pf[6] - w.z);
                    const float Z = (Pf[4] - w.x) + (Pf[7] - w.w);
                    const float fac = 34.986836655249725f * rs * Pf[1] * u.y;
                    float F[C::L + 1];
                    boysF32<C::L>(alpha * (X * X + Y * Y + Z * Z), reinterpret_cast<const float *>(btab), F);
#pragma unroll
                    for (int k = 0; k <= C::L; k++)
                        F[k] *= fac;
                    hermiteR<C::L, float>(-2.0f * alpha, F, X, Y, Z, reinterpret_cast<float *>(R));
                }
                const T *ec = Ek + (size_t)q * C::HCD * C::SCD;
#pragma unroll
                for (int hp = 0; hp < C::HCD; hp++)
                {
                    int tp = 0, up = 0, vp = 0;
                    // (t', u', v') of hp, resolved at compile time after unrolling
#pragma unroll
                    for (int n = 0, e = 0; n <= C::LCD; n++)
#pragma unroll
                        for (int t = n; t >= 0; t--)
#pragma unroll
                            for (int u = n - t; u >= 0; u--, e++)
                                if (e == hp)
                                {
                                    tp = t;
                                    up = u;
                                    vp = n - t - u;
                                }
                    T ecv[CW];
#pragma unroll
                    for (int c = 0; c < CW; c++)
                        ecv[c] = ((tp + up + vp) & 1) ? -ec[hp * C::SCD + c] : ec[hp * C::SCD + c];
#pragma unroll
                    for (int h = 0, n = 0; n <= C::LAB; n++)
#pragma unroll
                        for (int t = n; t >= 0; t--)
#pragma unroll
                            for (int u = n - t; u >= 0; u--, h++)
                            {
                                const int v = n - t - u;
                                const T r = R[hermIndex(t + tp, u + up, v + vp)];
#pragma unroll
                                for (int c = 0; c < CW; c++)
                                    RxE[h * CW + c] += r * ecv[c];
                            }
                }
            }
            const T *eb = sn ? braEs<T>(a) + sv.y + (size_t)(p - p0) * C::SAB * C::HAB * sn
                             : Eb + (size_t)p * C::SAB * C::HAB;
            const size_t es = sn ? sn : 1;
#pragma unroll
            for (int m = 0; m < C::SAB; m++)
#pragma unroll
                for (int h = 0; h < C::HAB; h++)
                {
                    const T e = __ldg(eb + (m * C::HAB + h) * es);
#pragma unroll
                    for (int c = 0; c < CW; c++)
                        V[m * CW + c] += e * RxE[h * CW + c];
                }
        }
    }

    // ---------------------------------------------------------------------------------------
    // G = 32 W: one thread group (the whole block) per contracted quartet.
    template <int LA, int LB, int LC, int LD, typename T, int SV = 0>
    __device__ __forceinline__ void quartetGroup(const QuartetArgs &a, uint32_t ib, uint32_t ik,
                                                 unsigned char *smem, T *vals)
    {
        using C = Cls<LA, LB, LC, LD>;
        using S = Shape<LA, LB, LC, LD, T, SV>;
        constexpr int G = S::G;
        const int tid = threadIdx.x;
        T *rb = reinterpret_cast<T *>(smem + S::off_rb);
        T *rm = reinterpret_cast<T *>(smem + S::off_rm);
        T *ecs = reinterpret_cast<T *>(smem + S::off_ec);
        T *eas = reinterpret_cast<T *>(smem + S::off_ea);
        T *rxs = reinterpret_cast<T *>(smem + S::off_rx);
        const short *rix = reinterpret_cast<const short *>(smem + S::off_ix);
        const char4 *ht = reinterpret_cast<const char4 *>(smem + S::off_ht);

#pragma unroll
        for (int k = 0; k < S::IB; k++)
            vals[k] = T(0);
        const uint32_t p0 = a.bra.pofs[ib], p1 = a.bra.pofs[ib + 1];
        const uint32_t q0 = a.ket.pofs[ik], q1 = a.ket.pofs[ik + 1];
        const T *Eb = braE<T>(a.bra);
        const T *Ek = ketE<T>(a.ket);
        for (uint32_t p = p0; p < p1; p++)
        {
            const PQ4 P = loadPQ(a.bra.pP, p);
            // the bra E tile lands while the ket loop runs (waited for before the second product)
            for (int e = tid; e < C::SAB * C::HAB; e += G)
                cpAsyncElem(eas + e, Eb + (size_t)p * C::SAB * C::HAB + e);
            T rxe[S::IK];
#pragma unroll
            for (int k = 0; k < S::IK; k++)
                rxe[k] = T(0);
            for (uint32_t q = q0; q < q1; q++)
            {
                // the ket E tile of this primitive lands during the Boys function and the R build
                for (int e = tid; e < C::HCD * C::SCD; e += G)
                    cpAsyncElem(ecs + e, Ek + (size_t)q * C::HCD * C::SCD + e);
                const PQ4 Q = loadPQ(a.ket.pP, q);
                const double rs = rsqrt(P.x + Q.x);
                const double alpha = P.x * Q.x * (rs * rs);
                const double X = P.y - Q.y, Y = P.z - Q.z, Z = P.w - Q.w;
                const double fac = 34.986836655249725 * rs * P.ip * Q.ip;
                double F[C::L + 1];
                boysF<C::L, false>(alpha * (X * X + Y * Y + Z * Z), a.boys + C::L * kBoysTerms * kBoysPitch, F);
                const double m2a = -2.0 * alpha;
                T *cur = rb, *nxt = rb + C::NR;
                if constexpr (closedFormR<C::L>())
                {
                    groupHermiteR<C::L, T>(F, fac, m2a, X, Y, Z, nxt, cur, ht, tid, G);
                }
                else
                {
                // level L
                double pw = 1.0;
                for (int k = 0; k < C::L; k++)
                    pw *= m2a;
                if (tid == 0)
                    cur[0] = T(F[C::L] * fac * pw);
                groupSync(G);
                for (int n = C::L - 1; n >= 0; n--)
                {
                    const int cnt = nherm(C::L - n);
                    for (int e = tid; e < cnt; e += G)
                    {
                        T r;
                        if (e == 0)
                        {
                            double pn = 1.0;
                            for (int k = 0; k < n; k++)
                                pn *= m2a;
                            r = T(F[n] * fac * pn);
                        }
                        else
                        {
                            const char4 tv = ht[e];
                            const int t = tv.x, u = tv.y, v = tv.z, m = tv.w;
                            if (t > 0)
                            {
                                r = T(X) * cur[nherm(m - 2) + cartIndex(u, v)];
                                if (t > 1)
                                    r += T(t - 1) * cur[nherm(m - 3) + cartIndex(u, v)];
                            }
                            else if (u > 0)
                            {
                                r = T(Y) * cur[nherm(m - 2) + cartIndex(u - 1, v)];
                                if (u > 1)
                                    r += T(u - 1) * cur[nherm(m - 3) + cartIndex(u - 2, v)];
                            }
                            else
                            {
                                r = T(Z) * cur[nherm(m - 2) + cartIndex(0, v - 1)];
                                if (v > 1)
                                    r += T(v - 1) * cur[nherm(m - 3) + cartIndex(0, v - 2)];
                            }
                        }
                        nxt[e] = r;
                    }
                    groupSync(G);
                    T *tmp = cur;
                    cur = nxt;
                    nxt = tmp;
                }
                }
                // signed R matrix [h'][h]; the ket E[q] [h'][cd] copies complete
                for (int e = tid; e < C::HCD * C::HAB; e += G)
                {
                    const short ix = rix[e];
                    const T r = cur[ix & 0x7fff];
                    rm[e] = (ix & 0x8000) ? -r : r;
                }
                cpAsyncWaitAll();
                groupSync(G);
#pragma unroll
                for (int k = 0; k < S::IK; k++)
                {
                    const int e = tid + G * k;
                    if (e < C::HAB * C::SCD)
                    {
                        const int h = e / C::SCD, c = e % C::SCD;
                        T s = rxe[k];
#pragma unroll 5
                        for (int hp = 0; hp < C::HCD; hp++)
                            s += rm[hp * C::HAB + h] * ecs[hp * C::SCD + c];
                        rxe[k] = s;
                    }
                }
                groupSync(G);
            }
#pragma unroll
            for (int k = 0; k < S::IK; k++)
            {
                const int e = tid + G * k;
                if (e < C::HAB * C::SCD)
                    rxs[e] = rxe[k];
            }
            cpAsyncWaitAll();  // the bra E tile (already complete unless the ket loop was empty)
            groupSync(G);
#pragma unroll
            for (int k = 0; k < S::IB; k++)
            {
                const int e = tid + G * k;
                if (e < C::SAB * C::SCD)
                {
                    const int m = e / C::SCD, c = e % C::SCD;
                    T s = vals[k];
#pragma unroll 5
                    for (int h = 0; h < C::HAB; h++)
                        s += eas[m * C::HAB + h] * rxs[h * C::SCD + c];
                    vals[k] = s;
                }
            }
            groupSync(G);
        }
    }

    // ---------------------------------------------------------------------------------------
    // FP64 group path on the DMMA pipe.  Per primitive quartet the block builds R (recursion in
    // shared memory), writes the signed R matrix rm[h'][h] and stages E_ket[q] ec[h'][c], both into
    // zero-padded tiles; every warp then accumulates its 8x8 tiles of R.E_ket^T over the ket
    // primitives in registers (acc).  Per bra primitive the R.E tiles go to shared memory and the
    // warps accumulate their 8x8 tiles of E_bra . (R.E) into `v`.  Padded rows and columns of the
    // operand tiles are zeroed once per block and never written afterwards.
    // `phase` is the parity of the block's mbarrier phase awaited next; it lives as long as the block
    // (one completed phase per ket primitive of every quartet), so it is carried across calls.
    // Returns false when a bounded wait on a ket tile gave up (status word set): the block has then
    // let any copy still in flight land (again bounded) and must stop without using the batch.
    template <int LA, int LB, int LC, int LD, int SV = 0>
    __device__ __forceinline__ bool quartetGroupMMA(const QuartetArgs &a, const GroupTask &g,
                                                    unsigned char *smem, double (&v)[Shape<LA, LB, LC, LD, double, SV>::TPW2][2],
                                                    unsigned &phase)
    {
        using C = Cls<LA, LB, LC, LD>;
        using S = Shape<LA, LB, LC, LD, double, SV>;
        constexpr int G = S::G;
        const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, r8 = lane >> 2, k4 = lane & 3;
        double *rb = reinterpret_cast<double *>(smem + S::m_off_rb);
        double *rm = reinterpret_cast<double *>(smem + S::m_off_rm);
        double *ec = reinterpret_cast<double *>(smem + S::m_off_ec);
        double *ea = reinterpret_cast<double *>(smem + S::m_off_ea);
        double *rx = reinterpret_cast<double *>(smem + S::m_off_rx);
        const short *rix = reinterpret_cast<const short *>(smem + S::m_off_ix);
        const char4 *ht = reinterpret_cast<const char4 *>(smem + S::m_off_ht);
        uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + S::m_off_mb);
        // the padded ket E tiles arrive by bulk copy (issued at the top of a ket-primitive iteration,
        // overlapping the Boys function and the R recursion); without them the block stages the tile
        const double *ket_tiles = a.ket_EtP;

#pragma unroll
        for (int i = 0; i < S::TPW2; i++)
            v[i][0] = v[i][1] = 0.0;
        const uint32_t p0 = g.p0, p1 = g.p1;
        const uint32_t q0 = g.q0, q1 = g.q1;
        for (uint32_t p = p0; p < p1; p++)
        {
            const PQ4 P = p == p0 ? g.P : loadPQ(a.bra.pP, p);
            // the bra E tile of this primitive lands while the ket loop runs; it is first read by
            // the second product, after the wait and the barrier in front of it
            for (int e = tid; e < C::SAB * C::HAB; e += G)
                cpAsync8(ea + (e / C::HAB) * S::P_EA + e % C::HAB, a.bra.E + (size_t)p * C::SAB * C::HAB + e);
            double acc[S::TPW][2];
#pragma unroll
            for (int i = 0; i < S::TPW; i++)
                acc[i][0] = acc[i][1] = 0.0;
            for (uint32_t q = q0; q < q1; q++)
            {
                if (ket_tiles && tid == 0 && !a.wait_inject)
                    bulkLoad(ec, ket_tiles + (size_t)q * (S::ec_tile_bytes / 8), S::ec_tile_bytes, mbar);
                const PQ4 Q = q == q0 ? g.Q : loadPQ(a.ket.pP, q);
                const double rs = rsqrt(P.x + Q.x);
                const double alpha = P.x * Q.x * (rs * rs);
                const double X = P.y - Q.y, Y = P.z - Q.z, Z = P.w - Q.w;
                const double fac = 34.986836655249725 * rs * P.ip * Q.ip;
                double F[C::L + 1];
                boysF<C::L, false>(alpha * (X * X + Y * Y + Z * Z), a.boys + C::L * kBoysTerms * kBoysPitch, F);
                const double m2a = -2.0 * alpha;
                double *cur = rb, *nxt = rb + C::NR;
                if constexpr (closedFormR<C::L>())
                {
                    groupHermiteR<C::L, double>(F, fac, m2a, X, Y, Z, nxt, cur, ht, tid, G);
                }
                else
                {
                double pw = 1.0;
                for (int k = 0; k < C::L; k++)
                    pw *= m2a;
                if (tid == 0)
                    cur[0] = F[C::L] * fac * pw;
                groupSync(G);
                // levels unrolled (L is a compile-time constant) so F[n] stays in registers
#pragma unroll
                for (int n = C::L - 1; n >= 0; n--)
                {
                    const int cnt = nherm(C::L - n);
                    for (int e = tid; e < cnt; e += G)
                    {
                        double r;
                        if (e == 0)
                        {
                            double pn = 1.0;
                            for (int k = 0; k < n; k++)
                                pn *= m2a;
                            r = F[n] * fac * pn;
                        }
                        else
                        {
                            const char4 tv = ht[e];
                            const int t = tv.x, u = tv.y, vv = tv.z, m = tv.w;
                            if (t > 0)
                            {
                                r = X * cur[nherm(m - 2) + cartIndex(u, vv)];
                                if (t > 1)
                                    r += (t - 1) * cur[nherm(m - 3) + cartIndex(u, vv)];
                            }
                            else if (u > 0)
                            {
                                r = Y * cur[nherm(m - 2) + cartIndex(u - 1, vv)];
                                if (u > 1)
                                    r += (u - 1) * cur[nherm(m - 3) + cartIndex(u - 2, vv)];
                            }
                            else
                            {
                                r = Z * cur[nherm(m - 2) + cartIndex(0, vv - 1)];
                                if (vv > 1)
                                    r += (vv - 1) * cur[nherm(m - 3) + cartIndex(0, vv - 2)];
                            }
                        }
                        nxt[e] = r;
                    }
                    groupSync(G);
                    double *tmp = cur;
                    cur = nxt;
                    nxt = tmp;
                }
                }
                // signed R matrix rm[h'][h] and the staged ket E[q] ec[h'][c]
                for (int e = tid; e < C::HCD * C::HAB; e += G)
                {
                    const short ix = rix[e];
                    const double r = cur[ix & 0x7fff];
                    rm[(e / C::HAB) * S::P_RM + e % C::HAB] = (ix & 0x8000) ? -r : r;
                }
                if (ket_tiles)
                {
                    const unsigned ph = phase;
                    const bool ok = mbarWait(mbar, ph, a.status, a.wait_inject ? a.wait_inject : kWaitPolls);
                    phase ^= 1u;
                    // the block agrees on the outcome; after a give-up no thread reads the tile
                    if (__syncthreads_or(!ok))
                    {
                        if (tid == 0 && !a.wait_inject)
                            mbarWait(mbar, ph, nullptr);  // a late copy lands before the block exits
                        cpAsyncWaitAll();                 // and so do the bra E copies
                        return false;
                    }
                }
                else
                    for (int e = tid; e < C::HCD * C::SCD; e += G)
                        ec[(e / C::SCD) * S::P_EC + e % C::SCD] = __ldg(a.ket.Et + (size_t)q * C::HCD * C::SCD + e);
                groupSync(G);
                // acc[tile] += R^T[h][h'] E_ket[h'][c] over h' (A = rm viewed transposed, row-major)
#pragma unroll
                for (int i = 0; i < S::TPW; i++)
                {
                    const int t = warp + i * S::WM;
                    if (t < S::TILES)
                    {
                        const int mt = t / S::NT, nt = t % S::NT;
                        const double *A = rm + k4 * S::P_RM + mt * 8 + r8;
                        const double *B = ec + k4 * S::P_EC + nt * 8 + r8;
#pragma unroll 4
                        for (int ks = 0; ks < S::KT; ks++)
                            dmma8x8x4(acc[i][0], acc[i][1], A[ks * 4 * S::P_RM], B[ks * 4 * S::P_EC]);
                    }
                }
                groupSync(G);
            }
            // R.E tiles to shared memory (rows h, columns c; padded entries are zero)
#pragma unroll
            for (int i = 0; i < S::TPW; i++)
            {
                const int t = warp + i * S::WM;
                if (t < S::TILES)
                {
                    const int mt = t / S::NT, nt = t % S::NT;
                    double *o = rx + (mt * 8 + r8) * S::P_EC + nt * 8 + 2 * k4;
                    o[0] = acc[i][0];
                    o[1] = acc[i][1];
                }
            }
            cpAsyncWaitAll();
            groupSync(G);
            // v[tile] += E_bra[m][h] (R.E)[h][c] over h
#pragma unroll
            for (int i = 0; i < S::TPW2; i++)
            {
                const int t = warp + i * S::WM;
                if (t < S::TILES2)
                {
                    const int mt = t / S::NT, nt = t % S::NT;
                    const double *A = ea + (mt * 8 + r8) * S::P_EA + k4;
                    const double *B = rx + k4 * S::P_EC + nt * 8 + r8;
#pragma unroll 4
                    for (int ks = 0; ks < S::KT2; ks++)
                        dmma8x8x4(v[i][0], v[i][1], A[ks * 4], B[ks * 4 * S::P_EC]);
                }
            }
            groupSync(G);
        }
        return true;
    }

    // Tables and zero padding of the DMMA layout (once per block).
    template <int LA, int LB, int LC, int LD, int SV = 0>
    __device__ __forceinline__ void buildGroupTablesMMA(unsigned char *smem)
    {
        using C = Cls<LA, LB, LC, LD>;
        using S = Shape<LA, LB, LC, LD, double, SV>;
        double *z = reinterpret_cast<double *>(smem + S::m_off_rm);
        const int nz = (int)((S::m_off_ix - S::m_off_rm) / 8);
        for (int e = threadIdx.x; e < nz; e += blockDim.x)
            z[e] = 0.0;
        short *rix = reinterpret_cast<short *>(smem + S::m_off_ix);
        char4 *ht = reinterpret_cast<char4 *>(smem + S::m_off_ht);
        for (int e = threadIdx.x; e < C::NR; e += blockDim.x)
        {
            int t, u, v;
            hermTuv(e, t, u, v);
            ht[e] = make_char4((char)t, (char)u, (char)v, (char)(t + u + v));
        }
        for (int e = threadIdx.x; e < C::HCD * C::HAB; e += blockDim.x)
        {
            const int hp = e / C::HAB, h = e % C::HAB;
            int t, u, v, tp, up, vp;
            hermTuv(h, t, u, v);
            hermTuv(hp, tp, up, vp);
            int ix = hermIndex(t + tp, u + up, v + vp);
            if ((tp + up + vp) & 1)
                ix |= 0x8000;
            rix[e] = (short)ix;
        }
        if (threadIdx.x == 0)
            mbarInit(reinterpret_cast<uint64_t *>(smem + S::m_off_mb));
        __syncthreads();
    }

    // Builds the per-block tables of the group shape: Hermite (t,u,v,order) list and the signed
    // combined index of (h + h') for the R matrix.
    template <int LA, int LB, int LC, int LD, typename T, int SV = 0>
    __device__ __forceinline__ void buildGroupTables(unsigned char *smem)
    {
        using C = Cls<LA, LB, LC, LD>;
        using S = Shape<LA, LB, LC, LD, T, SV>;
        short *rix = reinterpret_cast<short *>(smem + S::off_ix);
        char4 *ht = reinterpret_cast<char4 *>(smem + S::off_ht);
        for (int e = threadIdx.x; e < C::NR; e += blockDim.x)
        {
            int t, u, v;
            hermTuv(e, t, u, v);
            ht[e] = make_char4((char)t, (char)u, (char)v, (char)(t + u + v));
        }
        for (int e = threadIdx.x; e < C::HCD * C::HAB; e += blockDim.x)
        {
            const int hp = e / C::HAB, h = e % C::HAB;
            int t, u, v, tp, up, vp;
            hermTuv(h, t, u, v);
            hermTuv(hp, tp, up, vp);
            int ix = hermIndex(t + tp, u + up, v + vp);
            if ((tp + up + vp) & 1)
                ix |= 0x8000;
            rix[e] = (short)ix;
        }
        __syncthreads();
    }

    // Resident blocks per SM the compiler must allow for (register cap 65536 / (block * n)), for the
    // register-path classes where a higher occupancy measured faster on the (H2O)_32 cc-pVDZ J/K build
    // than the default bound (which lets the compiler use more registers): FP64 (dp|ps), (ds|ps),
    // (dp|ss) at 3 blocks and (ps|ss) at 6; FP32 (dp|ps), (ds|pp) at 3, (pp|ps) at 4, (ps|ps) at 6,
    // (ds|ss) at 8; and the DMMA group-path classes at 128 registers per thread where their shared
    // memory allows the blocks ((dd|dd): 166 -> 128 registers, 3 -> 4 blocks, 1.34 -> 1.15 ms on
    // (H2O)_8 cc-pVTZ).  1 = the default bound.
    template <int LA, int LB, int LC, int LD, typename T, int SV = 0>
    constexpr int minBlocksPerSM()
    {
        using S = Shape<LA, LB, LC, LD, T, SV>;
        if (SV != 0)
            return 1;
        if constexpr (S::MMA)
        {
            // DMMA group path: 128 registers per thread (4 blocks of 128 threads, 8 of 64, 2 of
            // 256), where the shared-memory layout lets that many blocks reside
            const int want = S::block <= 64 ? 8 : S::block <= 128 ? 4 : 2;
            const int fit = (int)((228 * 1024) / (S::m_smem + 1024));
            return want < fit ? want : fit;
        }
        if (S::W != 0)
            return 1;
        constexpr int c = LA * 1000 + LB * 100 + LC * 10 + LD;
        if (sizeof(T) == 8)
            return (c == 2110 || c == 2010 || c == 2100) ? 3 : c == 1000 ? 6 : 1;
        return (c == 2110 || c == 2011) ? 3 : c == 1110 ? 4 : c == 1010 ? 6 : c == 2000 ? 8 : 1;
    }

    // Forward kernel body: every mode except the derivative ones.
    template <int LA, int LB, int LC, int LD, typename T, int SV = 0>
    __device__ __forceinline__ void eriKernelBody(const QuartetArgs &a)
    {
        using C = Cls<LA, LB, LC, LD>;
        using S = Shape<LA, LB, LC, LD, T, SV>;
        constexpr int blk = C::SAB * C::SCD;
        if constexpr (S::W == 0)
        {
            constexpr int GT = S::GT, CW = S::CW, QPW = S::QPW;
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            const int slot = lane / GT, member = lane % GT;
            const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
            const long long gw = (long long)blockIdx.x * (blockDim.x >> 5) + warp;
            extern __shared__ __align__(16) unsigned char smem[];
            double *vs = reinterpret_cast<double *>(smem) + ((size_t)warp * QPW + slot) * blk;
            T *btab = reinterpret_cast<T *>(smem + S::off_boys);
            if constexpr (sizeof(T) == 8)
                stageBoys(a.boys, C::L, reinterpret_cast<double *>(btab));
            else
                stageBoys(a.boys_f, C::L, reinterpret_cast<float *>(btab));
            __syncthreads();
            // each warp walks chunks of consecutive tasks (QPW per iteration); consecutive tasks
            // share the major pair, so the task cursor rarely moves.  A warp's chunks come in
            // increasing task order, so the cursor carries over from one chunk to the next.
            int cur = 0;
            // tasks [start, end) of one chunk, QPW quartets per warp step
            auto processRange = [&](long long start, long long end) {
            if (!a.list)
                cur = advanceMajor(a, start, cur);
            for (long long base = start; base < end; base += QPW)
            {
                const long long t = base + slot;
                const bool valid = slot < QPW && t < end;
                uint32_t ib = 0, ik = 0;
                T V[C::SAB * CW];
                BraFields bf{0, 0, 0, 0, nullptr, 0};
                bool bsame = false;
                bool active = false;  // a valid task inside the launch's Schwarz window
                if (valid)
                {
                    int my = cur;
                    uint32_t pos;
                    decodeCursor(a, t, my, ib, ik, pos);
                    active = inWindow(a, ib, ik, pos, true);
                    const uint4 sv = a.bra_soa ? __ldg(a.bra_soa + pos) : make_uint4(0, 0, 0, 0);
                    int nk = -1;
                    if (a.bra_soa2)
                    {
                        // one coalesced 16-byte load instead of the pair's info record and
                        // primitive range
                        const int4 si = __ldg(a.bra_soa2 + pos);
                        bf = BraFields{si.x, si.y, si.w & 0xffff, (uint32_t)si.z,
                                       a.bra_Dab ? a.bra_Dab + pos : nullptr, a.bra_npos};
                        nk = (si.w >> 16) & 0x7fff;
                        bsame = si.w < 0;
                    }
                    else if (a.mode == kJK)
                    {
                        const int32_t *bi0 = a.bra.info + 8 * ib;
                        bf = braFields(bi0);
                        bsame = bi0[4] == bi0[5];
                    }
                    if (active)
                        quartetThread<LA, LB, LC, LD, T, SV>(a, ib, ik, member * CW, V, btab, sv, nk);
                    else
                    {
#pragma unroll
                        for (int x = 0; x < C::SAB * CW; x++)
                            V[x] = T(0);
                    }
                }
                if (!a.list)
                    cur = advanceMajor(a, base + QPW < end ? base + QPW : end - 1, cur);
                const int32_t *bi = a.bra.info + 8 * ib;
                const int32_t *ki = a.ket.info + 8 * ik;
                if (a.mode == kStore)
                {
                    if (active)
                    {
#pragma unroll
                        for (int m = 0; m < C::SAB; m++)
#pragma unroll
                            for (int c = 0; c < CW; c++)
                            {
                                const int kt = member * CW + c;
                                a.out[(size_t)t * blk + storeIndex<C::SA, C::SB, C::SC, C::SD>(
                                                            a.flags, m / C::SB, m % C::SB, kt / C::SD, kt % C::SD)] =
                                    (double)V[m * CW + c];
                            }
                    }
                }
                else if constexpr (GT == 1)
                {
                    auto val = [&](int e) { return (double)V[e]; };
                    // ket-major enumeration: consecutive lanes mostly share the ket pair, and the
                    // whole warp digests together (runs of equal ket pairs reduced)
                    if (a.mode == kJK)
                        digestJK<C::SA, C::SB, C::SC, C::SD, true>(a, quartetWeight(a, bsame, ib, ik), bf, ki, val, 0,
                                                                   1, true, active, ik);
                    else if (active)
                        digestRI<C::SA, C::SB, C::SC, C::SD, true>(a, bi, ki, val, 0, 1);
                }
                else
                {
                    // gather the quartet's columns in shared memory, then digest with the group
                    if (active)
                    {
#pragma unroll
                        for (int m = 0; m < C::SAB; m++)
#pragma unroll
                            for (int c = 0; c < CW; c++)
                                vs[m * C::SCD + member * CW + c] = (double)V[m * CW + c];
                    }
                    __syncwarp();
                    if (active)
                    {
                        auto val = [&](int e) { return vs[e]; };
                        if (a.mode == kJK)
                            digestJK<C::SA, C::SB, C::SC, C::SD, false>(a, quartetWeight(a, bsame, ib, ik), bf, ki,
                                                                        val, member, GT);
                        else
                            digestRI<C::SA, C::SB, C::SC, C::SD, false>(a, bi, ki, val, member, GT);
                    }
                    __syncwarp();
                }
            }
            };
            if (a.chunks)
            {
                // work queue: lane 0 claims the next chunk for the whole warp
                for (;;)
                {
                    unsigned long long c = 0;
                    if (lane == 0)
                        c = atomicAdd(a.counter, 1ULL);
                    c = __shfl_sync(0xffffffffu, c, 0);
                    if (c >= (unsigned long long)a.n_chunks)
                        break;
                    processRange((long long)__ldg(a.chunks + c), (long long)__ldg(a.chunks + c + 1));
                }
            }
            else
            {
                // static chunks of 8 warp steps, strided over the grid's warps
                constexpr long long CH = 8 * QPW;
                const long long n_chunks = (a.n_tasks + CH - 1) / CH;
                for (long long chunk = gw; chunk < n_chunks; chunk += warps)
                    processRange(chunk * CH, (chunk + 1) * CH < a.n_tasks ? (chunk + 1) * CH : a.n_tasks);
            }
        }
        else if constexpr (S::MMA)
        {
            extern __shared__ __align__(16) unsigned char smem[];
            buildGroupTablesMMA<LA, LB, LC, LD, SV>(smem);
            double *vs = reinterpret_cast<double *>(smem + S::m_off_rx);
            GroupTask *tasks = reinterpret_cast<GroupTask *>(smem + S::m_off_tb);
            const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, r8 = lane >> 2, k4 = lane & 3;
            unsigned phase = 0;  // parity of the block mbarrier's next phase
            // each thread's task cursor: a block's chunks, and a thread's tasks in them, come in
            // increasing task order, so the cursor only moves forward
            int cur = 0;
            // one quartet at a time for the whole block, tasks [start, end) of a chunk; false = a
            // bounded wait gave up and the block stops.  The tasks are decoded kGroupTaskBatch at a
            // time, one per thread, with their primitive ranges and first primitive records, so each
            // quartet starts from shared memory rather than a chain of dependent global loads.
            auto processRange = [&](long long start, long long end) -> bool {
            for (long long t0 = start; t0 < end; t0 += kGroupTaskBatch)
            {
            const int nb = (int)(end - t0 < kGroupTaskBatch ? end - t0 : kGroupTaskBatch);
            if ((int)threadIdx.x < nb)
                loadGroupTask(a, t0 + threadIdx.x, cur, tasks[threadIdx.x]);
            __syncthreads();
            for (int j = 0; j < nb; j++)
            {
                const GroupTask &gt = tasks[j];
                if (!gt.ok)
                    continue;
                const long long t = t0 + j;
                const uint32_t ib = gt.ib, ik = gt.ik;
                double v[S::TPW2][2];
                if (!quartetGroupMMA<LA, LB, LC, LD, SV>(a, gt, smem, v, phase))
                    return false;
                // element (m, c) of the batch held by this thread: tile rows / columns
#pragma unroll
                for (int i = 0; i < S::TPW2; i++)
                {
                    const int tt = warp + i * S::WM;
                    if (tt < S::TILES2)
                    {
                        const int m = (tt / S::NT) * 8 + r8;
#pragma unroll
                        for (int j = 0; j < 2; j++)
                        {
                            const int c = (tt % S::NT) * 8 + 2 * k4 + j;
                            if (m < C::SAB && c < C::SCD)
                            {
                                if (a.mode == kStore)
                                    a.out[(size_t)t * blk + storeIndex<C::SA, C::SB, C::SC, C::SD>(
                                                                a.flags, m / C::SB, m % C::SB, c / C::SD, c % C::SD)] =
                                        v[i][j];
                                else
                                    vs[m * C::SCD + c] = v[i][j];
                            }
                        }
                    }
                }
                if (a.mode != kStore)
                {
                    __syncthreads();
                    const int32_t *bi = a.bra.info + 8 * ib;
                    const int32_t *ki = a.ket.info + 8 * ik;
                    auto val = [&](int e) { return vs[e]; };
                    if (a.mode == kJK)
                        digestJK<C::SA, C::SB, C::SC, C::SD, false>(a, quartetWeight(a, ib, ik), braFields(bi), ki,
                                                                    val, threadIdx.x, S::G);
                    else
                        digestRI<C::SA, C::SB, C::SC, C::SD, false>(a, bi, ki, val, threadIdx.x, S::G);
                }
                __syncthreads();
            }
            __syncthreads();  // every thread is done with the batch's task records
            }
            return true;
            };
            if (a.chunks)
            {
                __shared__ unsigned long long claimed;
                for (;;)
                {
                    if (threadIdx.x == 0)
                        claimed = atomicAdd(a.counter, 1ULL);
                    __syncthreads();
                    const unsigned long long c = claimed;
                    __syncthreads();
                    if (c >= (unsigned long long)a.n_chunks)
                        break;
                    if (!processRange((long long)__ldg(a.chunks + c), (long long)__ldg(a.chunks + c + 1)))
                        break;
                }
            }
            else
            {
                constexpr long long CHB = 8;
                const long long n_chunks = (a.n_tasks + CHB - 1) / CHB;
                for (long long chunk = blockIdx.x; chunk < n_chunks; chunk += gridDim.x)
                    if (!processRange(chunk * CHB, (chunk + 1) * CHB < a.n_tasks ? (chunk + 1) * CHB : a.n_tasks))
                        break;
            }
        }
        else
        {
            extern __shared__ __align__(16) unsigned char smem[];
            buildGroupTables<LA, LB, LC, LD, T, SV>(smem);
            T *vs = reinterpret_cast<T *>(smem + S::off_rx);
            // the task cursor carries over between the block's chunks (increasing task order)
            int cur = 0;
            // one quartet at a time for the whole block, tasks [start, end) of a chunk
            auto processRange = [&](long long start, long long end) {
            for (long long t = start; t < end; t++)
            {
                uint32_t ib, ik;
                decodeCursor(a, t, cur, ib, ik);
                if (!inWindow(a, ib, ik, 0, false))
                    continue;
                T vals[S::IB];
                quartetGroup<LA, LB, LC, LD, T, SV>(a, ib, ik, smem, vals);
                if (a.mode == kStore)
                {
#pragma unroll
                    for (int k = 0; k < S::IB; k++)
                    {
                        const int e = threadIdx.x + S::G * k;
                        if (e < blk)
                        {
                            const int mn = e / C::SCD, kt = e % C::SCD;
                            a.out[(size_t)t * blk + storeIndex<C::SA, C::SB, C::SC, C::SD>(
                                                        a.flags, mn / C::SB, mn % C::SB, kt / C::SD, kt % C::SD)] =
                                (double)vals[k];
                        }
                    }
                }
                else
                {
#pragma unroll
                    for (int k = 0; k < S::IB; k++)
                    {
                        const int e = threadIdx.x + S::G * k;
                        if (e < blk)
                            vs[e] = vals[k];
                    }
                    __syncthreads();
                    const int32_t *bi = a.bra.info + 8 * ib;
                    const int32_t *ki = a.ket.info + 8 * ik;
                    auto val = [&](int e) { return (double)vs[e]; };
                    if (a.mode == kJK)
                        digestJK<C::SA, C::SB, C::SC, C::SD, false>(a, quartetWeight(a, ib, ik), braFields(bi), ki,
                                                                    val, threadIdx.x, S::G);
                    else
                        digestRI<C::SA, C::SB, C::SC, C::SD, false>(a, bi, ki, val, threadIdx.x, S::G);
                }
                __syncthreads();
            }
            };
            if (a.chunks)
            {
                __shared__ unsigned long long claimed;
                for (;;)
                {
                    if (threadIdx.x == 0)
                        claimed = atomicAdd(a.counter, 1ULL);
                    __syncthreads();
                    const unsigned long long c = claimed;
                    __syncthreads();
                    if (c >= (unsigned long long)a.n_chunks)
                        break;
                    processRange((long long)__ldg(a.chunks + c), (long long)__ldg(a.chunks + c + 1));
                }
            }
            else
            {
                // static chunks of 8 consecutive tasks, strided over the grid's blocks
                constexpr long long CHB = 8;
                const long long n_chunks = (a.n_tasks + CHB - 1) / CHB;
                for (long long chunk = blockIdx.x; chunk < n_chunks; chunk += gridDim.x)
                    processRange(chunk * CHB, (chunk + 1) * CHB < a.n_tasks ? (chunk + 1) * CHB : a.n_tasks);
            }
        }
    }

    // The class kernels: the default register bound, or (minBlocksPerSM > 1) one that lets that many
    // blocks reside per SM.  Only the selected one is instantiated per class (eriKernelFor).
    template <int LA, int LB, int LC, int LD, typename T, int SV = 0>
    __global__ void __launch_bounds__(Shape<LA, LB, LC, LD, T, SV>::block) eriKernel(QuartetArgs a)
    {
        eriKernelBody<LA, LB, LC, LD, T, SV>(a);
    }
    template <int LA, int LB, int LC, int LD, typename T, int SV = 0>
    __global__ void __launch_bounds__(Shape<LA, LB, LC, LD, T, SV>::block, minBlocksPerSM<LA, LB, LC, LD, T, SV>())
    eriKernelOcc(QuartetArgs a)
    {
        eriKernelBody<LA, LB, LC, LD, T, SV>(a);
    }
    // Whether shape variant 1 differs from the default (otherwise only variant 0 is instantiated).
    template <int LA, int LB, int LC, int LD, typename T>
    constexpr bool hasShapeVariant()
    {
        using S0 = Shape<LA, LB, LC, LD, T, 0>;
        using S1 = Shape<LA, LB, LC, LD, T, 1>;
        return S0::GT != S1::GT || S0::W != S1::W || minBlocksPerSM<LA, LB, LC, LD, T, 0>() > 1;
    }
    // Whether a J/K class (la lb | lc ld) with distinct pair types may also run in the other
    // orientation, (lc ld | la lb), the bra and ket exchanged: instantiated where that orientation
    // takes the register path.  The launch autotuner times it as shape 2 against shapes 0 and 1.
    template <int LA, int LB, int LC, int LD, typename T>
    constexpr bool hasFlippedShape()
    {
        return (LA != LC || LB != LD) && Shape<LC, LD, LA, LB, T, 0>::GT > 0;
    }

    template <int LA, int LB, int LC, int LD, typename T, int SV = 0>
    constexpr auto eriKernelFor()
    {
        if constexpr (minBlocksPerSM<LA, LB, LC, LD, T, SV>() > 1)
            return &eriKernelOcc<LA, LB, LC, LD, T, SV>;
        else
            return &eriKernel<LA, LB, LC, LD, T, SV>;
    }
}
