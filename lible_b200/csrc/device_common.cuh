// Device-side building blocks shared by the ERI kernels: class dimensions, the Boys function,
// the Hermite R recursion and the quartet-task decoding.
#pragma once

#include "lible_math.hpp"

#include <cstdint>
#include <cuda_runtime.h>

namespace lible_b200
{
    // Compile-time dimensions of a quartet class (la lb | lc ld).
    template <int LA, int LB, int LC, int LD>
    struct Cls
    {
        static constexpr int LAB = LA + LB, LCD = LC + LD, L = LAB + LCD;
        static constexpr int SA = 2 * LA + 1, SB = 2 * LB + 1, SC = 2 * LC + 1, SD = 2 * LD + 1;
        static constexpr int SAB = SA * SB, SCD = SC * SD;
        static constexpr int HAB = nherm(LAB), HCD = nherm(LCD), NR = nherm(L);
        static constexpr int NR1 = nherm(L + 1);
    };

    // Views of one pair class in device memory (see DevPairClass).
    struct PairView
    {
        const double *pP;      // [ppair][8] p, Px, Py, Pz, 1/p, a, b, 0
        const double *ab;      // [ppair][2] a, b
        const uint32_t *pofs;  // [pair + 1]
        const int32_t *info;   // [pair][8] ao_a, ao_b, atom_a, atom_b, shell_a, shell_b
        const double *E;       // [ppair][S_ab][H_ab]
        const double *Et;      // [ppair][H_ab][S_ab]
        const float *Ef;
        const float *Etf;
        const double *E1;      // [ppair][3][S_ab][H_ab]
        const double *E1t;     // [ppair][3][H_ab][S_ab]
        const float *pPf;      // [ppair][8] p, 1/p, P hi, P lo (FP32 classes only)
    };

    enum EpilogueMode : int
    {
        kStore = 0,      // write each contracted batch to out[task]
        kJK = 1,         // digest into J/K accumulators (before symmetrisation)
        kRIGamma = 2,    // gamma_P += sum_mn (mn|P) D_mn
        kRIJ = 3,        // J_mn += sum_P (mn|P) d_P
        kD1Store = 4,    // write the 12 derivative blocks
        kD1Grad = 5,     // contract the derivative blocks with the two-particle density
        kRIStore = 6,    // out[P - ri_lo][m][n] = out[P - ri_lo][n][m] = (mn|P), P in [ri_lo, ri_hi); with
                         // flags & kRIPacked only the lower triangle, out[P - ri_lo][i(i+1)/2 + j], j <= i
        kD1GradRI = 7,   // RI-J gradient: derivative blocks contracted with D_mn d_P (3c) or d_P d_Q (2c)
    };
    constexpr int kRIPacked = 8;  // kRIStore flag: packed lower-triangle rows of nao (nao + 1) / 2

    struct QuartetArgs
    {
        PairView bra, ket;
        const double *boys;               // Boys tables [kBoysMaxN + 1][kBoysTerms][kBoysPitch]
        const float *boys_f;              // FP32 Boys table [kBoysMaxN + kBoysTermsF][kBoysPitch], F_j(x_i)
        // task enumeration: explicit (bra pair, ket pair) list, or the implicit Schwarz prefix form:
        // task t belongs to major position i with prefix[i] <= t < prefix[i+1] and pairs with
        // minor position minor_begin[i] + (t - prefix[i]).  major_ket = 1 enumerates ket-major
        // (consecutive tasks share the ket pair), 0 bra-major.
        const uint32_t *list;             // [n_tasks][2] or null
        long long n_tasks;
        const unsigned long long *prefix; // [n_major + 1]
        const uint32_t *major_order;      // pair index of major position i
        const uint32_t *minor_order;      // pair index of minor position j
        const uint32_t *minor_begin;      // first minor position of major position i
        int n_major;
        int major_ket;
        int same_class;                   // bra and ket classes are the same pair list
        // work queue (optional): chunk c covers tasks [chunks[c], chunks[c+1]); workers claim chunk
        // indices from *counter (zeroed before the launch) until n_chunks is reached
        const unsigned long long *chunks;
        long long n_chunks;
        unsigned long long *counter;
        int grid_div;                     // persistent grid: resident blocks per SM / grid_div
        // bra-side structure-of-arrays copies indexed by the task's minor (Schwarz) position
        // (implicit ket-major enumeration only; null = read the per-pair records)
        const uint4 *bra_soa;
        const double *bra_pPs;
        const double *bra_Es;
        const float *bra_Efs;
        const float *bra_pPfs;
        // per-position bra fields (x = first AO of a, y = first AO of b, z = packed-block base,
        // w = block dimension | K << 16 | (a and b the same shell) << 31) and the D_ab blocks gathered
        // in Schwarz order ([mn][position]); J/K launches only
        const int4 *bra_soa2;
        const double *bra_Dab;
        int bra_npos;
        // Schwarz window of implicit enumerations: a task whose Q_bra Q_ket falls outside
        // [q_lo, q_hi) is skipped (plans hand out whole bra groups and leave the test to the
        // kernels); Q by Schwarz position (bra_qpos) or by pair index; ket_qpair null = no test
        const double *bra_qpos;
        const double *bra_qpair;
        const double *ket_qpair;
        double q_lo, q_hi;
        // ket E tiles zero-padded to the DMMA layout of this class (null: stage from Et)
        const double *ket_EtP;
        // epilogue
        int mode;
        int flags;                        // kStore: bit0 swap bra shells, bit1 swap ket shells, bit2 swap bra/ket;
                                          // kRIStore: kRIPacked
        int aux_side;                     // RI modes: 0 = ket is the auxiliary side, 1 = bra, 2 = both
        int ri_lo, ri_hi;                 // kRIStore: the block of auxiliary functions written
        double *out;
        const double *D;
        double *J;
        double *K;
        int nao;
        double *gamma;
        const double *dcoef;
        double *grad;                     // [n_atoms][3]
        int n_atoms;                      // gradient launches: rows of grad
        int *status;                      // error word (non-zero = failure)
        // failure-path check of the bulk-copy waits: > 0 = issue no copy and give up after this many
        // polls (the wait then fails exactly as a stalled copy's would); 0 = normal operation
        int wait_inject;
    };

    // Poll limit of the kernels' barrier waits on bulk copies.
    constexpr int kWaitPolls = 1 << 20;

    // Primitive-pair record as stored in DevPairClass::pP: [p, Px, Py, Pz, 1/p, a, b, 0].
    // x = p, (y, z, w) = P, ip = 1/p.
    struct PQ4
    {
        double x, y, z, w, ip;
    };

    __device__ __forceinline__ PQ4 loadPQ(const double *pP, uint32_t i)
    {
        const double2 *v = reinterpret_cast<const double2 *>(pP + 8 * (size_t)i);
        const double2 a = __ldg(v), b = __ldg(v + 1), c = __ldg(v + 2);
        return {a.x, a.y, b.x, b.y, c.x};
    }

    // One task of the block-per-quartet (group) paths, decoded ahead of its evaluation: pair
    // indices, primitive ranges, whether it lies in the launch's window, and the first bra / ket
    // primitive records.
    struct GroupTask
    {
        uint32_t ib, ik, p0, p1, q0, q1;
        int ok, pad;
        PQ4 P, Q;
    };
    constexpr int kGroupTaskBatch = 32;  // tasks a block decodes at once, one per thread

    // Largest major position i >= lo with prefix[i] <= t, given prefix[lo] <= t: gallops forward
    // from the caller's cursor, so walking consecutive tasks costs a load or two, not a full search.
    __device__ __forceinline__ int advanceMajor(const QuartetArgs &a, long long t, int lo)
    {
        const unsigned long long ut = (unsigned long long)t;
        if (lo + 1 >= a.n_major || __ldg(a.prefix + lo + 1) > ut)
            return lo;
        int step = 1, hi = lo + 1;
        while (hi < a.n_major && __ldg(a.prefix + hi) <= ut)
        {
            lo = hi;
            step <<= 1;
            hi = lo + step;
        }
        if (hi > a.n_major - 1)
            hi = a.n_major - 1;
        while (lo < hi)
        {
            int mid = (lo + hi + 1) >> 1;
            if (__ldg(a.prefix + mid) <= ut)
                lo = mid;
            else
                hi = mid - 1;
        }
        return lo;
    }

    // Task t decoded with a known major position (implicit enumeration only); `pos` receives the
    // minor (Schwarz) position.
    __device__ __forceinline__ void decodeAt(const QuartetArgs &a, long long t, int lo, uint32_t &ib, uint32_t &ik,
                                             uint32_t &pos)
    {
        const uint32_t maj = __ldg(a.major_order + lo);
        pos = __ldg(a.minor_begin + lo) + (uint32_t)((unsigned long long)t - __ldg(a.prefix + lo));
        const uint32_t mnr = __ldg(a.minor_order + pos);
        ib = a.major_ket ? mnr : maj;
        ik = a.major_ket ? maj : mnr;
    }

    // Cursor-based decode: explicit lists index directly; implicit ones advance `cur`.
    __device__ __forceinline__ void decodeCursor(const QuartetArgs &a, long long t, int &cur, uint32_t &ib, uint32_t &ik,
                                                 uint32_t &pos)
    {
        pos = 0;
        if (a.list)
        {
            ib = a.list[2 * t];
            ik = a.list[2 * t + 1];
            return;
        }
        cur = advanceMajor(a, t, cur);
        decodeAt(a, t, cur, ib, ik, pos);
    }
    __device__ __forceinline__ void decodeCursor(const QuartetArgs &a, long long t, int &cur, uint32_t &ib, uint32_t &ik)
    {
        uint32_t pos;
        decodeCursor(a, t, cur, ib, ik, pos);
    }

    __device__ __forceinline__ void decodeTask(const QuartetArgs &a, long long t, uint32_t &ib, uint32_t &ik)
    {
        if (a.list)
        {
            ib = a.list[2 * t];
            ik = a.list[2 * t + 1];
            return;
        }
        int lo = 0, hi = a.n_major - 1;
        while (lo < hi)
        {
            int mid = (lo + hi + 1) >> 1;
            if (__ldg(a.prefix + mid) <= (unsigned long long)t)
                lo = mid;
            else
                hi = mid - 1;
        }
        const uint32_t maj = __ldg(a.major_order + lo);
        const uint32_t mnr = __ldg(a.minor_order + __ldg(a.minor_begin + lo) +
                                   (uint32_t)((unsigned long long)t - __ldg(a.prefix + lo)));
        ib = a.major_ket ? mnr : maj;
        ik = a.major_ket ? maj : mnr;
    }

    // Whether task (bra pair ib at Schwarz position pos, ket pair ik) lies in the launch's window.
    __device__ __forceinline__ bool inWindow(const QuartetArgs &a, uint32_t ib, uint32_t ik, uint32_t pos, bool by_pos)
    {
        if (a.mode == kRIStore)
        {
            // only the auxiliary shells that start inside the block (blocks end at shell boundaries)
            const int P = __ldg(a.aux_side == 0 ? a.ket.info + 8 * ik : a.bra.info + 8 * ib);
            if (P < a.ri_lo || P >= a.ri_hi)
                return false;
        }
        if (!a.ket_qpair)
            return true;
        const double qb = (by_pos && a.bra_qpos) ? __ldg(a.bra_qpos + pos) : __ldg(a.bra_qpair + ib);
        const double qq = qb * __ldg(a.ket_qpair + ik);
        return qq >= a.q_lo && qq < a.q_hi;
    }

    // Decodes task t into g (the thread's cursor `cur` moves forward, as in decodeCursor).
    __device__ __forceinline__ void loadGroupTask(const QuartetArgs &a, long long t, int &cur, GroupTask &g)
    {
        uint32_t ib, ik;
        decodeCursor(a, t, cur, ib, ik);
        const bool ok = inWindow(a, ib, ik, 0, false);
        g.ib = ib;
        g.ik = ik;
        g.ok = ok;
        if (ok)
        {
            const uint32_t p0 = __ldg(a.bra.pofs + ib), p1 = __ldg(a.bra.pofs + ib + 1);
            const uint32_t q0 = __ldg(a.ket.pofs + ik), q1 = __ldg(a.ket.pofs + ik + 1);
            g.p0 = p0;
            g.p1 = p1;
            g.q0 = q0;
            g.q1 = q1;
            if (p0 < p1)
                g.P = loadPQ(a.bra.pP, p0);
            if (q0 < q1)
                g.Q = loadPQ(a.ket.pP, q0);
        }
    }

    // Degeneracy weight of a unique quartet: 1/2 for each coinciding shell pair / pair pair.
    __device__ __forceinline__ double quartetWeight(const QuartetArgs &a, bool bra_same_shell, uint32_t ib,
                                                    uint32_t ik)
    {
        const int32_t *ki = a.ket.info + 8 * ik;
        double f = bra_same_shell ? 0.5 : 1.0;
        if (ki[4] == ki[5])
            f *= 0.5;
        if (a.same_class && ib == ik)
            f *= 0.5;
        return f;
    }

    __device__ __forceinline__ double quartetWeight(const QuartetArgs &a, uint32_t ib, uint32_t ik)
    {
        const int32_t *bi = a.bra.info + 8 * ib;
        const int32_t *ki = a.ket.info + 8 * ik;
        double f = 1.0;
        if (bi[4] == bi[5])
            f *= 0.5;
        if (ki[4] == ki[5])
            f *= 0.5;
        if (a.same_class && ib == ik)
            f *= 0.5;
        return f;
    }

    // e^{-x} for 0 <= x <= 700 using only FP64 FMAs and integer adds (no special-function or
    // conversion instructions): Cody-Waite reduction x = k ln2 - r with k = round(x / ln2) taken
    // from the low mantissa bits of x/ln2 + 1.5*2^52, e^{-r} by its degree-13 Taylor polynomial
    // (|r| <= ln2/2, truncation < 2e-17), and 2^-k applied to the exponent field.  Within ~1 ulp
    // of exp().
    __device__ __forceinline__ double expNeg(double x)
    {
        constexpr double kMagic = 6755399441055744.0;  // 1.5 * 2^52
        const double t = fma(-x, 1.4426950408889634074, kMagic);
        const double kd = t - kMagic;
        const long long k = __double_as_longlong(t) - __double_as_longlong(kMagic);
        double r = fma(kd, -0.6931471805599453094, -x);
        r = fma(kd, -2.319046813846299558e-17, r);
        double p = 1.0 / 6227020800.0;  // 1/13!
        p = fma(p, r, 1.0 / 479001600.0);
        p = fma(p, r, 1.0 / 39916800.0);
        p = fma(p, r, 1.0 / 3628800.0);
        p = fma(p, r, 1.0 / 362880.0);
        p = fma(p, r, 1.0 / 40320.0);
        p = fma(p, r, 1.0 / 5040.0);
        p = fma(p, r, 1.0 / 720.0);
        p = fma(p, r, 1.0 / 120.0);
        p = fma(p, r, 1.0 / 24.0);
        p = fma(p, r, 1.0 / 6.0);
        p = fma(p, r, 0.5);
        p = fma(p, r, 1.0);
        p = fma(p, r, 1.0);
        return __longlong_as_double(__double_as_longlong(p) + k * 4503599627370496LL);
    }

    // Shared-memory load of a double / float (explicit ld.shared, so table lookups never fall back
    // to generic addressing).
    __device__ __forceinline__ double ldsD(const double *p)
    {
        double v;
        asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"((unsigned)__cvta_generic_to_shared(p)));
        return v;
    }
    __device__ __forceinline__ float ldsF(const float *p)
    {
        float v;
        asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"((unsigned)__cvta_generic_to_shared(p)));
        return v;
    }

    // Copies the order-N Boys table (kBoysTerms x kBoysPitch doubles, or the FP32 one) into shared
    // memory; the caller synchronises the block afterwards.
    __device__ __forceinline__ void stageBoys(const double *__restrict__ tables, int N, double *dst)
    {
        const double *src = tables + (size_t)N * kBoysTerms * kBoysPitch;
        for (int e = threadIdx.x; e < kBoysTerms * kBoysPitch; e += blockDim.x)
            dst[e] = __ldg(src + e);
    }
    // FP32: rows F_0 .. F_{N + kBoysTermsF - 1} of the unscaled table.
    __device__ __forceinline__ void stageBoys(const float *__restrict__ table, int N, float *dst)
    {
        for (int e = threadIdx.x; e < (N + kBoysTermsF) * kBoysPitch; e += blockDim.x)
            dst[e] = __ldg(table + e);
    }

    // Boys function F_n(x), n = 0..N.  Reference method (src/lible/ints/boys_function.hpp:68-109):
    // Taylor expansion of F_N about a grid point followed by downward recursion, and for x > 30 the
    // asymptotic F_0 = sqrt(pi/x)/2 with upward recursion.  Here the expansion point is the nearest
    // integer (|x - x_i| <= 1/2, 16 terms; table layout in lible_math.hpp), found with the
    // 1.5*2^52 rounding trick, and e^{-x} comes from expNeg(), so the only special-function
    // instruction on this path is the asymptote's rsqrt.  `tab` is the order-N table, in shared
    // memory when SMEM (staged by stageBoys), else in global memory (a.boys + N * terms * pitch).
    template <int N, bool SMEM>
    __device__ __forceinline__ void boysF(double x, const double *__restrict__ tab, double *F)
    {
        if (x > kBoysLargeX)
        {
            // sqrt(pi)/2 * x^{-1/2}, then F_k = F_{k-1} (k - 1/2) / x
            const double rs = rsqrt(x);
            const double rx = rs * rs;
            F[0] = 0.88622692545275801365 * rs;
#pragma unroll
            for (int k = 1; k <= N; k++)
                F[k] = F[k - 1] * ((k - 0.5) * rx);
            return;
        }
        constexpr double kMagic = 6755399441055744.0;  // 1.5 * 2^52
        const double t = x + kMagic;                    // nearest integer, exactly
        const int iv = (int)(__double_as_longlong(t) - __double_as_longlong(kMagic));
        const double m = (t - kMagic) - x;              // x_i - x
        const double *c = tab + iv;
        double s = SMEM ? ldsD(c + (kBoysTerms - 1) * kBoysPitch) : __ldg(c + (kBoysTerms - 1) * kBoysPitch);
#pragma unroll
        for (int k = kBoysTerms - 2; k >= 0; k--)
            s = fma(s, m, SMEM ? ldsD(c + k * kBoysPitch) : __ldg(c + k * kBoysPitch));
        F[N] = s;
        const double ex = expNeg(x);
        const double x2 = 2.0 * x;
#pragma unroll
        for (int k = N - 1; k >= 0; k--)
            F[k] = (x2 * F[k + 1] + ex) * (1.0 / (2 * k + 1));
    }

    // The Boys function for quartets evaluated in FP32, F_0..F_N as floats.  The large-x asymptote
    // stays FP64 (its inverse square root and upward products are formed in double and rounded
    // once).  Below x = 30 every order n comes from its own Taylor sum about the nearest integer,
    // sum_k F_{n+k}(x_i) (x_i - x)^k / k! with kBoysTermsF terms read from the staged FP32 table
    // (rows F_0 .. F_{N+kBoysTermsF-1}), so no recursion is evaluated in single precision.
    template <int N>
    __device__ __forceinline__ void boysF32(float x, const float *__restrict__ tabf, float *F)
    {
        if (x > (float)kBoysLargeX)
        {
            const double xd = x;
            const double rs = rsqrt(xd);
            const double rx = rs * rs;
            double f = 0.88622692545275801365 * rs;
            F[0] = (float)f;
#pragma unroll
            for (int k = 1; k <= N; k++)
            {
                f *= (k - 0.5) * rx;
                F[k] = (float)f;
            }
            return;
        }
        constexpr int T = kBoysTermsF;
        const int iv = __float2int_rn(x);
        const float m = (float)iv - x;
        float Fj[N + T];
#pragma unroll
        for (int j = 0; j < N + T; j++)
            Fj[j] = ldsF(tabf + j * kBoysPitch + iv);
        float mk[T];
#pragma unroll
        for (int k = 1; k < T; k++)
            mk[k] = m * (1.0f / k);
#pragma unroll
        for (int n = 0; n <= N; n++)
        {
            float s = Fj[n + T - 1];
#pragma unroll
            for (int k = T - 1; k >= 1; k--)
                s = fmaf(mk[k], s, Fj[n + k - 1]);
            F[n] = s;
        }
    }

    // Hermite Coulomb integrals R_{tuv} = R^{(0)}_{tuv} for t+u+v <= L in registers, by the
    // McMurchie-Davidson recursion R^{(n)}_{t+1,u,v} = t R^{(n+1)}_{t-1,u,v} + X R^{(n+1)}_{tuv}
    // (Helgaker, Jorgensen, Olsen 9.9.18-9.9.20) started from R^{(n)}_{000} = (-2 alpha)^n F_n.
    // One buffer is updated in place, highest order first, so every read still sees level n+1.
    // Reference: src/lible/ints/rints.hpp:112-175.  R is indexed by the combined Hermite index.
    template <int L, typename T>
    __device__ __forceinline__ void hermiteR(T m2a, const T *F, T X, T Y, T Z, T *R)
    {
        T pw[L + 1];
        pw[0] = T(1);
#pragma unroll
        for (int n = 1; n <= L; n++)
            pw[n] = pw[n - 1] * m2a;
        R[0] = F[L] * pw[L];
#pragma unroll
        for (int n = L - 1; n >= 0; n--)
        {
#pragma unroll
            for (int m = L - n; m >= 1; m--)
            {
#pragma unroll
                for (int t = m; t >= 0; t--)
                {
#pragma unroll
                    for (int u = m - t; u >= 0; u--)
                    {
                        const int v = m - t - u;
                        const int id = hermIndex(t, u, v);
                        if (t > 0)
                        {
                            T r = X * R[hermIndex(t - 1, u, v)];
                            if (t > 1)
                                r += T(t - 1) * R[hermIndex(t - 2, u, v)];
                            R[id] = r;
                        }
                        else if (u > 0)
                        {
                            T r = Y * R[hermIndex(t, u - 1, v)];
                            if (u > 1)
                                r += T(u - 1) * R[hermIndex(t, u - 2, v)];
                            R[id] = r;
                        }
                        else
                        {
                            T r = Z * R[hermIndex(t, u, v - 1)];
                            if (v > 1)
                                r += T(v - 1) * R[hermIndex(t, u, v - 2)];
                            R[id] = r;
                        }
                    }
                }
            }
            R[0] = F[n] * pw[n];
        }
    }

    // (t, u, v) of a combined Hermite index.
    __device__ __forceinline__ void hermTuv(int e, int &t, int &u, int &v)
    {
        int n = 0;
        while (nherm(n) <= e)
            n++;
        int c = e - nherm(n - 1);
        int jk = 0;
        while ((jk + 1) * (jk + 2) / 2 <= c)
            jk++;
        v = c - jk * (jk + 1) / 2;
        u = jk - v;
        t = n - jk;
    }
}
