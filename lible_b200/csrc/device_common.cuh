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
    };

    enum EpilogueMode : int
    {
        kStore = 0,      // write each contracted batch to out[task]
        kJK = 1,         // digest into J/K accumulators (before symmetrisation)
        kRIGamma = 2,    // gamma_P += sum_mn (mn|P) D_mn
        kRIJ = 3,        // J_mn += sum_P (mn|P) d_P
        kD1Store = 4,    // write the 12 derivative blocks
        kD1Grad = 5,     // contract the derivative blocks with the two-particle density
    };

    struct QuartetArgs
    {
        PairView bra, ket;
        const double *boys;               // Boys tables [kBoysMaxN + 1][kBoysRows][kBoysTerms]
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
        // epilogue
        int mode;
        int flags;                        // kStore: bit0 swap bra shells, bit1 swap ket shells, bit2 swap bra/ket
        int aux_side;                     // RI modes: 0 = ket is the auxiliary side, 1 = bra
        double *out;
        const double *D;
        double *J;
        double *K;
        int nao;
        double *gamma;
        const double *dcoef;
        double *grad;                     // [n_atoms][3]
        int *status;                      // error word (non-zero = failure)
    };

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

    // Task t decoded with a known major position (implicit enumeration only).
    __device__ __forceinline__ void decodeAt(const QuartetArgs &a, long long t, int lo, uint32_t &ib, uint32_t &ik)
    {
        const uint32_t maj = __ldg(a.major_order + lo);
        const uint32_t mnr = __ldg(a.minor_order + __ldg(a.minor_begin + lo) +
                                   (uint32_t)((unsigned long long)t - __ldg(a.prefix + lo)));
        ib = a.major_ket ? mnr : maj;
        ik = a.major_ket ? maj : mnr;
    }

    // Cursor-based decode: explicit lists index directly; implicit ones advance `cur`.
    __device__ __forceinline__ void decodeCursor(const QuartetArgs &a, long long t, int &cur, uint32_t &ib, uint32_t &ik)
    {
        if (a.list)
        {
            ib = a.list[2 * t];
            ik = a.list[2 * t + 1];
            return;
        }
        cur = advanceMajor(a, t, cur);
        decodeAt(a, t, cur, ib, ik);
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

    // Degeneracy weight of a unique quartet: 1/2 for each coinciding shell pair / pair pair.
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

    // Boys function F_n(x), n = 0..N.  Reference method (src/lible/ints/boys_function.hpp:68-109):
    // Taylor expansion of F_N about a grid point (7 terms, step 0.01) followed by downward
    // recursion, and for x > 30 the asymptotic F_0 = sqrt(pi/x)/2 with upward recursion.
    // Here the expansion point is the nearest grid point (|x - x_i| <= 0.005, half the reference's
    // truncation interval), found with the 1.5*2^52 rounding trick, and e^{-x} comes from expNeg(),
    // so the only special-function instruction on this path is the asymptote's rsqrt.
    template <int N>
    __device__ __forceinline__ void boysF(double x, const double *__restrict__ grid, double *F)
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
        const double t = fma(x, 1.0 / kBoysStep, kMagic);
        const long long iv = __double_as_longlong(t) - __double_as_longlong(kMagic);
        const double m = fma(t - kMagic, kBoysStep, -x);  // x_i - x
        // row of 10 coefficients F_{N+k}(x_i)/k! (80 bytes, 16-byte aligned)
        const double2 *row = reinterpret_cast<const double2 *>(grid + ((size_t)N * kBoysRows + iv) * kBoysTerms);
        static_assert(kBoysTerms == 10, "row load below assumes 10 terms");
        const double2 c01 = __ldg(row), c23 = __ldg(row + 1), c45 = __ldg(row + 2), c67 = __ldg(row + 3),
                      c89 = __ldg(row + 4);
        double s = fma(c89.y, m, c89.x);
        s = fma(s, m, c67.y);
        s = fma(s, m, c67.x);
        s = fma(s, m, c45.y);
        s = fma(s, m, c45.x);
        s = fma(s, m, c23.y);
        s = fma(s, m, c23.x);
        s = fma(s, m, c01.y);
        s = fma(s, m, c01.x);
        F[N] = s;
        const double ex = expNeg(x);
        const double x2 = 2.0 * x;
#pragma unroll
        for (int k = N - 1; k >= 0; k--)
            F[k] = (x2 * F[k + 1] + ex) * (1.0 / (2 * k + 1));
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
