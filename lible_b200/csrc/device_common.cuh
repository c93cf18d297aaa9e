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
        const double *pP;      // [ppair][4] p, Px, Py, Pz
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
        const double *boys;               // Boys grid [kBoysRows][kBoysCols]
        // task enumeration: explicit (bra pair, ket pair) list, or implicit Schwarz prefix form
        const uint32_t *list;             // [n_tasks][2] or null
        long long n_tasks;
        const unsigned long long *prefix; // [n_bra + 1]
        const uint32_t *bra_order;        // bra pair index of bra position i
        const uint32_t *ket_order;        // ket pair index of ket position j
        const uint32_t *ket_begin;        // first ket position of bra position i
        int n_bra;
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

    // Primitive-pair record: total exponent p and centre P = (x, y, z) in bohr (named w for z).
    struct PQ4
    {
        double x, y, z, w;
    };

    __device__ __forceinline__ PQ4 loadPQ(const double *pP, uint32_t i)
    {
        const double2 *v = reinterpret_cast<const double2 *>(pP) + 2 * (size_t)i;
        const double2 lo = __ldg(v), hi = __ldg(v + 1);
        return {lo.x, lo.y, hi.x, hi.y};
    }

    __device__ __forceinline__ void decodeTask(const QuartetArgs &a, long long t, uint32_t &ib, uint32_t &ik)
    {
        if (a.list)
        {
            ib = a.list[2 * t];
            ik = a.list[2 * t + 1];
            return;
        }
        int lo = 0, hi = a.n_bra - 1;
        while (lo < hi)
        {
            int mid = (lo + hi + 1) >> 1;
            if (a.prefix[mid] <= (unsigned long long)t)
                lo = mid;
            else
                hi = mid - 1;
        }
        ib = a.bra_order[lo];
        ik = a.ket_order[a.ket_begin[lo] + (uint32_t)((unsigned long long)t - a.prefix[lo])];
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

    // Boys function F_n(x), n = 0..N: Taylor expansion of F_N about the nearest lower grid point
    // (7 terms, step 0.01) followed by downward recursion; exact at x = 0; for x > 30 the
    // asymptotic F_0 = sqrt(pi/x)/2 and upward recursion.  Same method and constants as
    // src/lible/ints/boys_function.hpp:68-109.
    template <int N>
    __device__ __forceinline__ void boysF(double x, const double *__restrict__ grid, double *F)
    {
        if (x > kBoysLargeX)
        {
            F[0] = 0.5 * sqrt(M_PI / x);
            const double rx = 1.0 / x;
#pragma unroll
            for (int k = 1; k <= N; k++)
                F[k] = F[k - 1] * (k - 0.5) * rx;
            return;
        }
        const int iv = (int)(x / kBoysStep);
        const double dx = x - iv * kBoysStep;
        const double *row = grid + (size_t)iv * kBoysCols + N;
        double s = __ldg(row);
        double pk = 1.0, fact = 1.0;
#pragma unroll
        for (int k = 1; k < 7; k++)
        {
            pk *= -dx;
            fact *= k;
            s += __ldg(row + k) * pk / fact;
        }
        F[N] = s;
        const double ex = exp(-x);
#pragma unroll
        for (int k = N - 1; k >= 0; k--)
            F[k] = (2.0 * x * F[k + 1] + ex) / (2 * k + 1);
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
