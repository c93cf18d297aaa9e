// Index conventions and small recurrences shared by host and device code.
//
// Conventions (identical to the reference, because they decide per-integral parity):
//  * Cartesian order of a shell with angular momentum l: x-major descending,
//    (l,0,0), (l-1,1,0), (l-1,0,1), ... (src/lible/ints/utils.cpp:33-47);
//    index(i,j,k) = (j+k)(j+k+1)/2 + k (src/lible/ints/utils.hpp:27-31).
//  * Hermite order for a pair of total angular momentum L: by n = t+u+v ascending, then the
//    Cartesian order inside one n (src/lible/ints/utils.cpp:92-104, rints.hpp:58-69).  This order
//    does not depend on L, so one "combined" index serves every class.
//  * Spherical order inside a shell: m = 0, +1, -1, +2, -2, ... (src/lible/ints/spherical_trafo.cpp:13-60).
#pragma once

#include <cmath>
#include <cstddef>

#if defined(__CUDACC__)
#define LB_HD __host__ __device__ __forceinline__
#else
#define LB_HD inline
#endif

namespace lible_b200
{
    constexpr int kMaxL = 5;          // highest shell angular momentum handled (aux h shells)
    constexpr int kMaxLPair = 2 * kMaxL;
    constexpr int kMaxLTotal = 14;    // highest L of a quartet (+1 for first derivatives)
    // Boys tables: for every order N = 0..kBoysMaxN a table of Taylor coefficients of F_N about
    // the integers x_i = 0, 1, ..., 30: c_N[k][i] = F_{N+k}(x_i) / k!, k = 0..kBoysTerms-1, stored
    // term-major with a row pitch of kBoysPitch (index k * kBoysPitch + i; entry 31 repeats 30).
    // Expanding about the nearest integer (|x - x_i| <= 1/2) with 16 terms truncates below
    // 0.5^16/16! < 1e-18 relative.  One order is 4 KB, small enough to be staged in shared memory,
    // and the 31 possible rows of a warp's lookups fall on few distinct words (mostly broadcasts).
    // The reference grid is finer (step 0.01, 7 terms about the lower point,
    // src/lible/ints/boys_function.hpp:112-122); both are accurate to the last bits.
    // The FP32 table holds F_j(x_i) unscaled, j < kBoysMaxN + kBoysTermsF; FP32 quartets sum
    // kBoysTermsF Taylor terms per order (truncation 0.5^10/10! < 3e-10).
    constexpr int kBoysMaxN = 14;
    constexpr int kBoysTerms = 16;
    constexpr int kBoysTermsF = 10;
    constexpr int kBoysPitch = 32;
    constexpr int kBoysRows = 31;
    constexpr int kBoysCols = 32;     // F_n for n = 0 .. 31 computed when building the tables
    constexpr double kBoysLargeX = 30.0;
    constexpr double kPrimitiveThreshold = 1e-15;   // src/lible/ints/shell_pair_data.hpp:57
    constexpr double kBohrToAngstrom = 0.5291772083; // src/lible/ints/defs.hpp:9
    constexpr double kAngstromToBohr = 1.0 / kBohrToAngstrom;

    LB_HD constexpr int nsph(int l) { return 2 * l + 1; }
    LB_HD constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }
    // Number of Hermite functions with t+u+v <= l.
    LB_HD constexpr int nherm(int l) { return l < 0 ? 0 : (l + 1) * (l + 2) * (l + 3) / 6; }
    LB_HD constexpr int cartIndex(int j, int k) { return (j + k) * (j + k + 1) / 2 + k; }
    // Combined Hermite index of (t, u, v).
    LB_HD constexpr int hermIndex(int t, int u, int v)
    {
        return nherm(t + u + v - 1) + cartIndex(u, v);
    }

    // One-dimensional Hermite expansion behind the closed form of R_tuv: with g_n = (-2 alpha)^n F_n
    // and d/dX g_n = X g_{n+1}, d^t/dX^t g_0 = sum_{a <= t/2} h(t, a) X^{t-2a} g_{t-a} with
    // h(t, a) = t! / (a! (t - 2a)! 2^a).  Entry hermAxisOffset(t) + a of the table holds h(t, a)
    // and the power t - 2a, for t = 0..kMaxLTotal.
    LB_HD constexpr int hermAxisOffset(int t) { return (t / 2) * (t / 2 + 1) + ((t & 1) ? t / 2 + 1 : 0); }
    constexpr int kHermAxisEntries = hermAxisOffset(kMaxLTotal + 1);
    struct HermAxisTable
    {
        double c[kHermAxisEntries];
        int p[kHermAxisEntries];
    };
    constexpr HermAxisTable makeHermAxisTable()
    {
        HermAxisTable tab{};
        for (int t = 0; t <= kMaxLTotal; t++)
            for (int a = 0; 2 * a <= t; a++)
            {
                double h = 1.0;  // h(t, i + 1) = h(t, i) (t - 2i) (t - 2i - 1) / (2 (i + 1)), exact integers
                for (int i = 0; i < a; i++)
                    h = h * (t - 2 * i) * (t - 2 * i - 1) / (2.0 * (i + 1));
                tab.c[hermAxisOffset(t) + a] = h;
                tab.p[hermAxisOffset(t) + a] = t - 2 * a;
            }
        return tab;
    }

    // Derivative classes whose J/K-gradient contraction runs in registers (eriD1RegKernel): a group
    // of g threads per quartet, each owning S_cd / g ket columns, with its Gamma-weighted bra
    // coefficients (4 x H_ab x S_cd / g values) and the R vector to order L + 1 within 170 doubles
    // (the steady-state (H2O)_8 cc-pVTZ gradient measured 0.85 s at 120, 0.73 s at 170, 0.82 s at 230:
    // beyond 170 the spills outweigh the block kernel's synchronisation).  Returns the smallest such
    // g (a divisor of S_cd), 0 when none fits.
    LB_HD constexpr int d1RegisterGroup(int la, int lb, int lc, int ld)
    {
        const int scd = nsph(lc) * nsph(ld);
        for (int g = 1; g <= 32 && g <= scd; g++)
            if (scd % g == 0 && 4 * nherm(la + lb) * (scd / g) + nherm(la + lb + lc + ld + 1) <= 170)
                return g;
        return 0;
    }
    LB_HD constexpr bool d1RegisterClass(int la, int lb, int lc, int ld)
    {
        return d1RegisterGroup(la, lb, lc, ld) > 0;
    }

    // Hermite expansion coefficients of a primitive pair along one axis, McMurchie-Davidson
    // recurrences (Helgaker, Jorgensen, Olsen, Molecular Electronic-Structure Theory, 9.5.6-9.5.7).
    // E[i][j][t] is stored at E[(i * (lb + 1) + j) * (la + lb + 1) + t].  `one_o_2p` = 1/(2p),
    // `pa` = P - A, `pb` = P - B, `kab` = exp(-mu (A-B)^2) on this axis.
    // Follows src/lible/ints/ecoeffs.cpp:33-68.
    LB_HD void hermiteE(int la, int lb, double one_o_2p, double pa, double pb, double kab, double *E)
    {
        const int nt = la + lb + 1;
        for (int x = 0; x < (la + 1) * (lb + 1) * nt; x++)
            E[x] = 0.0;
        auto at = [&](int i, int j, int t) -> double & { return E[(i * (lb + 1) + j) * nt + t]; };
        at(0, 0, 0) = kab;
        for (int i = 1; i <= la; i++)
            for (int t = 0; t <= i; t++)
            {
                double v = pa * at(i - 1, 0, t);
                if (t > 0)
                    v += one_o_2p * at(i - 1, 0, t - 1);
                if (t + 1 <= i - 1)
                    v += (t + 1) * at(i - 1, 0, t + 1);
                at(i, 0, t) = v;
            }
        for (int j = 1; j <= lb; j++)
            for (int i = 0; i <= la; i++)
                for (int t = 0; t <= i + j; t++)
                {
                    double v = pb * at(i, j - 1, t);
                    if (t > 0)
                        v += one_o_2p * at(i, j - 1, t - 1);
                    if (t + 1 <= i + j - 1)
                        v += (t + 1) * at(i, j - 1, t + 1);
                    at(i, j, t) = v;
                }
    }

    // Derivative of E[i][j][t] with respect to the separation R = A - B on this axis, at fixed
    // exponents.  With PA = -(b/p) R, PB = (a/p) R and K = exp(-mu R^2) the product rule applied
    // to the recurrences above gives the same three-term form plus the derivative of PA / PB.
    // Follows src/lible/ints/ecoeffs.cpp:70-111.
    LB_HD void hermiteE1(int la, int lb, double a, double b, double rab, const double *E, double *E1)
    {
        const double p = a + b;
        const double one_o_2p = 0.5 / p;
        const double pa = -(b / p) * rab, pb = (a / p) * rab;
        const int nt = la + lb + 1;
        for (int x = 0; x < (la + 1) * (lb + 1) * nt; x++)
            E1[x] = 0.0;
        auto e0 = [&](int i, int j, int t) -> double { return E[(i * (lb + 1) + j) * nt + t]; };
        auto at = [&](int i, int j, int t) -> double & { return E1[(i * (lb + 1) + j) * nt + t]; };
        at(0, 0, 0) = -2.0 * (a * b / p) * rab * e0(0, 0, 0);
        for (int i = 1; i <= la; i++)
            for (int t = 0; t <= i; t++)
            {
                double v = pa * at(i - 1, 0, t) - (b / p) * e0(i - 1, 0, t);
                if (t > 0)
                    v += one_o_2p * at(i - 1, 0, t - 1);
                if (t + 1 <= i - 1)
                    v += (t + 1) * at(i - 1, 0, t + 1);
                at(i, 0, t) = v;
            }
        for (int j = 1; j <= lb; j++)
            for (int i = 0; i <= la; i++)
                for (int t = 0; t <= i + j; t++)
                {
                    double v = pb * at(i, j - 1, t) + (a / p) * e0(i, j - 1, t);
                    if (t > 0)
                        v += one_o_2p * at(i, j - 1, t - 1);
                    if (t + 1 <= i + j - 1)
                        v += (t + 1) * at(i, j - 1, t + 1);
                    at(i, j, t) = v;
                }
    }

    // Second derivative of the Hermite coefficients with respect to the same axis' A - B, from the
    // first (E1, hermiteE1) and the plain ones (E): differentiating the hermiteE1 recurrences once
    // more gives
    //   E2[0][0][0] = -2 (ab/p) (R E1[0][0][0] + E[0][0][0]),
    //   E2[i][0][t] = -(b/p) (R E2[i-1][0][t] + 2 E1[i-1][0][t]) + E2[i-1][0][t-1] / 2p + (t+1) E2[i-1][0][t+1],
    //   E2[i][j][t] =  (a/p) (R E2[i][j-1][t] + 2 E1[i][j-1][t]) + E2[i][j-1][t-1] / 2p + (t+1) E2[i][j-1][t+1]
    // (the reference's ecoeffsRecurrence2_n2, src/lible/ints/ecoeffs.cpp:113-160).  Same layout as E.
    LB_HD void hermiteE2(int la, int lb, double a, double b, double rab, const double *E, const double *E1,
                         double *E2)
    {
        const double p = a + b;
        const double one_o_2p = 0.5 / p;
        const int nt = la + lb + 1;
        for (int x = 0; x < (la + 1) * (lb + 1) * nt; x++)
            E2[x] = 0.0;
        auto e0 = [&](int i, int j, int t) -> double { return E[(i * (lb + 1) + j) * nt + t]; };
        auto e1 = [&](int i, int j, int t) -> double { return E1[(i * (lb + 1) + j) * nt + t]; };
        auto at = [&](int i, int j, int t) -> double & { return E2[(i * (lb + 1) + j) * nt + t]; };
        at(0, 0, 0) = -2.0 * (a * b / p) * (rab * e1(0, 0, 0) + e0(0, 0, 0));
        for (int i = 1; i <= la; i++)
            for (int t = 0; t <= i; t++)
            {
                double v = -(b / p) * (rab * at(i - 1, 0, t) + 2.0 * e1(i - 1, 0, t));
                if (t > 0)
                    v += one_o_2p * at(i - 1, 0, t - 1);
                if (t + 1 <= i - 1)
                    v += (t + 1) * at(i - 1, 0, t + 1);
                at(i, 0, t) = v;
            }
        for (int j = 1; j <= lb; j++)
            for (int i = 0; i <= la; i++)
                for (int t = 0; t <= i + j; t++)
                {
                    double v = (a / p) * (rab * at(i, j - 1, t) + 2.0 * e1(i, j - 1, t));
                    if (t > 0)
                        v += one_o_2p * at(i, j - 1, t - 1);
                    if (t + 1 <= i + j - 1)
                        v += (t + 1) * at(i, j - 1, t + 1);
                    at(i, j, t) = v;
                }
    }
}
