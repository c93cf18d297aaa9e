// Host-side tables: real solid-harmonic (spherical) transformation and the Boys-function grid.
#include "engine.hpp"

#include <algorithm>
#include <stdexcept>

namespace lible_b200
{
    namespace
    {
        double binom(int n, int k)
        {
            if (k < 0 || k > n)
                return 0.0;
            double r = 1.0;
            for (int i = 1; i <= k; i++)
                r = r * (n - k + i) / i;
            return r;
        }

        double factorial(int n)
        {
            double r = 1.0;
            for (int i = 2; i <= n; i++)
                r *= i;
            return r;
        }
    }

    // Cartesian -> real solid harmonic coefficients for shell l, built from the closed form of
    // Helgaker, Jorgensen, Olsen, Molecular Electronic-Structure Theory, eqs. 6.4.47-6.4.50:
    //   S_lm = N_lm sum_t sum_u sum_v C^{lm}_{tuv} x^{2t+|m|-2(u+v)} y^{2(u+v)} z^{l-2t-|m|}
    // with C = (-1)^{t+v-v_m} (1/4)^t binom(l,t) binom(l-t,|m|+t) binom(t,u) binom(|m|,2v),
    // v_m = 0 (m >= 0) or 1/2 (m < 0), N_lm = sqrt(2 (l+|m|)! (l-|m|)! / 2^{delta_m0}) / (2^|m| l!).
    // Rows are ordered m = 0, +1, -1, +2, -2, ... as in the reference
    // (src/lible/ints/spherical_trafo.cpp:9-690, whose printed values are these to 14 decimals).
    std::vector<SphTerm> sphericalTrafo(int l)
    {
        if (l < 0 || l > 8)
            throw std::runtime_error("sphericalTrafo(): angular momentum out of range");
        std::vector<SphTerm> out;
        for (int row = 0; row < 2 * l + 1; row++)
        {
            int m = (row == 0) ? 0 : ((row % 2 == 1) ? (row + 1) / 2 : -(row / 2));
            int am = m < 0 ? -m : m;
            double nlm = std::sqrt(2.0 * factorial(l + am) * factorial(l - am) / (m == 0 ? 2.0 : 1.0)) /
                         (std::pow(2.0, am) * factorial(l));
            // accumulate per Cartesian component
            std::vector<double> coef(ncart(l), 0.0);
            for (int t = 0; t <= (l - am) / 2; t++)
                for (int u = 0; u <= t; u++)
                {
                    // 2v runs over even values (m >= 0) or odd values (m < 0) up to |m|
                    for (int two_v = (m < 0 ? 1 : 0); two_v <= am; two_v += 2)
                    {
                        int vv = two_v / 2;  // integer part; exponent of y uses 2(u+v)
                        double sign_exp = t + (m < 0 ? (two_v - 1) / 2 : two_v / 2);
                        double c = ((int)sign_exp % 2 == 0 ? 1.0 : -1.0) * std::pow(0.25, t) * binom(l, t) *
                                   binom(l - t, am + t) * binom(t, u) * binom(am, two_v);
                        int py = 2 * u + two_v;
                        int px = 2 * t + am - 2 * u - two_v;
                        int pz = l - 2 * t - am;
                        (void)vv;
                        if (px < 0 || py < 0 || pz < 0)
                            continue;
                        coef[cartIndex(py, pz)] += nlm * c;
                    }
                }
            for (int c = 0; c < ncart(l); c++)
                if (coef[c] != 0.0)
                    out.push_back({row, c, coef[c]});
        }
        return out;
    }

    // Host evaluation with the same method and tables as the device boysF<N>() (device_common.cuh).
    void boysHost(int n, double x, const std::vector<double> &tables, double *F)
    {
        if (x > kBoysLargeX)
        {
            F[0] = 0.5 * std::sqrt(M_PI / x);
            for (int k = 1; k <= n; k++)
                F[k] = F[k - 1] * (k - 0.5) / x;
            return;
        }
        const int iv = (int)std::nearbyint(x);
        const double m = iv - x;
        const double *c = tables.data() + (size_t)n * kBoysTerms * kBoysPitch + iv;
        double s = c[(kBoysTerms - 1) * kBoysPitch];
        for (int k = kBoysTerms - 2; k >= 0; k--)
            s = std::fma(s, m, c[k * kBoysPitch]);
        F[n] = s;
        const double ex = std::exp(-x);
        for (int k = n - 1; k >= 0; k--)
            F[k] = (2.0 * x * F[k + 1] + ex) / (2 * k + 1);
    }

    // Boys function tables (layout in lible_math.hpp).  At each integer x_i, F_n(x_i) for
    // n = 0..kBoysCols-1 is computed as the reference builds its grid: the top order by the
    // convergent series F_N(x) = e^{-x} sum_i x^i / ((N+1/2)(N+3/2)...(N+i+1/2)) stopped when a term
    // falls below 1e-17 of the sum, lower orders by downward recursion F_n = (2x F_{n+1} + e^{-x}) / (2n+1)
    // (Helgaker, Jorgensen, Olsen, eqs. 9.8.11-9.8.14; src/lible/ints/boys_function.cpp:40-69).
    std::vector<double> boysGrid()
    {
        std::vector<double> g((size_t)(kBoysMaxN + 1) * kBoysTerms * kBoysPitch, 0.0);
        const int nmax = kBoysCols - 1;
        std::vector<double> col(kBoysCols);
        for (int i = 0; i < kBoysPitch; i++)
        {
            const double x = std::min(i, kBoysRows - 1);
            double term = 1.0 / (2.0 * nmax + 1.0);
            double sum = term;
            for (int k = 1;; k++)
            {
                term *= x / (nmax + 0.5 + k);
                sum += term;
                if (std::fabs(term) < 1e-17 * sum)
                    break;
            }
            const double ex = std::exp(-x);
            col[nmax] = ex * sum;
            for (int n = nmax - 1; n >= 0; n--)
                col[n] = (2.0 * x * col[n + 1] + ex) / (2 * n + 1);
            for (int N = 0; N <= kBoysMaxN; N++)
            {
                double fact = 1.0;
                for (int k = 0; k < kBoysTerms; k++)
                {
                    if (k > 0)
                        fact *= k;
                    g[((size_t)N * kBoysTerms + k) * kBoysPitch + i] = col[N + k] / fact;
                }
            }
        }
        return g;
    }

    // The FP32 table: F_j(x_i) for j = 0 .. kBoysMaxN + kBoysTermsF - 1 at the same integer points,
    // unscaled and rounded to float, layout [j][kBoysPitch].  FP32 quartets evaluate every order
    // n <= N from its own Taylor sum sum_k F_{n+k}(x_i) (x_i - x)^k / k!, so no recursion runs in FP32.
    std::vector<float> boysGridF()
    {
        const std::vector<double> g = boysGrid();
        const int nj = kBoysMaxN + kBoysTermsF;
        std::vector<float> f((size_t)nj * kBoysPitch);
        for (int j = 0; j < nj; j++)
        {
            // F_j(x_i) = c_N[k][i] k! with N + k = j, taken from the lowest available order N
            const int N = std::max(0, j - (kBoysTerms - 1));
            const int k = j - N;
            double fact = 1.0;
            for (int q = 2; q <= k; q++)
                fact *= q;
            for (int i = 0; i < kBoysPitch; i++)
                f[(size_t)j * kBoysPitch + i] = (float)(g[((size_t)N * kBoysTerms + k) * kBoysPitch + i] * fact);
        }
        return f;
    }
}
