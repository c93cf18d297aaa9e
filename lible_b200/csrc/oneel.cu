// One-electron integrals over the main basis: overlap, kinetic energy and the Coulomb attraction of
// point charges (the nuclear attraction takes the nuclei as the charges).  The formulation is the
// reference's McMurchie-Davidson one (src/lible/ints/oneelints.cpp: overlapKernel :57-98,
// kineticEnergyKernel :199-276, externalChargesKernel :508-585, nuclearAttraction :1703-1744):
//   S_ij = d_a d_b (pi/p)^{3/2} E^x_{ii'0} E^y_{jj'0} E^z_{kk'0}
//   T_ij = d_a d_b (pi/p)^{3/2} (T_x E^y E^z + E^x T_y E^z + E^x E^y T_z),
//          T_x = -2 b^2 E^x_{i,i'+2,0} + b (2i'+1) E^x_{i,i',0} - i'(i'-1)/2 E^x_{i,i'-2,0}
//   V_ij = -(2 pi / p) d_a d_b sum_C q_C sum_tuv E^x_{ii't} E^y_{jj'u} E^z_{kk'v} R_tuv(p, P - C)
// accumulated over the primitive pairs of a contracted shell pair, then transformed to spherical
// functions and scaled by the contracted AO norms.
//
// Kernel shape: one warp per contracted shell pair.  Per primitive pair, three lanes build the
// x / y / z Hermite tables (with b's angular momentum raised by 2 for the kinetic term) in shared
// memory; the lanes split the point charges for the charge-summed Hermite integrals, reduced by
// warp shuffles; then the lanes split the Cartesian (a, b) elements, each accumulating S, T and V
// in registers.  The spherical transform runs once per pair at the end.
#include "device_common.cuh"
#include "engine_api.hpp"
#include "ri_solve.hpp"

#include <algorithm>
#include <vector>

namespace lible_b200
{
    namespace
    {
        struct OneArgs
        {
            int n_pairs, nao;
            const double *exps, *coeffs, *coords, *norms_a, *norms_b;  // per class, host layout
            const uint32_t *pofs;
            const int32_t *ao;      // [n_pairs][2]
            const double *charges;  // [n][4] x, y, z, q
            int n_charges;
            const double *boys;     // Boys tables (all orders)
            const int *sph_rc;      // spherical transform entries (row, cart) and values
            const double *sph_val;
            int sph_ofs_a0, sph_ofs_a1, sph_ofs_b0, sph_ofs_b1;
            double *S, *T, *V;      // full nao x nao outputs (any may be null)
        };

        // Cartesian exponents of index c in a shell of angular momentum l (x-major descending).
        __device__ __forceinline__ void cartExps(int l, int c, int &i, int &j, int &k)
        {
            i = j = k = 0;
            for (int x = l, n = 0; x >= 0; x--)
                for (int y = l - x; y >= 0; y--, n++)
                    if (n == c)
                    {
                        i = x;
                        j = y;
                        k = l - x - y;
                    }
        }

        template <int LA, int LB>
        struct OneShape
        {
            static constexpr int L = LA + LB;
            static constexpr int NCA = (LA + 1) * (LA + 2) / 2, NCB = (LB + 1) * (LB + 2) / 2;
            static constexpr int NC = NCA * NCB;
            static constexpr int PER_LANE = (NC + 31) / 32;
            static constexpr int NT = LA + LB + 3;                       // t range of the raised tables
            static constexpr int EAX = (LA + 1) * (LB + 3) * NT;         // one axis
            static constexpr int NR = (L + 1) * (L + 2) * (L + 3) / 6;
            static constexpr int WARP_DOUBLES = 3 * EAX + NR + 3 * NC;   // E tables, R sum, Cartesian blocks
        };

        template <int LA, int LB>
        __global__ void __launch_bounds__(128) oneElKernel(OneArgs a)
        {
            using S = OneShape<LA, LB>;
            constexpr int L = S::L, NT = S::NT, NB = LB + 3;
            extern __shared__ __align__(16) double smem1[];
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            double *E = smem1 + (size_t)warp * S::WARP_DOUBLES;  // [axis][i][j][t]
            double *Rs = E + 3 * S::EAX;
            double *cart = Rs + S::NR;                            // [op][ca][cb]
            const int ipair = blockIdx.x * (blockDim.x >> 5) + warp;
            if (ipair >= a.n_pairs)
                return;
            auto ex = [&](int axis, int i, int j, int t) { return E[axis * S::EAX + (i * NB + j) * NT + t]; };
            double accS[S::PER_LANE], accT[S::PER_LANE], accV[S::PER_LANE];
#pragma unroll
            for (int w = 0; w < S::PER_LANE; w++)
                accS[w] = accT[w] = accV[w] = 0.0;
            const double *A = a.coords + 6 * (size_t)ipair, *B = A + 3;
            for (uint32_t pp = a.pofs[ipair]; pp < a.pofs[ipair + 1]; pp++)
            {
                const double ea = a.exps[2 * pp], eb = a.exps[2 * pp + 1];
                const double dadb = a.coeffs[2 * pp] * a.coeffs[2 * pp + 1];
                const double p = ea + eb, mu = ea * eb / p;
                double P[3];
#pragma unroll
                for (int k = 0; k < 3; k++)
                    P[k] = (ea * A[k] + eb * B[k]) / p;
                if (lane < 3)
                {
                    const double d = A[lane] - B[lane];
                    hermiteE(LA, LB + 2, 0.5 / p, P[lane] - A[lane], P[lane] - B[lane], exp(-mu * d * d),
                             E + lane * S::EAX);
                }
                if (a.V)
                {
                    // sum_C q_C R_tuv(p, P - C) over this lane's charges, then across the warp
                    double r[S::NR];
#pragma unroll
                    for (int h = 0; h < S::NR; h++)
                        r[h] = 0.0;
                    for (int c = lane; c < a.n_charges; c += 32)
                    {
                        const double *q = a.charges + 4 * (size_t)c;
                        const double X = P[0] - q[0], Y = P[1] - q[1], Z = P[2] - q[2];
                        double F[L + 1], R[S::NR];
                        boysF<L, false>(p * (X * X + Y * Y + Z * Z), a.boys + (size_t)L * kBoysTerms * kBoysPitch, F);
#pragma unroll
                        for (int n = 0; n <= L; n++)
                            F[n] *= q[3];
                        hermiteR<L, double>(-2.0 * p, F, X, Y, Z, R);
#pragma unroll
                        for (int h = 0; h < S::NR; h++)
                            r[h] += R[h];
                    }
#pragma unroll
                    for (int h = 0; h < S::NR; h++)
                    {
                        double v = r[h];
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1)
                            v += __shfl_xor_sync(0xffffffffu, v, o);
                        if (lane == 0)
                            Rs[h] = v;
                    }
                }
                __syncwarp();
                const double fs = dadb * pow(3.14159265358979323846 / p, 1.5);
                const double fv = -2.0 * 3.14159265358979323846 / p * dadb;  // -1: the electron's charge
                const double b2 = eb * eb;
#pragma unroll
                for (int w = 0; w < S::PER_LANE; w++)
                {
                    const int e = lane + 32 * w;
                    if (e >= S::NC)
                        break;
                    int i, j, k, i_, j_, k_;
                    cartExps(LA, e / S::NCB, i, j, k);
                    cartExps(LB, e % S::NCB, i_, j_, k_);
                    const double sx = ex(0, i, i_, 0), sy = ex(1, j, j_, 0), sz = ex(2, k, k_, 0);
                    accS[w] += fs * sx * sy * sz;
                    if (a.T)
                    {
                        auto kin = [&](int axis, int m, int m_) {
                            double t = -2.0 * b2 * ex(axis, m, m_ + 2, 0) + eb * (2 * m_ + 1) * ex(axis, m, m_, 0);
                            if (m_ >= 2)
                                t -= 0.5 * m_ * (m_ - 1) * ex(axis, m, m_ - 2, 0);
                            return t;
                        };
                        accT[w] += fs * (kin(0, i, i_) * sy * sz + sx * kin(1, j, j_) * sz + sx * sy * kin(2, k, k_));
                    }
                    if (a.V)
                    {
                        double v = 0.0;
                        for (int t = 0; t <= i + i_; t++)
                            for (int u = 0; u <= j + j_; u++)
                            {
                                const double exy = ex(0, i, i_, t) * ex(1, j, j_, u);
                                for (int s = 0; s <= k + k_; s++)
                                    v += exy * ex(2, k, k_, s) * Rs[hermIndex(t, u, s)];
                            }
                        accV[w] += fv * v;
                    }
                }
                __syncwarp();
            }
            // spherical transform of both shells and the AO norms
#pragma unroll
            for (int w = 0; w < S::PER_LANE; w++)
            {
                const int e = lane + 32 * w;
                if (e < S::NC)
                {
                    cart[e] = accS[w];
                    cart[S::NC + e] = accT[w];
                    cart[2 * S::NC + e] = accV[w];
                }
            }
            __syncwarp();
            constexpr int SA = 2 * LA + 1, SB = 2 * LB + 1;
            const int oa = a.ao[2 * ipair], ob = a.ao[2 * ipair + 1];
            const size_t n = (size_t)a.nao;
            for (int e = lane; e < SA * SB; e += 32)
            {
                const int m = e / SB, nn = e % SB;
                double s[3] = {0.0, 0.0, 0.0};
                for (int ta = a.sph_ofs_a0; ta < a.sph_ofs_a1; ta++)
                {
                    if (a.sph_rc[2 * ta] != m)
                        continue;
                    const int ca = a.sph_rc[2 * ta + 1];
                    const double va = a.sph_val[ta];
                    for (int tb = a.sph_ofs_b0; tb < a.sph_ofs_b1; tb++)
                    {
                        if (a.sph_rc[2 * tb] != nn)
                            continue;
                        const int x = ca * S::NCB + a.sph_rc[2 * tb + 1];
                        const double f = va * a.sph_val[tb];
                        s[0] += f * cart[x];
                        s[1] += f * cart[S::NC + x];
                        s[2] += f * cart[2 * S::NC + x];
                    }
                }
                const double nrm = a.norms_a[(size_t)ipair * SA + m] * a.norms_b[(size_t)ipair * SB + nn];
                double *outs[3] = {a.S, a.T, a.V};
                for (int op = 0; op < 3; op++)
                    if (outs[op])
                    {
                        outs[op][(oa + m) * n + ob + nn] = nrm * s[op];
                        outs[op][(ob + nn) * n + oa + m] = nrm * s[op];
                    }
            }
        }

        // ---- per-pair blocks (the reference's kernel API) and the gradient contraction --------------
        // Operators of the per-pair form: forward S, T, V ([S_a][S_b] per pair) and their first
        // derivatives ([6][S_a][S_b]: A_x, A_y, A_z, B_x, B_y, B_z), V being the orbital part
        // (src/lible/ints/oneelints.cpp: overlapD1Kernel :103-164, kineticEnergyD1Kernel :278-346,
        // externalChargesD1Kernel :682-789).  The derivatives use dE/d(A - B) (hermiteE1) and, for
        // V, the charge-summed Hermite integrals of one order higher:
        //   d/dA = -((a/p) dP + dR),  d/dB = -((b/p) dP - dR),
        //   dP_x = f sum E_t E_u E_v R_{t+1,u,v},  dR_x = f sum E1_t E_u E_v R_{tuv}.
        // Multipole-type operators of one pair, three blocks each (x, y, z), with O the caller's origin
        // (src/lible/ints/oneelints.cpp: dipoleMomentKernel :379-473, momentumKernel :1513-1577,
        // angularMomentumKernel :1617-1701), from the same Hermite tables:
        //   dipole:   fs (E^x_{ii'1} + PO_x E^x_{ii'0}) E^y E^z             (and y, z)
        //   momentum: -fs D^x E^y E^z,  D^x = -2b E^x_{i,i'+1,0} + i' E^x_{i,i'-1,0}
        //   angular:  -fs E^x (S^y D^z - S^z D^y),  S^y = E^y_{jj'1} + PO_y E^y_{jj'0}   (cyclic)
        // and the erf-attenuated Coulomb attraction of point charges with a range parameter w_C each
        // (externalChargesErfKernel :587-680): the charge's R_tuv taken with the exponent
        // p w^2 / (p + w^2) and scaled by q_C w / sqrt(w^2 + p).
        enum OneOp : int
        {
            kOpS = 0,
            kOpT = 1,
            kOpV = 2,
            kOpSD1 = 3,
            kOpTD1 = 4,
            kOpVD1 = 5,
            kOpDipole = 6,
            kOpMomentum = 7,
            kOpAngular = 8,
            kOpVErf = 9,
            kOpVErfD1 = 10,   // externalChargesErfD1Kernel: orbital part, [6] blocks
            kOpVOpD1 = 11,    // externalChargesOperatorD1Kernel for the charges summed: d/dC_xyz, [3]
            kOpVErfOpD1 = 12, // the same, erf-attenuated
            kOpSOC = 13,      // spinOrbitCoupling1ElKernel, [3]
            kOpPVP = 14,      // pVpKernel, [3][3] (pvpPairKernel)
        };
        __host__ __device__ constexpr int oneOpBlocks(int op)
        {
            return op == kOpPVP                                                              ? 9
                   : ((op >= kOpSD1 && op <= kOpVD1) || op == kOpVErfD1)                   ? 6
                   : ((op >= kOpDipole && op <= kOpAngular) || op >= kOpVOpD1) ? 3
                                                                                          : 1;
        }
        __host__ __device__ constexpr bool oneOpUsesCharges(int op)
        {
            return op == kOpV || op == kOpVD1 || op >= kOpVErf;
        }
        __host__ __device__ constexpr bool oneOpUsesOmegas(int op)
        {
            return op == kOpVErf || op == kOpVErfD1 || op == kOpVErfOpD1;
        }

        struct OnePairArgs
        {
            int op;                  // OneOp (store mode)
            int swap;                // store mode: the class is stored with a and b exchanged; write the
                                     // caller's orientation (blocks transposed, d/dA and d/dB exchanged)
            long long n_tasks;
            const uint32_t *list;    // pair index of each task (store mode), null = every pair
            int n_pairs, nao;
            const double *exps, *coeffs, *coords, *norms_a, *norms_b;
            const uint32_t *pofs;
            const int32_t *ao;       // [n_pairs][2]
            const int32_t *atoms;    // [n_pairs][2] (gradient mode)
            const int32_t *same;     // [n_pairs]: 1 when a and b are the same shell (gradient mode)
            const double *charges;   // [n][4]
            const double *omegas;    // [n] range parameters (kOpVErf), else null
            int n_charges;
            double origin[3];        // multipole origin (kOpDipole, kOpAngular)
            const double *boys;
            const int *sph_rc;
            const double *sph_val;
            int sph_ofs_a0, sph_ofs_a1, sph_ofs_b0, sph_ofs_b1;
            double *out;             // store mode: [task][blocks][S_a][S_b]
            const double *D, *W;     // gradient mode: full nao x nao (either may be null)
            double *grad;            // [n_atoms][3]
        };

        template <int LA, int LB>
        struct PairShape
        {
            static constexpr int L = LA + LB, L1 = L + 1;
            static constexpr int NCA = (LA + 1) * (LA + 2) / 2, NCB = (LB + 1) * (LB + 2) / 2;
            static constexpr int NC = NCA * NCB;
            static constexpr int PER_LANE = (NC + 31) / 32;
            static constexpr int NT = LA + LB + 3;
            static constexpr int EAX = (LA + 1) * (LB + 3) * NT;
            static constexpr int NR = (L + 1) * (L + 2) * (L + 3) / 6;
            static constexpr int NR1 = (L1 + 1) * (L1 + 2) * (L1 + 3) / 6;
            static constexpr int SA = 2 * LA + 1, SB = 2 * LB + 1;
            // E and E1 tables, the charge-summed R (order L + 1), the density-weighted Hermite
            // vector, then 6 Cartesian blocks (store) or the Cartesian D and W blocks (gradient)
            static constexpr int WARP_DOUBLES = 6 * EAX + NR1 + NR + 6 * NC;
        };

        template <int LA, int LB, bool GRAD>
        __global__ void __launch_bounds__(128) onePairKernel(OnePairArgs a)
        {
            using S = PairShape<LA, LB>;
            constexpr int L = S::L, L1 = S::L1, NT = S::NT, NB = LB + 3;
            extern __shared__ __align__(16) double smem2[];
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            double *E = smem2 + (size_t)warp * S::WARP_DOUBLES;  // [axis][i][j][t]
            double *E1 = E + 3 * S::EAX;
            double *Rs = E1 + 3 * S::EAX;                         // order L + 1
            double *dt = Rs + S::NR1;                             // density-weighted Hermite vector
            double *blk = dt + S::NR;                             // 6 x NC
            const long long task = (long long)blockIdx.x * (blockDim.x >> 5) + warp;
            if (task >= a.n_tasks)
                return;
            const int ipair = a.list ? (int)a.list[task] : (int)task;
            auto ex = [&](int axis, int i, int j, int t) { return E[axis * S::EAX + (i * NB + j) * NT + t]; };
            auto ex1 = [&](int axis, int i, int j, int t) { return E1[axis * S::EAX + (i * NB + j) * NT + t]; };
            const int op = GRAD ? -1 : a.op;
            const bool wantV = GRAD ? a.D != nullptr : oneOpUsesCharges(op);
            const bool d1 = GRAD || oneOpBlocks(op) == 6 || op == kOpSOC;
            const int oa = a.ao[2 * ipair], ob = a.ao[2 * ipair + 1];
            const size_t n = (size_t)a.nao;
            const double *nA = a.norms_a + (size_t)ipair * S::SA, *nB = a.norms_b + (size_t)ipair * S::SB;
            if constexpr (GRAD)
            {
                // Cartesian D and W blocks of the pair, with the AO norms and the pair's multiplicity
                // in sum_{mn} (both orientations of an off-diagonal pair)
                const double mult = a.same[ipair] ? 1.0 : 2.0;
                for (int e = lane; e < S::NC; e += 32)
                {
                    const int ca = e / S::NCB, cb = e % S::NCB;
                    double sd = 0.0, sw = 0.0;
                    for (int ta = a.sph_ofs_a0; ta < a.sph_ofs_a1; ta++)
                    {
                        if (a.sph_rc[2 * ta + 1] != ca)
                            continue;
                        const int m = a.sph_rc[2 * ta];
                        const double va = a.sph_val[ta] * nA[m];
                        for (int tb = a.sph_ofs_b0; tb < a.sph_ofs_b1; tb++)
                        {
                            if (a.sph_rc[2 * tb + 1] != cb)
                                continue;
                            const int nn = a.sph_rc[2 * tb];
                            const double f = va * a.sph_val[tb] * nB[nn];
                            const size_t idx = (oa + m) * n + ob + nn;
                            if (a.D)
                                sd += f * a.D[idx];
                            if (a.W)
                                sw += f * a.W[idx];
                        }
                    }
                    blk[e] = mult * sd;
                    blk[S::NC + e] = mult * sw;
                }
                __syncwarp();
            }
            double acc[6][S::PER_LANE];
#pragma unroll
            for (int d = 0; d < 6; d++)
#pragma unroll
                for (int w = 0; w < S::PER_LANE; w++)
                    acc[d][w] = 0.0;
            double gA[3] = {0, 0, 0}, gB[3] = {0, 0, 0};
            const double *A = a.coords + 6 * (size_t)ipair, *B = A + 3;
            for (uint32_t pp = a.pofs[ipair]; pp < a.pofs[ipair + 1]; pp++)
            {
                const double ea = a.exps[2 * pp], eb = a.exps[2 * pp + 1];
                const double dadb = a.coeffs[2 * pp] * a.coeffs[2 * pp + 1];
                const double p = ea + eb, mu = ea * eb / p;
                double P[3];
#pragma unroll
                for (int k = 0; k < 3; k++)
                    P[k] = (ea * A[k] + eb * B[k]) / p;
                if (lane < 3)
                {
                    const double d = A[lane] - B[lane];
                    hermiteE(LA, LB + 2, 0.5 / p, P[lane] - A[lane], P[lane] - B[lane], exp(-mu * d * d),
                             E + lane * S::EAX);
                    if (d1)
                        hermiteE1(LA, LB + 2, ea, eb, d, E + lane * S::EAX, E1 + lane * S::EAX);
                }
                if (wantV)
                {
                    double r[S::NR1];
#pragma unroll
                    for (int h = 0; h < S::NR1; h++)
                        r[h] = 0.0;
                    for (int c = lane; c < a.n_charges; c += 32)
                    {
                        const double *q = a.charges + 4 * (size_t)c;
                        const double X = P[0] - q[0], Y = P[1] - q[1], Z = P[2] - q[2];
                        double F[L1 + 1], R[S::NR1];
                        // erf attenuation: exponent p w^2 / (p + w^2), scale w / sqrt(w^2 + p); the
                        // reference's derivative kernels scale by sqrt(w^2 / (w^2 + p)) instead
                        // (oneelints.cpp:1907-1909, 2028-2030 against :628), which differs for w < 0
                        double pe = p, qs = q[3];
                        if (a.omegas)
                        {
                            const double w = a.omegas[c], w2 = w * w;
                            pe = p * w2 / (p + w2);
                            qs *= (op == kOpVErfD1 || op == kOpVErfOpD1 ? fabs(w) : w) / sqrt(w2 + p);
                        }
                        boysF<L1, false>(pe * (X * X + Y * Y + Z * Z), a.boys + (size_t)L1 * kBoysTerms * kBoysPitch, F);
#pragma unroll
                        for (int k = 0; k <= L1; k++)
                            F[k] *= qs;
                        hermiteR<L1, double>(-2.0 * pe, F, X, Y, Z, R);
#pragma unroll
                        for (int h = 0; h < S::NR1; h++)
                            r[h] += R[h];
                    }
#pragma unroll
                    for (int h = 0; h < S::NR1; h++)
                    {
                        double v = r[h];
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1)
                            v += __shfl_xor_sync(0xffffffffu, v, o);
                        if (lane == 0)
                            Rs[h] = v;
                    }
                }
                __syncwarp();
                const double fs = dadb * pow(3.14159265358979323846 / p, 1.5);
                const double fv = 2.0 * 3.14159265358979323846 / p * dadb;
                const double b2 = eb * eb;
#pragma unroll
                for (int w = 0; w < S::PER_LANE; w++)
                {
                    const int e = lane + 32 * w;
                    if (e >= S::NC)
                        break;
                    int ijk[3], ijk_[3];
                    cartExps(LA, e / S::NCB, ijk[0], ijk[1], ijk[2]);
                    cartExps(LB, e % S::NCB, ijk_[0], ijk_[1], ijk_[2]);
                    double s0[3], s1[3];
#pragma unroll
                    for (int x = 0; x < 3; x++)
                    {
                        s0[x] = ex(x, ijk[x], ijk_[x], 0);
                        s1[x] = d1 ? ex1(x, ijk[x], ijk_[x], 0) : 0.0;
                    }
                    // kinetic factor of one axis from table E (tab 0) or E1 (tab 1)
                    auto kin = [&](int tab, int x) {
                        const int m = ijk[x], m_ = ijk_[x];
                        auto g = [&](int jj) { return tab ? ex1(x, m, jj, 0) : ex(x, m, jj, 0); };
                        double t = -2.0 * b2 * g(m_ + 2) + eb * (2 * m_ + 1) * g(m_);
                        if (m_ >= 2)
                            t -= 0.5 * m_ * (m_ - 1) * g(m_ - 2);
                        return t;
                    };
                    // V pieces: sum over t <= i + i', u, v of the E products times R (optionally shifted)
                    auto vsum = [&](int dx, int use1) {
                        double v = 0.0;
                        for (int t = 0; t <= ijk[0] + ijk_[0]; t++)
                            for (int u = 0; u <= ijk[1] + ijk_[1]; u++)
                                for (int s = 0; s <= ijk[2] + ijk_[2]; s++)
                                {
                                    const double e0 = (use1 == 0 ? ex1(0, ijk[0], ijk_[0], t) : ex(0, ijk[0], ijk_[0], t)) *
                                                      (use1 == 1 ? ex1(1, ijk[1], ijk_[1], u) : ex(1, ijk[1], ijk_[1], u)) *
                                                      (use1 == 2 ? ex1(2, ijk[2], ijk_[2], s) : ex(2, ijk[2], ijk_[2], s));
                                    v += e0 * Rs[hermIndex(t + (dx == 0), u + (dx == 1), s + (dx == 2))];
                                }
                        return v;
                    };
                    if (!GRAD)
                    {
                        if (op == kOpS)
                            acc[0][w] += fs * s0[0] * s0[1] * s0[2];
                        else if (op == kOpT)
                            acc[0][w] += fs * (kin(0, 0) * s0[1] * s0[2] + s0[0] * kin(0, 1) * s0[2] +
                                               s0[0] * s0[1] * kin(0, 2));
                        else if (op == kOpV || op == kOpVErf)
                            acc[0][w] -= fv * vsum(-1, -1);
                        else if (op == kOpSOC)
                        {
                            // the reference's SOC form (oneelints.cpp:1209-1316): with
                            // [d, e] = sum E(E1 on axis e) R_{+1 on axis d},
                            // x: -f ([z, y] - [y, z]), y: -f ([x, z] - [z, x]), z: -f ([y, x] - [x, y])
                            acc[0][w] -= fv * (vsum(2, 1) - vsum(1, 2));
                            acc[1][w] -= fv * (vsum(0, 2) - vsum(2, 0));
                            acc[2][w] -= fv * (vsum(1, 0) - vsum(0, 1));
                        }
                        else if (op == kOpVOpD1 || op == kOpVErfOpD1)
                        {
                            // d/dC of -f q sum E R(P - C): +f q sum E R_{t+1} (and u, v)
#pragma unroll
                            for (int x = 0; x < 3; x++)
                                acc[x][w] += fv * vsum(x, -1);
                        }
                        else if (op >= kOpDipole && op <= kOpAngular)
                        {
                            // first moments about the origin and first derivatives on b, per axis
                            double m1[3], dd[3];
#pragma unroll
                            for (int x = 0; x < 3; x++)
                            {
                                const int i = ijk[x], i_ = ijk_[x];
                                m1[x] = ex(x, i, i_, 1) + (P[x] - a.origin[x]) * s0[x];
                                dd[x] = -2.0 * eb * ex(x, i, i_ + 1, 0) + (i_ > 0 ? i_ * ex(x, i, i_ - 1, 0) : 0.0);
                            }
                            if (op == kOpDipole)
                            {
                                acc[0][w] += fs * m1[0] * s0[1] * s0[2];
                                acc[1][w] += fs * s0[0] * m1[1] * s0[2];
                                acc[2][w] += fs * s0[0] * s0[1] * m1[2];
                            }
                            else if (op == kOpMomentum)
                            {
                                acc[0][w] -= fs * dd[0] * s0[1] * s0[2];
                                acc[1][w] -= fs * s0[0] * dd[1] * s0[2];
                                acc[2][w] -= fs * s0[0] * s0[1] * dd[2];
                            }
                            else
                            {
                                acc[0][w] -= fs * s0[0] * (m1[1] * dd[2] - m1[2] * dd[1]);
                                acc[1][w] -= fs * s0[1] * (m1[2] * dd[0] - m1[0] * dd[2]);
                                acc[2][w] -= fs * s0[2] * (m1[0] * dd[1] - m1[1] * dd[0]);
                            }
                        }
                        else
                        {
#pragma unroll
                            for (int x = 0; x < 3; x++)
                            {
                                double dA, dB;
                                if (op == kOpSD1)
                                {
                                    const double v = fs * (x == 0 ? s1[0] : s0[0]) * (x == 1 ? s1[1] : s0[1]) *
                                                     (x == 2 ? s1[2] : s0[2]);
                                    dA = v;
                                    dB = -v;
                                }
                                else if (op == kOpTD1)
                                {
                                    // the x-axis table replaced by E1 in every term
                                    const double sx = x == 0 ? s1[0] : s0[0], sy = x == 1 ? s1[1] : s0[1],
                                                 sz = x == 2 ? s1[2] : s0[2];
                                    const double v = fs * (kin(x == 0, 0) * sy * sz + sx * kin(x == 1, 1) * sz +
                                                           sx * sy * kin(x == 2, 2));
                                    dA = v;
                                    dB = -v;
                                }
                                else
                                {
                                    const double dp = fv * vsum(x, -1), dr = fv * vsum(-1, x);
                                    dA = -((ea / p) * dp + dr);
                                    dB = -((eb / p) * dp - dr);
                                }
                                acc[x][w] += dA;
                                acc[3 + x][w] += dB;
                            }
                        }
                    }
                    else
                    {
                        const double dd = blk[e], ww = blk[S::NC + e];
#pragma unroll
                        for (int x = 0; x < 3; x++)
                        {
                            const double sx = x == 0 ? s1[0] : s0[0], sy = x == 1 ? s1[1] : s0[1],
                                         sz = x == 2 ? s1[2] : s0[2];
                            // overlap (with W) and kinetic (with D): d/dB = -d/dA
                            double g = -ww * fs * sx * sy * sz;
                            if (a.D)
                                g += dd * fs * (kin(x == 0, 0) * sy * sz + sx * kin(x == 1, 1) * sz + sx * sy * kin(x == 2, 2));
                            gA[x] += g;
                            gB[x] -= g;
                            if (a.D)
                            {
                                const double dp = fv * vsum(x, -1), dr = fv * vsum(-1, x);
                                gA[x] -= dd * ((ea / p) * dp + dr);
                                gB[x] -= dd * ((eb / p) * dp - dr);
                            }
                        }
                    }
                }
                if (GRAD && a.D)
                {
                    // operator part: d/dC_x of -f q_C sum D E R(P - C) = f q_C sum D E R_{t+1}
                    __syncwarp();
                    for (int h = lane; h < S::NR; h += 32)
                    {
                        int t0 = 0, u0 = 0, v0 = 0;
                        for (int nn = 0, idx = 0; nn <= L; nn++)
                            for (int t = nn; t >= 0; t--)
                                for (int u = nn - t; u >= 0; u--, idx++)
                                    if (idx == h)
                                    {
                                        t0 = t;
                                        u0 = u;
                                        v0 = nn - t - u;
                                    }
                        double v = 0.0;
                        for (int e = 0; e < S::NC; e++)
                        {
                            int i, j, k, i_, j_, k_;
                            cartExps(LA, e / S::NCB, i, j, k);
                            cartExps(LB, e % S::NCB, i_, j_, k_);
                            if (t0 > i + i_ || u0 > j + j_ || v0 > k + k_)
                                continue;
                            v += blk[e] * ex(0, i, i_, t0) * ex(1, j, j_, u0) * ex(2, k, k_, v0);
                        }
                        dt[h] = fv * v;
                    }
                    __syncwarp();
                    for (int c = lane; c < a.n_charges; c += 32)
                    {
                        const double *q = a.charges + 4 * (size_t)c;
                        const double X = P[0] - q[0], Y = P[1] - q[1], Z = P[2] - q[2];
                        double F[L1 + 1], R[S::NR1];
                        boysF<L1, false>(p * (X * X + Y * Y + Z * Z), a.boys + (size_t)L1 * kBoysTerms * kBoysPitch, F);
                        hermiteR<L1, double>(-2.0 * p, F, X, Y, Z, R);
                        double g[3] = {0, 0, 0};
                        for (int nn = 0, h = 0; nn <= L; nn++)
                            for (int t = nn; t >= 0; t--)
                                for (int u = nn - t; u >= 0; u--, h++)
                                {
                                    const int v = nn - t - u;
                                    g[0] += dt[h] * R[hermIndex(t + 1, u, v)];
                                    g[1] += dt[h] * R[hermIndex(t, u + 1, v)];
                                    g[2] += dt[h] * R[hermIndex(t, u, v + 1)];
                                }
                        // charge c is atom c (the nuclei in atom order)
                        for (int x = 0; x < 3; x++)
                            atomicAdd(a.grad + 3 * (size_t)c + x, q[3] * g[x]);
                    }
                }
                __syncwarp();
            }
            if constexpr (GRAD)
            {
#pragma unroll
                for (int x = 0; x < 3; x++)
                {
                    double u = gA[x], v = gB[x];
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1)
                    {
                        u += __shfl_xor_sync(0xffffffffu, u, o);
                        v += __shfl_xor_sync(0xffffffffu, v, o);
                    }
                    if (lane == 0)
                    {
                        atomicAdd(a.grad + 3 * (size_t)a.atoms[2 * ipair] + x, u);
                        atomicAdd(a.grad + 3 * (size_t)a.atoms[2 * ipair + 1] + x, v);
                    }
                }
            }
            else
            {
                // spherical transform and norms of each stored block; a swapped class is written in the
                // caller's orientation: blocks transposed, d/dA and d/dB exchanged, and the
                // antisymmetric operators (momentum, angular momentum) negated
                const int nblk = oneOpBlocks(op);
                const double sgn = (a.swap && (op == kOpMomentum || op == kOpAngular || op == kOpSOC)) ? -1.0 : 1.0;
                for (int d = 0; d < nblk; d++)
#pragma unroll
                    for (int w = 0; w < S::PER_LANE; w++)
                    {
                        const int e = lane + 32 * w;
                        if (e < S::NC)
                            blk[d * S::NC + e] = acc[d][w];
                    }
                __syncwarp();
                double *out = a.out + (size_t)task * nblk * S::SA * S::SB;
                for (int o = lane; o < nblk * S::SA * S::SB; o += 32)
                {
                    const int d = o / (S::SA * S::SB), m = (o / S::SB) % S::SA, nn = o % S::SB;
                    const int dst = a.swap ? ((nblk == 6 ? (d + 3) % 6 : d) * S::SA * S::SB + nn * S::SA + m) : o;
                    double sum = 0.0;
                    for (int ta = a.sph_ofs_a0; ta < a.sph_ofs_a1; ta++)
                    {
                        if (a.sph_rc[2 * ta] != m)
                            continue;
                        const int ca = a.sph_rc[2 * ta + 1];
                        for (int tb = a.sph_ofs_b0; tb < a.sph_ofs_b1; tb++)
                            if (a.sph_rc[2 * tb] == nn)
                                sum += a.sph_val[ta] * a.sph_val[tb] * blk[d * S::NC + ca * S::NCB + a.sph_rc[2 * tb + 1]];
                    }
                    out[dst] = sgn * nA[m] * nB[nn] * sum;
                }
            }
        }

        // pVp integrals of one pair, [3][3][S_a][S_b]: <d_i a| V |d_j b> for the point charges, the
        // quantity of the reference's pVpKernel (src/lible/ints/oneelints.cpp:1318-1475).  With
        // d/dA = (a/p) d/dP + d/dR and d/dB = (b/p) d/dP - d/dR applied to the Hermite expansion
        // -f sum_tuv E_tuv(R) R_tuv(P - C) of the attraction (R = A - B, f = 2 pi / p d_a d_b):
        //   pVp_ij = -f sum_tuv ( (ab/p^2) E R_{+e_i+e_j} - (a/p) E1_j R_{+e_i} + (b/p) E1_i R_{+e_j}
        //                         - E2_ij R_tuv ),
        // E1_j: the j-axis table replaced by its first derivative (hermiteE1), E2_ij: both first
        // derivatives (i != j) or the i-axis second derivative (hermiteE2, i = j), R to order L + 2.
        // The reference's kernel leaves out the E factor of its first term and the R factor of its
        // last, and forms the x second-derivative table from the y first derivatives
        // (oneelints.cpp:1392-1460, ecoeffs.cpp:205); this kernel follows the derivation, which the
        // tests check against central finite differences of the point-charge integrals.  One warp
        // per pair, as onePairKernel.
        template <int LA, int LB>
        struct PvpShape
        {
            static constexpr int L = LA + LB, L2 = L + 2;
            static constexpr int NCA = (LA + 1) * (LA + 2) / 2, NCB = (LB + 1) * (LB + 2) / 2;
            static constexpr int NC = NCA * NCB;
            static constexpr int PER_LANE = (NC + 31) / 32;
            static constexpr int NT = L + 1;
            static constexpr int EAX = (LA + 1) * (LB + 1) * NT;
            static constexpr int NR2 = (L2 + 1) * (L2 + 2) * (L2 + 3) / 6;
            static constexpr int SA = 2 * LA + 1, SB = 2 * LB + 1;
            static constexpr int WARP_DOUBLES = 9 * EAX + NR2 + 9 * NC;  // E, E1, E2; R; 9 blocks
        };

        template <int LA, int LB>
        __global__ void __launch_bounds__(128) pvpPairKernel(OnePairArgs a)
        {
            using S = PvpShape<LA, LB>;
            constexpr int L2 = S::L2, NT = S::NT, NB = LB + 1;
            extern __shared__ __align__(16) double smem3[];
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            double *E = smem3 + (size_t)warp * S::WARP_DOUBLES;  // [table][axis][i][j][t]
            double *Rs = E + 9 * S::EAX;
            double *blk = Rs + S::NR2;
            const long long task = (long long)blockIdx.x * (blockDim.x >> 5) + warp;
            if (task >= a.n_tasks)
                return;
            const int ipair = a.list ? (int)a.list[task] : (int)task;
            auto ex = [&](int tab, int axis, int i, int j, int t) {
                return E[(tab * 3 + axis) * S::EAX + (i * NB + j) * NT + t];
            };
            const double *nA = a.norms_a + (size_t)ipair * S::SA, *nB = a.norms_b + (size_t)ipair * S::SB;
            double acc[9][S::PER_LANE];
#pragma unroll
            for (int d = 0; d < 9; d++)
#pragma unroll
                for (int w = 0; w < S::PER_LANE; w++)
                    acc[d][w] = 0.0;
            const double *A = a.coords + 6 * (size_t)ipair, *B = A + 3;
            for (uint32_t pp = a.pofs[ipair]; pp < a.pofs[ipair + 1]; pp++)
            {
                const double ea = a.exps[2 * pp], eb = a.exps[2 * pp + 1];
                const double dadb = a.coeffs[2 * pp] * a.coeffs[2 * pp + 1];
                const double p = ea + eb, mu = ea * eb / p;
                double P[3];
#pragma unroll
                for (int k = 0; k < 3; k++)
                    P[k] = (ea * A[k] + eb * B[k]) / p;
                if (lane < 3)
                {
                    const double d = A[lane] - B[lane];
                    double *e0 = E + lane * S::EAX, *e1 = E + (3 + lane) * S::EAX, *e2 = E + (6 + lane) * S::EAX;
                    hermiteE(LA, LB, 0.5 / p, P[lane] - A[lane], P[lane] - B[lane], exp(-mu * d * d), e0);
                    hermiteE1(LA, LB, ea, eb, d, e0, e1);
                    hermiteE2(LA, LB, ea, eb, d, e0, e1, e2);
                }
                double r[S::NR2];
#pragma unroll
                for (int h = 0; h < S::NR2; h++)
                    r[h] = 0.0;
                for (int c = lane; c < a.n_charges; c += 32)
                {
                    const double *q = a.charges + 4 * (size_t)c;
                    const double X = P[0] - q[0], Y = P[1] - q[1], Z = P[2] - q[2];
                    double F[L2 + 1], R[S::NR2];
                    boysF<L2, false>(p * (X * X + Y * Y + Z * Z), a.boys + (size_t)L2 * kBoysTerms * kBoysPitch, F);
#pragma unroll
                    for (int k = 0; k <= L2; k++)
                        F[k] *= q[3];
                    hermiteR<L2, double>(-2.0 * p, F, X, Y, Z, R);
#pragma unroll
                    for (int h = 0; h < S::NR2; h++)
                        r[h] += R[h];
                }
#pragma unroll
                for (int h = 0; h < S::NR2; h++)
                {
                    double v = r[h];
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1)
                        v += __shfl_xor_sync(0xffffffffu, v, o);
                    if (lane == 0)
                        Rs[h] = v;
                }
                __syncwarp();
                const double fv = 2.0 * 3.14159265358979323846 / p * dadb;
                const double cpp = ea * eb / (p * p), ca = ea / p, cb = eb / p;
#pragma unroll
                for (int w = 0; w < S::PER_LANE; w++)
                {
                    const int e = lane + 32 * w;
                    if (e >= S::NC)
                        break;
                    int ijk[3], ijk_[3];
                    cartExps(LA, e / S::NCB, ijk[0], ijk[1], ijk[2]);
                    cartExps(LB, e % S::NCB, ijk_[0], ijk_[1], ijk_[2]);
                    double s[9];
#pragma unroll
                    for (int d = 0; d < 9; d++)
                        s[d] = 0.0;
                    for (int t = 0; t <= ijk[0] + ijk_[0]; t++)
                        for (int u = 0; u <= ijk[1] + ijk_[1]; u++)
                            for (int v = 0; v <= ijk[2] + ijk_[2]; v++)
                            {
                                const int tuv[3] = {t, u, v};
                                double g0[3], g1[3], g2[3];
#pragma unroll
                                for (int x = 0; x < 3; x++)
                                {
                                    g0[x] = ex(0, x, ijk[x], ijk_[x], tuv[x]);
                                    g1[x] = ex(1, x, ijk[x], ijk_[x], tuv[x]);
                                    g2[x] = ex(2, x, ijk[x], ijk_[x], tuv[x]);
                                }
                                const double e000 = g0[0] * g0[1] * g0[2];
                                // E products with the first derivative on one axis, and on two / twice
                                const double e1x[3] = {g1[0] * g0[1] * g0[2], g0[0] * g1[1] * g0[2], g0[0] * g0[1] * g1[2]};
                                const double r0 = Rs[hermIndex(t, u, v)];
                                double r1[3];
#pragma unroll
                                for (int x = 0; x < 3; x++)
                                    r1[x] = Rs[hermIndex(t + (x == 0), u + (x == 1), v + (x == 2))];
#pragma unroll
                                for (int i = 0; i < 3; i++)
#pragma unroll
                                    for (int j = 0; j < 3; j++)
                                    {
                                        const double r2 = Rs[hermIndex(t + (i == 0) + (j == 0), u + (i == 1) + (j == 1),
                                                                       v + (i == 2) + (j == 2))];
                                        double rr;
                                        if (i == j)
                                            rr = (i == 0 ? g2[0] * g0[1] * g0[2]
                                                  : i == 1 ? g0[0] * g2[1] * g0[2] : g0[0] * g0[1] * g2[2]);
                                        else
                                        {
                                            const int k = 3 - i - j;
                                            rr = g1[i] * g1[j] * g0[k];
                                        }
                                        s[3 * i + j] += cpp * r2 * e000 - ca * r1[i] * e1x[j] + cb * r1[j] * e1x[i] - rr * r0;
                                    }
                            }
#pragma unroll
                    for (int d = 0; d < 9; d++)
                        acc[d][w] -= fv * s[d];
                }
                __syncwarp();
            }
            // spherical transform and norms; a swapped class is written in the caller's orientation:
            // blocks transposed and components (i, j) -> (j, i)
#pragma unroll
            for (int d = 0; d < 9; d++)
#pragma unroll
                for (int w = 0; w < S::PER_LANE; w++)
                {
                    const int e = lane + 32 * w;
                    if (e < S::NC)
                        blk[d * S::NC + e] = acc[d][w];
                }
            __syncwarp();
            double *out = a.out + (size_t)task * 9 * S::SA * S::SB;
            for (int o = lane; o < 9 * S::SA * S::SB; o += 32)
            {
                const int d = o / (S::SA * S::SB), m = (o / S::SB) % S::SA, nn = o % S::SB;
                const int dst = a.swap ? (((d % 3) * 3 + d / 3) * S::SA * S::SB + nn * S::SA + m) : o;
                double sum = 0.0;
                for (int ta = a.sph_ofs_a0; ta < a.sph_ofs_a1; ta++)
                {
                    if (a.sph_rc[2 * ta] != m)
                        continue;
                    const int ca2 = a.sph_rc[2 * ta + 1];
                    for (int tb = a.sph_ofs_b0; tb < a.sph_ofs_b1; tb++)
                        if (a.sph_rc[2 * tb] == nn)
                            sum += a.sph_val[ta] * a.sph_val[tb] * blk[d * S::NC + ca2 * S::NCB + a.sph_rc[2 * tb + 1]];
                }
                out[dst] = nA[m] * nB[nn] * sum;
            }
        }

        template <int LA, int LB>
        void launchPvp(const OnePairArgs &a, cudaStream_t s, bool)
        {
            constexpr int warps = 4;
            const size_t smem = sizeof(double) * warps * PvpShape<LA, LB>::WARP_DOUBLES;
            auto k = pvpPairKernel<LA, LB>;
            if (smem > 48 * 1024)
                cudaCheck(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "attr");
            k<<<(unsigned)((a.n_tasks + warps - 1) / warps), 32 * warps, smem, s>>>(a);
            cudaCheck(cudaGetLastError(), "pVp pair kernel");
        }

        using PairFn = void (*)(const OnePairArgs &, cudaStream_t, bool);
        template <int LA, int LB>
        void launchPair(const OnePairArgs &a, cudaStream_t s, bool grad)
        {
            constexpr int warps = 4;
            const size_t smem = sizeof(double) * warps * PairShape<LA, LB>::WARP_DOUBLES;
            auto k = grad ? onePairKernel<LA, LB, true> : onePairKernel<LA, LB, false>;
            if (smem > 48 * 1024)
                cudaCheck(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "attr");
            k<<<(unsigned)((a.n_tasks + warps - 1) / warps), 32 * warps, smem, s>>>(a);
            cudaCheck(cudaGetLastError(), "one-electron pair kernel");
        }

        PairFn lookupPvp(int la, int lb)
        {
            static const PairFn table[4][4] = {
                {&launchPvp<0, 0>, &launchPvp<0, 1>, &launchPvp<0, 2>, &launchPvp<0, 3>},
                {&launchPvp<1, 0>, &launchPvp<1, 1>, &launchPvp<1, 2>, &launchPvp<1, 3>},
                {&launchPvp<2, 0>, &launchPvp<2, 1>, &launchPvp<2, 2>, &launchPvp<2, 3>},
                {&launchPvp<3, 0>, &launchPvp<3, 1>, &launchPvp<3, 2>, &launchPvp<3, 3>},
            };
            return (la < 4 && lb < 4) ? table[la][lb] : nullptr;
        }

        PairFn lookupPair(int la, int lb)
        {
            static const PairFn table[4][4] = {
                {&launchPair<0, 0>, &launchPair<0, 1>, &launchPair<0, 2>, &launchPair<0, 3>},
                {&launchPair<1, 0>, &launchPair<1, 1>, &launchPair<1, 2>, &launchPair<1, 3>},
                {&launchPair<2, 0>, &launchPair<2, 1>, &launchPair<2, 2>, &launchPair<2, 3>},
                {&launchPair<3, 0>, &launchPair<3, 1>, &launchPair<3, 2>, &launchPair<3, 3>},
            };
            return (la < 4 && lb < 4) ? table[la][lb] : nullptr;
        }

        using OneFn = void (*)(const OneArgs &, cudaStream_t, int);
        template <int LA, int LB>
        void launchOne(const OneArgs &a, cudaStream_t s, int)
        {
            constexpr int warps = 4;
            const size_t smem = sizeof(double) * warps * OneShape<LA, LB>::WARP_DOUBLES;
            auto k = oneElKernel<LA, LB>;
            if (smem > 48 * 1024)
                cudaCheck(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "attr");
            k<<<(unsigned)((a.n_pairs + warps - 1) / warps), 32 * warps, smem, s>>>(a);
            cudaCheck(cudaGetLastError(), "one-electron kernel");
        }

        OneFn lookupOne(int la, int lb)
        {
            static const OneFn table[4][4] = {
                {&launchOne<0, 0>, nullptr, nullptr, nullptr},
                {&launchOne<1, 0>, &launchOne<1, 1>, nullptr, nullptr},
                {&launchOne<2, 0>, &launchOne<2, 1>, &launchOne<2, 2>, nullptr},
                {&launchOne<3, 0>, &launchOne<3, 1>, &launchOne<3, 2>, &launchOne<3, 3>},
            };
            return (la < 4 && lb <= la) ? table[la][lb] : nullptr;
        }

        template <class T>
        void upload(DevBuf<T> &d, const std::vector<T> &h, cudaStream_t s)
        {
            d.reset(h.size());
            if (!h.empty())
                cudaCheck(cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s), "upload");
        }
    }

    namespace
    {
        // Device copies of the host fields of one pair class that the one-electron kernels read.
        struct OneClassData
        {
            DevBuf<double> ex, co, xy, na, nb;
            DevBuf<uint32_t> po;
            DevBuf<int32_t> ao, atoms, same;
            OneClassData(const PairClass &pc, cudaStream_t s)
            {
                std::vector<int32_t> ao_h(2 * pc.n_pairs), at_h(2 * pc.n_pairs), same_h(pc.n_pairs);
                for (size_t i = 0; i < pc.n_pairs; i++)
                {
                    ao_h[2 * i] = pc.ao_a[i];
                    ao_h[2 * i + 1] = pc.ao_b[i];
                    at_h[2 * i] = pc.atom_a[i];
                    at_h[2 * i + 1] = pc.atom_b[i];
                    same_h[i] = pc.shell_a[i] == pc.shell_b[i];
                }
                upload(ex, pc.exps, s);
                upload(co, pc.coeffs, s);
                upload(xy, pc.coords, s);
                upload(na, pc.norms_a, s);
                upload(nb, pc.norms_b, s);
                upload(po, pc.pofs, s);
                upload(ao, ao_h, s);
                upload(atoms, at_h, s);
                upload(same, same_h, s);
            }
        };
    }

    // The nuclei as point charges, one per atom in atom order: x, y, z (bohr), Z.
    std::vector<double> Engine::nucleiCharges() const
    {
        std::vector<double> q;
        int next = 0;
        for (const Shell &sh : shells_)
            if ((int)sh.atom == next)
            {
                q.insert(q.end(), {sh.xyz[0], sh.xyz[1], sh.xyz[2], (double)sh.z});
                next++;
            }
        if (next != n_atoms_)
            throw EngineError(kStatusInternal, "atoms without basis shells");
        return q;
    }

    namespace
    {
        // M[d][a][b] = blk, M[d'][b][a] = sign * blk for every stored pair block [pair][d][S_a][S_b];
        // d' = d, or the component (j, i) of d = (i, j) for the nine pVp blocks (comp_t).
        __global__ void scatterPairBlocks(const double *__restrict__ blocks, long long n_pairs, int nblk, int sa,
                                          int sb, const int32_t *__restrict__ ao, long long nao, double sign,
                                          int comp_t, double *__restrict__ M)
        {
            const long long per = (long long)nblk * sa * sb, total = n_pairs * per;
            for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
                 g += (long long)gridDim.x * blockDim.x)
            {
                const long long ip = g / per;
                const int o = (int)(g % per), d = o / (sa * sb), m = (o / sb) % sa, nn = o % sb;
                const long long r = ao[2 * ip] + m, c = ao[2 * ip + 1] + nn;
                const double v = blocks[g];
                const int dt = comp_t ? (d % 3) * 3 + d / 3 : d;
                M[((size_t)d * nao + r) * nao + c] = v;
                M[((size_t)dt * nao + c) * nao + r] = sign * v;
            }
        }

        // M[d] = (M[d] + sign M[d]^T) / 2, so the matrices are exactly symmetric (sign 1) or
        // antisymmetric with a zero diagonal (sign -1): the diagonal shell blocks are written from both
        // orientations of their element pairs, which agree only to rounding.
        __global__ void symmetrizeBlocks(double *M, long long nao, int nblk, double sign)
        {
            const long long total = (long long)nblk * nao * nao;
            for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
                 g += (long long)gridDim.x * blockDim.x)
            {
                const long long d = g / (nao * nao), r = (g / nao) % nao, c = g % nao;
                if (c < r)
                    continue;
                double *a = M + (d * nao + r) * nao + c, *b = M + (d * nao + c) * nao + r;
                if (c == r)
                {
                    if (sign < 0)
                        *a = 0.0;
                    continue;
                }
                const double m = 0.5 * (*a + sign * *b);
                *a = m;
                *b = sign * m;
            }
        }

        // pVp: M[(i,j)][r][c] and M[(j,i)][c][r] made equal (their mean), one unordered pair per thread.
        __global__ void symmetrizePvp(double *M, long long nao)
        {
            const long long total = 9 * nao * nao;
            for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
                 g += (long long)gridDim.x * blockDim.x)
            {
                const int d = (int)(g / (nao * nao));
                const long long r = (g / nao) % nao, c = g % nao;
                const int pd = (d % 3) * 3 + d / 3;
                if (pd < d || (pd == d && c <= r))
                    continue;
                double *x = M + ((size_t)d * nao + r) * nao + c, *y = M + ((size_t)pd * nao + c) * nao + r;
                const double m = 0.5 * (*x + *y);
                *x = m;
                *y = m;
            }
        }

        void checkOneOp(int op, const double *omegas_host, const double *origin)
        {
            if (op < 0 || op > kOpPVP)
                throw EngineError(kStatusInvalid, "bad one-electron operator");
            if (oneOpUsesOmegas(op) && !omegas_host)
                throw EngineError(kStatusInvalid, "the erf-attenuated operator needs one omega per charge");
            if ((op == kOpDipole || op == kOpAngular) && !origin)
                throw EngineError(kStatusInvalid, "the operator needs an origin");
        }
    }

    void Engine::oneElectronOperator(int op, const double *charges_host, int n_charges, const double *omegas_host,
                                     const double *origin, double *out_dev)
    {
        requireSingle();
        if (op < kOpDipole || (op > kOpVErf && op != kOpSOC && op != kOpPVP))
            throw EngineError(kStatusInvalid, "the whole-matrix operator form covers ops 6..9, 13 and 14");
        checkOneOp(op, omegas_host, origin);
        if (max_l_ > 3)
            throw EngineError(kStatusUnsupported, "one-electron kernels are instantiated for l <= 3");
        const std::vector<double> q = charges_host
                                          ? std::vector<double>(charges_host, charges_host + 4 * (size_t)n_charges)
                                          : nucleiCharges();
        const int nq = (int)(q.size() / 4);
        DevBuf<double> dq, dw;
        upload(dq, q, stream_);
        if (op == kOpVErf)
            upload(dw, std::vector<double>(omegas_host, omegas_host + nq), stream_);
        const int nblk = oneOpBlocks(op);
        const size_t n = nao_;
        cudaCheck(cudaMemsetAsync(out_dev, 0, (size_t)nblk * n * n * sizeof(double), stream_), "memset");
        const double sign = (op == kOpMomentum || op == kOpAngular || op == kOpSOC) ? -1.0 : 1.0;
        ClassSet &cs = mainSet(true);
        for (size_t c = 0; c < cs.host.size(); c++)
        {
            const PairClass &pc = cs.host[c];
            if (pc.n_pairs == 0)
                continue;
            const PairFn fn = op == kOpPVP ? lookupPvp(pc.la, pc.lb) : lookupPair(pc.la, pc.lb);
            if (!fn)
                throw EngineError(kStatusUnsupported, "one-electron kernels are instantiated for l <= 3");
            OneClassData d(pc, stream_);
            const int sa = 2 * pc.la + 1, sb = 2 * pc.lb + 1;
            DevBuf<double> blocks((size_t)pc.n_pairs * nblk * sa * sb);
            OnePairArgs a{};
            a.op = op;
            a.swap = 0;  // blocks in the stored orientation, scattered both ways below
            a.n_tasks = (long long)pc.n_pairs;
            a.list = nullptr;
            a.n_pairs = (int)pc.n_pairs;
            a.nao = (int)n;
            a.exps = d.ex.p;
            a.coeffs = d.co.p;
            a.coords = d.xy.p;
            a.norms_a = d.na.p;
            a.norms_b = d.nb.p;
            a.pofs = d.po.p;
            a.ao = d.ao.p;
            a.atoms = d.atoms.p;
            a.same = d.same.p;
            a.charges = dq.p;
            a.omegas = op == kOpVErf ? dw.p : nullptr;
            a.n_charges = nq;
            if (origin)
                for (int x = 0; x < 3; x++)
                    a.origin[x] = origin[x];
            a.boys = boys_;
            a.sph_rc = sph_rc_;
            a.sph_val = sph_val_;
            a.sph_ofs_a0 = sph_ofs_[pc.la];
            a.sph_ofs_a1 = sph_ofs_[pc.la + 1];
            a.sph_ofs_b0 = sph_ofs_[pc.lb];
            a.sph_ofs_b1 = sph_ofs_[pc.lb + 1];
            a.out = blocks.p;
            fn(a, stream_, false);
            const long long total = (long long)pc.n_pairs * nblk * sa * sb;
            scatterPairBlocks<<<(unsigned)std::min<long long>((total + 255) / 256, 148LL * 16), 256, 0, stream_>>>(
                blocks.p, (long long)pc.n_pairs, nblk, sa, sb, d.ao.p, (long long)n, sign, op == kOpPVP ? 1 : 0,
                out_dev);
            cudaCheck(cudaGetLastError(), "scatter");
            cudaCheck(cudaStreamSynchronize(stream_), "one-electron operator");
        }
        const long long total = (long long)nblk * (long long)n * (long long)n;
        const unsigned grid = (unsigned)std::min<long long>((total + 255) / 256, 148LL * 16);
        if (op == kOpPVP)
            symmetrizePvp<<<grid, 256, 0, stream_>>>(out_dev, (long long)n);
        else
            symmetrizeBlocks<<<grid, 256, 0, stream_>>>(out_dev, (long long)n, nblk, sign);
        cudaCheck(cudaGetLastError(), "symmetrize");
        cudaCheck(cudaStreamSynchronize(stream_), "one-electron operator");
    }

    void Engine::oneElectronBatch(bool use_symm, int cls, int op, long long n_tasks, const uint32_t *pairs_host,
                                  const double *charges_host, int n_charges, double *out_dev,
                                  const double *omegas_host, const double *origin)
    {
        requireSingle();
        ClassSet &cs = mainSet(use_symm);
        if (cls < 0 || cls >= (int)cs.host.size())
            throw EngineError(kStatusInvalid, "bad class index");
        checkOneOp(op, omegas_host, origin);
        const PairClass &pc = cs.host[cls];
        const PairFn fn = op == kOpPVP ? lookupPvp(pc.la, pc.lb) : lookupPair(pc.la, pc.lb);
        if (!fn)
            throw EngineError(kStatusUnsupported, "one-electron kernels are instantiated for l <= 3");
        if (n_tasks <= 0)
            return;
        std::vector<uint32_t> list(pairs_host, pairs_host + n_tasks);
        for (uint32_t i : list)
            if (i >= pc.n_pairs)
                throw EngineError(kStatusInvalid, "pair index out of range");
        std::vector<double> q = charges_host ? std::vector<double>(charges_host, charges_host + 4 * (size_t)n_charges)
                                             : nucleiCharges();
        OneClassData d(pc, stream_);
        DevBuf<uint32_t> dl;
        DevBuf<double> dq, dw;
        upload(dl, list, stream_);
        upload(dq, q, stream_);
        if (oneOpUsesOmegas(op))
            upload(dw, std::vector<double>(omegas_host, omegas_host + q.size() / 4), stream_);
        OnePairArgs a{};
        a.op = op;
        a.omegas = oneOpUsesOmegas(op) ? dw.p : nullptr;
        if (origin)
            for (int x = 0; x < 3; x++)
                a.origin[x] = origin[x];
        a.swap = cs.swapped[cls] ? 1 : 0;
        a.n_tasks = n_tasks;
        a.list = dl.p;
        a.n_pairs = (int)pc.n_pairs;
        a.nao = (int)nao_;
        a.exps = d.ex.p;
        a.coeffs = d.co.p;
        a.coords = d.xy.p;
        a.norms_a = d.na.p;
        a.norms_b = d.nb.p;
        a.pofs = d.po.p;
        a.ao = d.ao.p;
        a.atoms = d.atoms.p;
        a.same = d.same.p;
        a.charges = dq.p;
        a.n_charges = (int)(q.size() / 4);
        a.boys = boys_;
        a.sph_rc = sph_rc_;
        a.sph_val = sph_val_;
        a.sph_ofs_a0 = sph_ofs_[pc.la];
        a.sph_ofs_a1 = sph_ofs_[pc.la + 1];
        a.sph_ofs_b0 = sph_ofs_[pc.lb];
        a.sph_ofs_b1 = sph_ofs_[pc.lb + 1];
        a.out = out_dev;
        fn(a, stream_, false);
        cudaCheck(cudaStreamSynchronize(stream_), "one-electron batch");
    }

    void Engine::oneElectronGrad(const double *D_dev, const double *W_dev, double *grad_dev)
    {
        requireSingle();
        if (max_l_ > 3)
            throw EngineError(kStatusUnsupported, "one-electron kernels are instantiated for l <= 3");
        cudaCheck(cudaMemsetAsync(grad_dev, 0, (size_t)n_atoms_ * 3 * sizeof(double), stream_), "memset");
        if (!D_dev && !W_dev)
            return;
        const std::vector<double> q = nucleiCharges();
        DevBuf<double> dq;
        upload(dq, q, stream_);
        ClassSet &cs = mainSet(true);
        for (size_t c = 0; c < cs.host.size(); c++)
        {
            const PairClass &pc = cs.host[c];
            if (pc.n_pairs == 0)
                continue;
            OneClassData d(pc, stream_);
            OnePairArgs a{};
            a.n_tasks = (long long)pc.n_pairs;
            a.list = nullptr;
            a.n_pairs = (int)pc.n_pairs;
            a.nao = (int)nao_;
            a.exps = d.ex.p;
            a.coeffs = d.co.p;
            a.coords = d.xy.p;
            a.norms_a = d.na.p;
            a.norms_b = d.nb.p;
            a.pofs = d.po.p;
            a.ao = d.ao.p;
            a.atoms = d.atoms.p;
            a.same = d.same.p;
            a.charges = dq.p;
            a.n_charges = (int)(q.size() / 4);
            a.boys = boys_;
            a.sph_rc = sph_rc_;
            a.sph_val = sph_val_;
            a.sph_ofs_a0 = sph_ofs_[pc.la];
            a.sph_ofs_a1 = sph_ofs_[pc.la + 1];
            a.sph_ofs_b0 = sph_ofs_[pc.lb];
            a.sph_ofs_b1 = sph_ofs_[pc.lb + 1];
            a.D = D_dev;
            a.W = W_dev;
            a.grad = grad_dev;
            lookupPair(pc.la, pc.lb)(a, stream_, true);
            cudaCheck(cudaStreamSynchronize(stream_), "one-electron gradient");
        }
    }

    void Engine::oneElectron(const double *charges_host, int n_charges, bool nuclei, double *S_dev, double *T_dev,
                             double *V_dev)
    {
        requireSingle();
        if (max_l_ > 3)
            throw EngineError(kStatusUnsupported, "one-electron integrals are instantiated for l <= 3");
        const size_t n = nao_;
        // the point charges: the nuclei (one per atom, in atom order) or the caller's list
        std::vector<double> q;
        if (nuclei)
            q = nucleiCharges();
        else if (n_charges > 0)
            q.assign(charges_host, charges_host + 4 * (size_t)n_charges);
        DevBuf<double> dq;
        upload(dq, q, stream_);
        for (double *o : {S_dev, T_dev, V_dev})
            if (o)
                cudaCheck(cudaMemsetAsync(o, 0, n * n * sizeof(double), stream_), "memset");
        ClassSet &cs = mainSet(true);
        for (size_t c = 0; c < cs.host.size(); c++)
        {
            const PairClass &pc = cs.host[c];
            if (pc.n_pairs == 0)
                continue;
            const OneFn fn = lookupOne(pc.la, pc.lb);
            if (!fn)
                throw EngineError(kStatusUnsupported, "one-electron class not instantiated");
            std::vector<int32_t> ao(2 * pc.n_pairs);
            for (size_t i = 0; i < pc.n_pairs; i++)
            {
                ao[2 * i] = pc.ao_a[i];
                ao[2 * i + 1] = pc.ao_b[i];
            }
            DevBuf<double> ex, co, xy, na, nb;
            DevBuf<uint32_t> po;
            DevBuf<int32_t> dao;
            upload(ex, pc.exps, stream_);
            upload(co, pc.coeffs, stream_);
            upload(xy, pc.coords, stream_);
            upload(na, pc.norms_a, stream_);
            upload(nb, pc.norms_b, stream_);
            upload(po, pc.pofs, stream_);
            upload(dao, ao, stream_);
            OneArgs a{};
            a.n_pairs = (int)pc.n_pairs;
            a.nao = (int)n;
            a.exps = ex.p;
            a.coeffs = co.p;
            a.coords = xy.p;
            a.norms_a = na.p;
            a.norms_b = nb.p;
            a.pofs = po.p;
            a.ao = dao.p;
            a.charges = dq.p;
            a.n_charges = (int)(q.size() / 4);
            a.boys = boys_;
            a.sph_rc = sph_rc_;
            a.sph_val = sph_val_;
            a.sph_ofs_a0 = sph_ofs_[pc.la];
            a.sph_ofs_a1 = sph_ofs_[pc.la + 1];
            a.sph_ofs_b0 = sph_ofs_[pc.lb];
            a.sph_ofs_b1 = sph_ofs_[pc.lb + 1];
            a.S = S_dev;
            a.T = T_dev;
            a.V = V_dev;
            fn(a, stream_, num_sms_);
            // the class's staging buffers are freed at the end of this iteration
            cudaCheck(cudaStreamSynchronize(stream_), "one-electron");
        }
    }
}
