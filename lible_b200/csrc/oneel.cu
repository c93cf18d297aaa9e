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
        {
            std::vector<int> seen;
            for (const Shell &sh : shells_)
            {
                if (std::find(seen.begin(), seen.end(), (int)sh.atom) != seen.end())
                    continue;
                seen.push_back((int)sh.atom);
                q.insert(q.end(), {sh.xyz[0], sh.xyz[1], sh.xyz[2], (double)sh.z});
            }
        }
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
