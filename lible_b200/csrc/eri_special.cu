// The reference's less common two-electron kernels, as batched calls:
//   ERI4SOCKernel / ERI3SOCKernel (src/lible/ints/twoel/eri_kernel_funs.hpp:846-1090): spin-orbit
//     integrals, three Cartesian components of  E1_ab x (dR/dP E_cd^T),
//       x: E1_y R_z - E1_z R_y,  y: E1_z R_x - E1_x R_z,  z: E1_x R_y - E1_y R_x,
//     with R_k the Hermite matrix shifted by one along k (Boys to L + 1) and E1 the bra's Hermite
//     coefficients differentiated with respect to A - B;
//   ERI2D2Kernel (eri_kernel_funs.hpp:736-842): second derivatives of (P|Q), the 3 x 3 block
//     d2/dA dA from the Hermite matrix shifted by two (Boys to L + 2), completed by symmetry and
//     translational invariance (AB = -AA, BB = AA) into 6 x 6 blocks.
// These are not on a hot path, so one kernel serves every class with runtime sizes: one warp per
// quartet, the Boys values and the McMurchie-Davidson recursion in shared memory (the lanes split
// each level of the recursion), the ket contraction and the bra contraction split over the lanes.
#include "device_common.cuh"
#include "engine_api.hpp"
#include "ri_solve.hpp"

#include <vector>

namespace lible_b200
{
    namespace
    {
        constexpr int kSpecialSOC = 0, kSpecialD2 = 1;

        struct SpecialArgs
        {
            int mode;
            PairView bra, ket;
            int la, lb, lc, ld;        // class (auxiliary shells: lb / ld = 0)
            const double *boys;
            const uint32_t *list;      // [n][2]
            long long n_tasks;
            double *out;
            int flags;                 // bit 0: bra class stored with a and b exchanged, bit 1: ket
        };

        // (t, u, v) of combined Hermite index h.
        __device__ __forceinline__ void tuvOf(int h, int &t, int &u, int &v)
        {
            int n = 0;
            while (nherm(n) <= h)
                n++;
            int c = h - nherm(n - 1);
            // Cartesian index c inside level n: (j + k)(j + k + 1)/2 + k
            int jk = 0;
            while ((jk + 1) * (jk + 2) / 2 <= c)
                jk++;
            v = c - jk * (jk + 1) / 2;
            u = jk - v;
            t = n - jk;
        }

        // Boys F_0..F_N(x) with a runtime order (same method as boysF: Taylor sum of F_N about the
        // nearest grid point, downward recursion; asymptote beyond x = 30).
        __device__ void boysDyn(int N, double x, const double *tables, double *F)
        {
            if (x > kBoysLargeX)
            {
                const double rs = rsqrt(x), rx = rs * rs;
                F[0] = 0.88622692545275801365 * rs;
                for (int k = 1; k <= N; k++)
                    F[k] = F[k - 1] * ((k - 0.5) * rx);
                return;
            }
            const double *tab = tables + (size_t)N * kBoysTerms * kBoysPitch;
            const int iv = (int)rint(x);
            const double m = (double)iv - x;
            double s = __ldg(tab + (kBoysTerms - 1) * kBoysPitch + iv);
            for (int k = kBoysTerms - 2; k >= 0; k--)
                s = fma(s, m, __ldg(tab + k * kBoysPitch + iv));
            F[N] = s;
            const double ex = exp(-x);
            for (int k = N - 1; k >= 0; k--)
                F[k] = (2.0 * x * F[k + 1] + ex) / (2 * k + 1);
        }

        // R_tuv (t + u + v <= L) into the warp's buffer R from F (prefactors included), the
        // recursion of hermiteR with runtime L; the lanes split the entries of each level.
        __device__ void hermiteRWarp(int L, double m2a, const double *F, double X, double Y, double Z, double *R,
                                     int lane)
        {
            double pw[16];
            pw[0] = 1.0;
            for (int n = 1; n <= L; n++)
                pw[n] = pw[n - 1] * m2a;
            if (lane == 0)
                R[0] = F[L] * pw[L];
            __syncwarp();
            for (int n = L - 1; n >= 0; n--)
            {
                for (int m = L - n; m >= 1; m--)
                {
                    const int lo = nherm(m - 1), hi = nherm(m);
                    for (int id = lo + lane; id < hi; id += 32)
                    {
                        int t, u, v;
                        tuvOf(id, t, u, v);
                        double r;
                        if (t > 0)
                        {
                            r = X * R[hermIndex(t - 1, u, v)];
                            if (t > 1)
                                r += (t - 1) * R[hermIndex(t - 2, u, v)];
                        }
                        else if (u > 0)
                        {
                            r = Y * R[hermIndex(t, u - 1, v)];
                            if (u > 1)
                                r += (u - 1) * R[hermIndex(t, u - 2, v)];
                        }
                        else
                        {
                            r = Z * R[hermIndex(t, u, v - 1)];
                            if (v > 1)
                                r += (v - 1) * R[hermIndex(t, u, v - 2)];
                        }
                        R[id] = r;
                    }
                    __syncwarp();
                }
                if (lane == 0)
                    R[0] = F[n] * pw[n];
                __syncwarp();
            }
        }

        __global__ void __launch_bounds__(32) specialKernel(SpecialArgs a)
        {
            extern __shared__ __align__(16) double sm[];
            const int lane = threadIdx.x;
            const long long task = blockIdx.x;
            if (task >= a.n_tasks)
                return;
            const uint32_t ib = a.list[2 * task], ik = a.list[2 * task + 1];
            const bool soc = a.mode == kSpecialSOC;
            const int lab = a.la + a.lb, lcd = a.lc + a.ld, L = lab + lcd, sh = soc ? 1 : 2;
            const int sab = nsph(a.la) * nsph(a.lb), scd = nsph(a.lc) * nsph(a.ld);
            const int hab = nherm(lab), hcd = nherm(lcd);
            const int ncomp = soc ? 3 : 6;
            double *F = sm;                              // L + 3
            double *R = F + 16;                          // nherm(L + sh)
            double *rxe = R + nherm(L + sh);             // ncomp x hab x scd
            double *acc = rxe + ncomp * hab * scd;       // ncomp x sab x scd
            for (int e = lane; e < ncomp * sab * scd; e += 32)
                acc[e] = 0.0;
            // shifts of the R matrix per component: SOC x, y, z; D2 xx, xy, xz, yy, yz, zz
            const int sx[6] = {1, 0, 0, 2, 1, 1}, sy[6] = {0, 1, 0, 0, 1, 0}, sz[6] = {0, 0, 1, 0, 0, 1};
            const int d2x[6] = {2, 1, 1, 0, 0, 0}, d2y[6] = {0, 1, 0, 2, 1, 0}, d2z[6] = {0, 0, 1, 0, 1, 2};
            for (uint32_t p = a.bra.pofs[ib]; p < a.bra.pofs[ib + 1]; p++)
            {
                const PQ4 P = loadPQ(a.bra.pP, p);
                for (int e = lane; e < ncomp * hab * scd; e += 32)
                    rxe[e] = 0.0;
                __syncwarp();
                for (uint32_t q = a.ket.pofs[ik]; q < a.ket.pofs[ik + 1]; q++)
                {
                    const PQ4 Q = loadPQ(a.ket.pP, q);
                    const double pq = P.x + Q.x, alpha = P.x * Q.x / pq;
                    const double X = P.y - Q.y, Y = P.z - Q.z, Z = P.w - Q.w;
                    const double fac = 34.986836655249725 / (P.x * Q.x * sqrt(pq));  // 2 pi^{5/2}
                    if (lane == 0)
                    {
                        boysDyn(L + sh, alpha * (X * X + Y * Y + Z * Z), a.boys, F);
                        for (int k = 0; k <= L + sh; k++)
                            F[k] *= fac;
                    }
                    __syncwarp();
                    hermiteRWarp(L + sh, -2.0 * alpha, F, X, Y, Z, R, lane);
                    // rxe[c][h][k] += sum_h' (-1)^{|h'|} R[h + h' + shift_c] Et_cd[q][h'][k]
                    const double *et = a.ket.Et + (size_t)q * hcd * scd;
                    for (int e = lane; e < ncomp * hab * scd; e += 32)
                    {
                        const int c = e / (hab * scd), h = (e / scd) % hab, k = e % scd;
                        int t, u, v;
                        tuvOf(h, t, u, v);
                        const int ax = soc ? sx[c] : d2x[c], ay = soc ? sy[c] : d2y[c], az = soc ? sz[c] : d2z[c];
                        double s = 0.0;
                        for (int hp = 0; hp < hcd; hp++)
                        {
                            int tp, up, vp;
                            tuvOf(hp, tp, up, vp);
                            const double r = R[hermIndex(t + tp + ax, u + up + ay, v + vp + az)];
                            const double ev = __ldg(et + (size_t)hp * scd + k);
                            s += ((tp + up + vp) & 1) ? -r * ev : r * ev;
                        }
                        rxe[e] += s;
                    }
                    __syncwarp();
                }
                // bra contraction of this primitive pair
                for (int e = lane; e < ncomp * sab * scd; e += 32)
                {
                    const int c = e / (sab * scd), mn = (e / scd) % sab, k = e % scd;
                    double s = 0.0;
                    if (soc)
                    {
                        // component c uses (E1_j, R_k) - (E1_k, R_j) with (j, k) = (y, z), (z, x), (x, y)
                        const int j = (c + 1) % 3, kk = (c + 2) % 3;
                        const double *e1 = a.bra.E1 + (size_t)p * 3 * sab * hab;
                        for (int h = 0; h < hab; h++)
                            s += __ldg(e1 + ((size_t)j * sab + mn) * hab + h) * rxe[(kk * hab + h) * scd + k] -
                                 __ldg(e1 + ((size_t)kk * sab + mn) * hab + h) * rxe[(j * hab + h) * scd + k];
                    }
                    else
                    {
                        const double *e0 = a.bra.E + (size_t)p * sab * hab;
                        for (int h = 0; h < hab; h++)
                            s += __ldg(e0 + (size_t)mn * hab + h) * rxe[(c * hab + h) * scd + k];
                    }
                    acc[e] += s;
                }
                __syncwarp();
            }
            const int blk = sab * scd;
            if (soc)
            {
                // the caller's orientation: a stored bra (ket) pair with exchanged shells is written
                // transposed; for the bra, E1 = d/d(A - B) also changes sign
                const int sa = nsph(a.la), sb = nsph(a.lb), sc = nsph(a.lc), sd = nsph(a.ld);
                const double sgn = (a.flags & 1) ? -1.0 : 1.0;
                double *out = a.out + (size_t)task * 3 * blk;
                for (int e = lane; e < 3 * blk; e += 32)
                {
                    const int c = e / blk, mn = (e / scd) % sab, k = e % scd;
                    const int mo = (a.flags & 1) ? (mn % sb) * sa + mn / sb : mn;
                    const int ko = (a.flags & 2) ? (k % sd) * sc + k / sd : k;
                    out[(size_t)c * blk + mo * scd + ko] = sgn * acc[e];
                }
            }
            else
            {
                // [6][6][Sa][Sb]: AA from the 6 unique components, AB = BA = -AA, BB = AA
                const int uidx[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
                double *out = a.out + (size_t)task * 36 * blk;
                for (int e = lane; e < 36 * blk; e += 32)
                {
                    const int i = e / (6 * blk), j = (e / blk) % 6, x = e % blk;
                    const double v = acc[uidx[i % 3][j % 3] * blk + x];
                    out[e] = ((i < 3) == (j < 3)) ? v : -v;
                }
            }
        }
    }

    void Engine::specialBatch(int kind, bool use_symm, int c_ab, int c_cd, long long n, const uint32_t *pairs_host,
                              double *out_dev)
    {
        requireSingle();
        if (n <= 0)
            return;
        // kind 0: ERI4SOC (main, main), 1: ERI3SOC (main, aux), 2: ERI2D2 (aux, aux)
        ClassSet &bs = kind == 2 ? auxSet() : mainSet(use_symm);
        ClassSet &ks = kind == 0 ? mainSet(use_symm) : auxSet();
        if (c_ab < 0 || c_ab >= (int)bs.dev.size() || c_cd < 0 || c_cd >= (int)ks.dev.size())
            throw EngineError(kStatusInvalid, "bad class index");
        const DevPairClass &B = bs.dev[c_ab], &K = ks.dev[c_cd];
        for (long long i = 0; i < n; i++)
            if (pairs_host[2 * i] >= B.n_pairs || pairs_host[2 * i + 1] >= K.n_pairs)
                throw EngineError(kStatusInvalid, "pair index out of range");
        SpecialArgs a{};
        a.mode = kind == 2 ? kSpecialD2 : kSpecialSOC;
        a.flags = (kind != 2 && bs.swapped[c_ab] ? 1 : 0) | (kind == 0 && ks.swapped[c_cd] ? 2 : 0);
        a.bra = view(B);
        a.ket = view(K);
        a.la = B.la;
        a.lb = B.lb;
        a.lc = K.la;
        a.ld = K.lb;
        if (a.la + a.lb + a.lc + a.ld + (kind == 2 ? 2 : 1) > kBoysMaxN)
            throw EngineError(kStatusUnsupported, "class beyond the Boys tables");
        a.boys = boys_;
        const int lab = a.la + a.lb, lcd = a.lc + a.ld, L = lab + lcd, sh = kind == 2 ? 2 : 1;
        const int sab = nsph(a.la) * nsph(a.lb), scd = nsph(a.lc) * nsph(a.ld), nc = kind == 2 ? 6 : 3;
        const size_t doubles = 16 + nherm(L + sh) + (size_t)nc * nherm(lab) * scd + (size_t)nc * sab * scd;
        const size_t smem = doubles * sizeof(double);
        if (smem > 227 * 1024)
            throw EngineError(kStatusUnsupported, "class too large for the special-kernel layout");
        DevBuf<uint32_t> dl(2 * (size_t)n);
        cudaCheck(cudaMemcpyAsync(dl.p, pairs_host, 2 * (size_t)n * sizeof(uint32_t), cudaMemcpyHostToDevice, stream_),
                  "upload");
        a.list = dl.p;
        a.n_tasks = n;
        a.out = out_dev;
        if (smem > 48 * 1024)
            cudaCheck(cudaFuncSetAttribute(specialKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                      "attr");
        for (long long t0 = 0; t0 < n; t0 += 1LL << 30)
        {
            SpecialArgs b = a;
            b.list = a.list + 2 * t0;
            b.n_tasks = std::min<long long>(n - t0, 1LL << 30);
            b.out = a.out + (size_t)t0 * (kind == 2 ? 36 : 3) * sab * scd;
            specialKernel<<<(unsigned)b.n_tasks, 32, smem, stream_>>>(b);
            cudaCheck(cudaGetLastError(), "special kernel");
        }
        cudaCheck(cudaStreamSynchronize(stream_), "special batch");
    }
}
