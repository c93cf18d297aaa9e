// Host orchestration of the B200 ERI engine: device residency of the pair classes, the
// E-coefficient kernel, Schwarz screening, the drivers (eri4 / eri4Diagonal / eri3 / eri2 /
// eri2Diagonal, kernel-API batches, direct J/K, RI-J, J/K gradient) and their support kernels.
#include "engine_api.hpp"
#include "eri_kernel.cuh"  // operand pitches and the bounded barrier wait
#include "eri_launch.cuh"

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <numeric>
#include <stdexcept>

namespace lible_b200
{
    // ------------------------------------------------------------------------------------------
    // Support kernels

    struct SphTables
    {
        const int *rc;       // [n][2] row, cart
        const double *val;   // [n]
        int ofs[kMaxL + 2];  // first entry of shell l
    };

    struct EArgs
    {
        int la, lb;
        size_t n_pairs, n_ppairs;
        const double *exps, *coeffs, *coords, *norms_a, *norms_b;
        const uint32_t *pofs;
        SphTables sph;
        double *pP, *ab, *E, *Et, *E1, *E1t;
        float *Ef, *Etf;
        float *pPf;  // FP32 record [ppair][8]: p, 1/p, P (hi), P - hi (lo)
    };

    // Hermite E matrices of every primitive pair of one class, with the spherical transforms of both
    // shells, the AO norms and the contraction coefficients folded in:
    //   E[mu nu][tuv] = N_mu N_nu d_a d_b sum_{i in mu} sum_{j in nu} T_a T_b E^x_{ij,t} E^y E^z
    // (src/lible/ints/ecoeffs.cpp:314-403) and its derivative with respect to A - B
    // (src/lible/ints/ecoeffs.cpp:405-517).  One thread per primitive pair.
    __global__ void ecoeffKernel(EArgs a)
    {
        const size_t ip = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (ip >= a.n_ppairs)
            return;
        // owning pair by binary search over the primitive offsets
        size_t lo = 0, hi = a.n_pairs - 1;
        while (lo < hi)
        {
            size_t mid = (lo + hi + 1) / 2;
            if (a.pofs[mid] <= ip)
                lo = mid;
            else
                hi = mid - 1;
        }
        const size_t ipair = lo;
        const int la = a.la, lb = a.lb, lab = la + lb;
        const int sa = nsph(la), sb = nsph(lb), hab = nherm(lab), sab = sa * sb;
        const double ea = a.exps[2 * ip], eb = a.exps[2 * ip + 1];
        const double dadb = a.coeffs[2 * ip] * a.coeffs[2 * ip + 1];
        const double *A = a.coords + 6 * ipair, *B = A + 3;
        const double p = ea + eb, mu = ea * eb / p;
        double P[3], Ex[3][128], E1x[3][128];
        for (int k = 0; k < 3; k++)
        {
            P[k] = (ea * A[k] + eb * B[k]) / p;
            const double kab = exp(-mu * (A[k] - B[k]) * (A[k] - B[k]));
            hermiteE(la, lb, 1.0 / (2 * p), P[k] - A[k], P[k] - B[k], kab, Ex[k]);
            if (a.E1)
                hermiteE1(la, lb, ea, eb, A[k] - B[k], Ex[k], E1x[k]);
        }
        a.pP[8 * ip + 0] = p;
        a.pP[8 * ip + 1] = P[0];
        a.pP[8 * ip + 2] = P[1];
        a.pP[8 * ip + 3] = P[2];
        a.pP[8 * ip + 4] = 1.0 / p;
        a.pP[8 * ip + 5] = ea;
        a.pP[8 * ip + 6] = eb;
        a.pP[8 * ip + 7] = 0.0;
        if (a.pPf)
        {
            // P split into float hi + lo parts: (P - Q) then keeps float relative accuracy even for
            // nearby centres far from the origin
            float *f = a.pPf + 8 * ip;
            f[0] = (float)p;
            f[1] = (float)(1.0 / p);
            for (int k = 0; k < 3; k++)
            {
                const float hi = (float)P[k];
                f[2 + k] = hi;
                f[5 + k] = (float)(P[k] - (double)hi);
            }
        }
        a.ab[2 * ip + 0] = ea;
        a.ab[2 * ip + 1] = eb;
        const int nt = lab + 1;
        auto ex = [&](const double *E, int i, int j, int t) { return E[(i * (lb + 1) + j) * nt + t]; };
        const double *na = a.norms_a + ipair * sa, *nb = a.norms_b + ipair * sb;
        double acc[4][84];
        for (int m = 0; m < sa; m++)
            for (int n = 0; n < sb; n++)
            {
                for (int x = 0; x < 4; x++)
                    for (int h = 0; h < hab; h++)
                        acc[x][h] = 0.0;
                for (int ta = a.sph.ofs[la]; ta < a.sph.ofs[la + 1]; ta++)
                {
                    if (a.sph.rc[2 * ta] != m)
                        continue;
                    int ca = a.sph.rc[2 * ta + 1];
                    // Cartesian exponents of index ca in shell la
                    int ia = 0, ja = 0, ka = 0;
                    for (int x = la, c = 0; x >= 0; x--)
                        for (int y = la - x; y >= 0; y--, c++)
                            if (c == ca)
                            {
                                ia = x;
                                ja = y;
                                ka = la - x - y;
                            }
                    for (int tb = a.sph.ofs[lb]; tb < a.sph.ofs[lb + 1]; tb++)
                    {
                        if (a.sph.rc[2 * tb] != n)
                            continue;
                        int cb = a.sph.rc[2 * tb + 1];
                        int ib = 0, jb = 0, kb = 0;
                        for (int x = lb, c = 0; x >= 0; x--)
                            for (int y = lb - x; y >= 0; y--, c++)
                                if (c == cb)
                                {
                                    ib = x;
                                    jb = y;
                                    kb = lb - x - y;
                                }
                        const double w = a.sph.val[ta] * a.sph.val[tb];
                        for (int t = 0; t <= ia + ib; t++)
                            for (int u = 0; u <= ja + jb; u++)
                                for (int v = 0; v <= ka + kb; v++)
                                {
                                    const int h = hermIndex(t, u, v);
                                    const double gx = ex(Ex[0], ia, ib, t), gy = ex(Ex[1], ja, jb, u),
                                                 gz = ex(Ex[2], ka, kb, v);
                                    acc[0][h] += w * gx * gy * gz;
                                    if (a.E1)
                                    {
                                        acc[1][h] += w * ex(E1x[0], ia, ib, t) * gy * gz;
                                        acc[2][h] += w * gx * ex(E1x[1], ja, jb, u) * gz;
                                        acc[3][h] += w * gx * gy * ex(E1x[2], ka, kb, v);
                                    }
                                }
                    }
                }
                const double s = na[m] * nb[n] * dadb;
                const int mn = m * sb + n;
                for (int h = 0; h < hab; h++)
                {
                    const double v = s * acc[0][h];
                    a.E[(ip * sab + mn) * hab + h] = v;
                    a.Et[(ip * hab + h) * sab + mn] = v;
                    if (a.Ef)
                    {
                        a.Ef[(ip * sab + mn) * hab + h] = (float)v;
                        a.Etf[(ip * hab + h) * sab + mn] = (float)v;
                    }
                    if (a.E1)
                        for (int x = 0; x < 3; x++)
                        {
                            const double v1 = s * acc[1 + x][h];
                            a.E1[((ip * 3 + x) * sab + mn) * hab + h] = v1;
                            a.E1t[((ip * 3 + x) * hab + h) * sab + mn] = v1;
                        }
                }
            }
    }

    // eri4 scatter with 8-fold permutational symmetry (src/lible/ints/twoel/eri4.cpp:70-89).
    __global__ void scatter4Kernel(const double *batches, const uint32_t *list, long long n_tasks,
                                   const int32_t *bra_info, const int32_t *ket_info, int sa, int sb,
                                   int sc, int sd, long long n, double *out)
    {
        const long long blk = (long long)sa * sb * sc * sd;
        const long long total = n_tasks * blk;
        for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
             g += (long long)gridDim.x * blockDim.x)
        {
            const long long t = g / blk;
            int e = (int)(g % blk);
            const int l = e % sd;
            e /= sd;
            const int k = e % sc;
            e /= sc;
            const int j = e % sb;
            const int i = e / sb;
            const int32_t *bi = bra_info + 8 * list[2 * t];
            const int32_t *ki = ket_info + 8 * list[2 * t + 1];
            const long long m = bi[0] + i, nu = bi[1] + j, ka = ki[0] + k, ta = ki[1] + l;
            const double v = batches[g];
            out[((m * n + nu) * n + ka) * n + ta] = v;
            out[((m * n + nu) * n + ta) * n + ka] = v;
            out[((nu * n + m) * n + ka) * n + ta] = v;
            out[((nu * n + m) * n + ta) * n + ka] = v;
            out[((ka * n + ta) * n + m) * n + nu] = v;
            out[((ka * n + ta) * n + nu) * n + m] = v;
            out[((ta * n + ka) * n + m) * n + nu] = v;
            out[((ta * n + ka) * n + nu) * n + m] = v;
        }
    }

    // eri3 scatter: (mn|P) and (nm|P) (src/lible/ints/twoel/eri3.cpp:30-43).  Batches are stored in
    // the caller orientation [S_a][S_b][S_P].
    __global__ void scatter3Kernel(const double *batches, const uint32_t *list, long long n_tasks,
                                   const int32_t *main_info, const int32_t *aux_info, int swap, int sa,
                                   int sb, int sc, long long n, long long naux, double *out)
    {
        const long long blk = (long long)sa * sb * sc;
        const long long total = n_tasks * blk;
        for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
             g += (long long)gridDim.x * blockDim.x)
        {
            const long long t = g / blk;
            int e = (int)(g % blk);
            const int k = e % sc;
            e /= sc;
            const int j = e % sb;
            const int i = e / sb;
            const uint32_t im = swap ? list[2 * t + 1] : list[2 * t];
            const uint32_t ix = swap ? list[2 * t] : list[2 * t + 1];
            const int32_t *mi = main_info + 8 * im;
            const int32_t *xi = aux_info + 8 * ix;
            const long long m = mi[0] + i, nu = mi[1] + j, P = xi[0] + k;
            out[(m * n + nu) * naux + P] = batches[g];
            out[(nu * n + m) * naux + P] = batches[g];
        }
    }

    // eri2 scatter (src/lible/ints/twoel/eri2.cpp:61-66); batches [S_a][S_b] in caller order.
    __global__ void scatter2Kernel(const double *batches, const uint32_t *list, long long n_tasks,
                                   const int32_t *a_info, const int32_t *b_info, int swap, int sa, int sb,
                                   long long naux, double *out)
    {
        const long long blk = (long long)sa * sb;
        const long long total = n_tasks * blk;
        for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
             g += (long long)gridDim.x * blockDim.x)
        {
            const long long t = g / blk;
            const int e = (int)(g % blk);
            const int j = e % sb, i = e / sb;
            const uint32_t ia = swap ? list[2 * t + 1] : list[2 * t];
            const uint32_t ibb = swap ? list[2 * t] : list[2 * t + 1];
            const long long P = a_info[8 * ia] + i, Q = b_info[8 * ibb] + j;
            out[P * naux + Q] = batches[g];
            out[Q * naux + P] = batches[g];
        }
    }

    // X = A + A^T for the unsymmetrised J / K accumulators (in place, n x n).
    __global__ void symmetrizeKernel(double *A, long long n)
    {
        for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < n * n;
             g += (long long)gridDim.x * blockDim.x)
        {
            const long long r = g / n, c = g % n;
            if (c > r)
                continue;
            const double v = A[r * n + c] + A[c * n + r];
            A[r * n + c] = v;
            A[c * n + r] = v;
        }
    }

    // Builds the bra-side structure-of-arrays copies of one class in Schwarz order (layout in
    // DevPairClass): block-strided over positions, threads over (primitive, field).
    __global__ void soaGatherKernel(const double *E, const float *Ef, const double *pP, const float *pPf,
                                    const uint32_t *pofs, const uint32_t *order, const uint4 *soa, long long n_pos,
                                    int sabhab, double *Es, float *Efs, double *pPs, float *pPfs)
    {
        for (long long j = blockIdx.x; j < n_pos; j += gridDim.x)
        {
            const uint32_t pair = order[j], p0 = pofs[pair], K = pofs[pair + 1] - p0;
            const uint4 sv = soa[j];
            const size_t n = sv.z;
            for (int idx = threadIdx.x; idx < (int)K * sabhab; idx += blockDim.x)
            {
                const size_t src = (size_t)p0 * sabhab + idx;
                Es[sv.y + (size_t)idx * n] = E[src];
                if (Efs)
                    Efs[sv.y + (size_t)idx * n] = Ef[src];
            }
            for (int idx = threadIdx.x; idx < (int)K * 5; idx += blockDim.x)
            {
                const int k = idx / 5, f = idx % 5;
                pPs[sv.x + (size_t)idx * n] = pP[8 * ((size_t)p0 + k) + (f < 4 ? f : 4)];
            }
            if (pPfs)
                for (int idx = threadIdx.x; idx < (int)K * 8; idx += blockDim.x)
                    pPfs[sv.w + (size_t)idx * n] = pPf[8 * (size_t)p0 + idx];
        }
    }

    // Ket E tiles zero-padded to the DMMA operand layout of their class: out[pp][rows][pitch] with
    // the Et[pp][h'][c] entries for h' < hcd, c < scd and zeros elsewhere (bulk-copied whole).
    __global__ void padEtKernel(const double *Et, long long n_pp, int hcd, int scd, int rows, int pitch, double *out)
    {
        const long long total = n_pp * rows * pitch;
        for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
             idx += (long long)gridDim.x * blockDim.x)
        {
            const long long pp = idx / ((long long)rows * pitch);
            const int r = (int)((idx / pitch) % rows), c = (int)(idx % pitch);
            out[idx] = (r < hcd && c < scd) ? Et[((size_t)pp * hcd + r) * scd + c] : 0.0;
        }
    }

    // D_ab blocks of every bra pair of a class in Schwarz order: Dab[mn * n_pos + position].
    __global__ void dabGatherKernel(const double *D, const int4 *soa2, long long n_pos, int sa, int sb, double *Dab)
    {
        const long long total = n_pos * sa * sb;
        for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
             idx += (long long)gridDim.x * blockDim.x)
        {
            const long long pos = idx % n_pos;
            const int mn = (int)(idx / n_pos), m = mn / sb, nn = mn % sb;
            const int4 si = soa2[pos];
            const int n = si.w & 0xffff;
            Dab[idx] = D[(size_t)(uint32_t)si.z + (size_t)(si.x + m) * n + si.y + nn];
        }
    }

    // A_m <- A_m + A_m^T for every packed block m = blockIdx.y (blocks[2m] = first element,
    // blocks[2m+1] = N_m).
    __global__ void symmetrizeBlocksKernel(double *A, const long long *blocks)
    {
        const long long base = blocks[2 * blockIdx.y], n = blocks[2 * blockIdx.y + 1];
        double *M = A + base;
        for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < n * n;
             g += (long long)gridDim.x * blockDim.x)
        {
            const long long r = g / n, c = g % n;
            if (c > r)
                continue;
            const double v = M[r * n + c] + M[c * n + r];
            M[r * n + c] = v;
            M[c * n + r] = v;
        }
    }

    // Reorders D1 batches from the internal orientation to the caller's, selecting the caller's
    // derivative blocks: out[t][slot(c)*3 + x][caller element] = in[t][c*3 + x][internal element].
    __global__ void reorderD1Kernel(const double *in, long long n_tasks, int sa, int sb, int sc, int sd,
                                    int flags, int4 slot, int nblk_out, double *out)
    {
        const long long blk = (long long)sa * sb * sc * sd;
        const long long total = n_tasks * 12 * blk;
        for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
             g += (long long)gridDim.x * blockDim.x)
        {
            const long long t = g / (12 * blk);
            const int bl = (int)((g / blk) % 12);
            int e = (int)(g % blk);
            const int centre = bl / 3, x = bl % 3;
            const int s = centre == 0 ? slot.x : centre == 1 ? slot.y : centre == 2 ? slot.z : slot.w;
            if (s < 0)
                continue;
            const int tt = e % sd;
            e /= sd;
            const int k = e % sc;
            e /= sc;
            const int nn = e % sb;
            const int m = e / sb;
            int b0 = m, b1 = nn, k0 = k, k1 = tt, db0 = sa, db1 = sb, dk0 = sc, dk1 = sd;
            if (flags & 1)
            {
                b0 = nn; b1 = m; db0 = sb; db1 = sa;
            }
            if (flags & 2)
            {
                k0 = tt; k1 = k; dk0 = sd; dk1 = sc;
            }
            const long long d = (flags & 4) ? (((long long)k0 * dk1 + k1) * db0 + b0) * db1 + b1
                                            : (((long long)b0 * db1 + b1) * dk0 + k0) * dk1 + k1;
            out[(t * nblk_out + s * 3 + x) * blk + d] = in[g];
        }
    }

    // ------------------------------------------------------------------------------------------
    // Engine

    void cudaCheck(cudaError_t e, const char *what)
    {
        if (e != cudaSuccess)
            throw EngineError(kStatusCuda, std::string(what) + ": " + cudaGetErrorString(e));
    }

    template <class T>
    static T *devAlloc(size_t n)
    {
        T *p = nullptr;
        if (n == 0)
            n = 1;
        cudaCheck(cudaMalloc(&p, n * sizeof(T)), "cudaMalloc");
        return p;
    }

    template <class T>
    static T *devUpload(const std::vector<T> &v, cudaStream_t s)
    {
        T *p = devAlloc<T>(v.size());
        if (!v.empty())
            cudaCheck(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s), "upload");
        return p;
    }

    // Device allocation released on scope exit, also when a check throws (cudaFree synchronises,
    // so a kernel still reading the buffer finishes first).
    struct CudaFreeDeleter
    {
        void operator()(void *p) const { cudaFree(p); }
    };
    template <class T>
    using DevPtr = std::unique_ptr<T, CudaFreeDeleter>;

    Engine::Engine(int device) : device_(device)
    {
        cudaCheck(cudaSetDevice(device), "cudaSetDevice");
        cudaCheck(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
        cudaDeviceProp prop;
        cudaCheck(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
        num_sms_ = prop.multiProcessorCount;
        gpu_name_ = prop.name;
        for (int b = 0; b < kBranches; b++)
        {
            cudaCheck(cudaStreamCreateWithFlags(&branch_[b], cudaStreamNonBlocking), "cudaStreamCreate");
            cudaCheck(cudaEventCreateWithFlags(&join_[b], cudaEventDisableTiming), "cudaEventCreate");
        }
        cudaCheck(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming), "cudaEventCreate");
        d_status_ = devAlloc<int>(1);
        cudaCheck(cudaMemset(d_status_, 0, sizeof(int)), "memset");
        boys_ = devUpload(boysGrid(), stream_);
        boys_f_ = devUpload(boysGridF(), stream_);
        std::vector<int> rc;
        std::vector<double> val;
        sph_ofs_.assign(kMaxL + 2, 0);
        for (int l = 0; l <= kMaxL; l++)
        {
            sph_ofs_[l] = (int)val.size();
            for (const auto &t : sphericalTrafo(l))
            {
                rc.push_back(t.row);
                rc.push_back(t.cart);
                val.push_back(t.val);
            }
        }
        sph_ofs_[kMaxL + 1] = (int)val.size();
        sph_rc_ = devUpload(rc, stream_);
        sph_val_ = devUpload(val, stream_);
        cudaCheck(cudaStreamSynchronize(stream_), "init");
    }

    Engine::~Engine()
    {
        cudaSetDevice(device_);
        clearStructure();
        for (void *p : persistent_)
            cudaFree(p);
        for (double *p : staging_)
            cudaFree(p);
        cudaFree(d_status_);
        cudaFree(boys_);
        cudaFree(boys_f_);
        cudaFree(sph_rc_);
        cudaFree(sph_val_);
        for (int b = 0; b < kBranches; b++)
        {
            cudaStreamDestroy(branch_[b]);
            cudaEventDestroy(join_[b]);
        }
        cudaEventDestroy(fork_);
        cudaStreamDestroy(stream_);
    }

    void Engine::releaseGraph()
    {
        if (graph_exec_)
            cudaGraphExecDestroy(graph_exec_);
        graph_exec_ = nullptr;
        graph_key_.clear();
    }

    void Engine::freeSet(ClassSet &cs)
    {
        for (auto &d : cs.dev)
            for (void *p : {(void *)d.pP, (void *)d.ab, (void *)d.pofs, (void *)d.info, (void *)d.coords,
                            (void *)d.E, (void *)d.Et, (void *)d.Ef, (void *)d.Etf, (void *)d.E1,
                            (void *)d.E1t, (void *)d.Q, (void *)d.pPs, (void *)d.Es, (void *)d.Efs,
                            (void *)d.soa, (void *)d.pPf, (void *)d.pPfs, (void *)d.soa2, (void *)d.Dab,
                            (void *)d.EtP})
                cudaFree(p);
        for (auto &o : cs.orders)
        {
            cudaFree(o.d_order);
            cudaFree(o.d_q);
        }
        cs = ClassSet();
    }

    void Engine::clearStructure()
    {
        releaseGraph();
        cudaFree(d_blocks_);
        d_blocks_ = nullptr;
        batch_ = false;
        mol_shells_.clear();
        mol_nao_.clear();
        mol_base_.clear();
        packed_ = 0;
        freeSet(symm_);
        freeSet(nosymm_);
        freeSet(aux_);
        for (auto &kv : plans_)
            freePlan(kv.second);
        plans_.clear();
        for (auto &kv : ri_plans_)
            freePlan(kv.second);
        ri_plans_.clear();
        shells_.clear();
        aux_shells_.clear();
        nao_ = naux_ = 0;
        n_atoms_ = 0;
        has_structure_ = false;
    }

    void Engine::setStructure(const std::vector<BasisAtom> &main, const std::vector<BasisAtom> *aux,
                              const std::vector<std::array<double, 3>> &xyz_bohr)
    {
        clearStructure();
        shells_ = constructShells(main, xyz_bohr);
        nao_ = 0;
        max_l_ = 0;
        for (const auto &s : shells_)
        {
            nao_ += nsph(s.l);
            max_l_ = std::max(max_l_, s.l);
        }
        if (max_l_ > 3)
            throw EngineError(kStatusUnsupported, "main basis shells with l > 3 are not supported");
        n_atoms_ = (int)xyz_bohr.size();
        has_aux_ = aux != nullptr;
        if (aux)
        {
            aux_shells_ = constructShells(*aux, xyz_bohr);
            naux_ = 0;
            max_l_aux_ = 0;
            for (const auto &s : aux_shells_)
            {
                naux_ += nsph(s.l);
                max_l_aux_ = std::max(max_l_aux_, s.l);
            }
        }
        mol_nao_ = {(long long)nao_};
        mol_base_ = {0};
        packed_ = (long long)(nao_ * nao_);
        d_blocks_ = devUpload(std::vector<long long>{0, (long long)nao_}, stream_);
        cudaCheck(cudaStreamSynchronize(stream_), "upload");
        has_structure_ = true;
    }

    void Engine::setBatch(const std::vector<std::vector<BasisAtom>> &mols,
                          const std::vector<std::vector<std::array<double, 3>>> &xyz_bohr)
    {
        clearStructure();
        if (mols.empty() || mols.size() != xyz_bohr.size())
            throw EngineError(kStatusInvalid, "a batch needs one coordinate set per molecule");
        size_t shell_ofs = 0, atom_ofs = 0;
        std::vector<long long> blocks;
        max_l_ = 0;
        nao_ = 0;
        for (size_t m = 0; m < mols.size(); m++)
        {
            auto sh = constructShells(mols[m], xyz_bohr[m]);
            long long n = 0;
            for (auto &x : sh)
            {
                x.mol = (int)m;
                x.idx += shell_ofs;
                x.atom += atom_ofs;
                n += nsph(x.l);
                max_l_ = std::max(max_l_, x.l);
            }
            shell_ofs += sh.size();
            atom_ofs += xyz_bohr[m].size();
            mol_nao_.push_back(n);
            mol_base_.push_back(packed_);
            blocks.push_back(packed_);
            blocks.push_back(n);
            packed_ += n * n;
            nao_ += (size_t)n;
            shells_.insert(shells_.end(), sh.begin(), sh.end());
            mol_shells_.push_back(std::move(sh));
        }
        if (max_l_ > 3)
            throw EngineError(kStatusUnsupported, "main basis shells with l > 3 are not supported");
        if (packed_ >= (1LL << 31))
            throw EngineError(kStatusInvalid, "batch too large: packed matrices exceed 2^31 elements");
        n_atoms_ = (int)atom_ofs;
        has_aux_ = false;
        batch_ = true;
        d_blocks_ = devUpload(blocks, stream_);
        cudaCheck(cudaStreamSynchronize(stream_), "upload");
        has_structure_ = true;
    }

    std::vector<Shell> Engine::shellsL(const std::vector<Shell> &all, int l)
    {
        std::vector<Shell> out;
        for (const auto &s : all)
            if (s.l == l)
                out.push_back(s);
        return out;
    }

    void Engine::uploadClass(const PairClass &pc, bool with_d1, bool with_f32, DevPairClass &d)
    {
        d.la = pc.la;
        d.lb = pc.lb;
        d.single = pc.single;
        d.n_pairs = pc.n_pairs;
        d.n_ppairs = pc.n_ppairs;
        std::vector<int32_t> info(8 * pc.n_pairs, 0);
        for (size_t i = 0; i < pc.n_pairs; i++)
        {
            info[8 * i + 0] = pc.ao_a[i];
            info[8 * i + 1] = pc.ao_b[i];
            info[8 * i + 2] = pc.atom_a[i];
            info[8 * i + 3] = pc.atom_b[i];
            info[8 * i + 4] = pc.shell_a[i];
            info[8 * i + 5] = pc.shell_b[i];
            info[8 * i + 6] = pc.mat_base.empty() ? 0 : pc.mat_base[i];
            info[8 * i + 7] = pc.mat_n.empty() ? (int32_t)nao_ : pc.mat_n[i];
        }
        d.info = devUpload(info, stream_);
        d.pofs = devUpload(pc.pofs, stream_);
        d.coords = devUpload(pc.coords, stream_);
        const size_t np = std::max<size_t>(pc.n_ppairs, 1);
        const int sab = nsph(pc.la) * nsph(pc.lb), hab = nherm(pc.la + pc.lb);
        d.pP = devAlloc<double>(8 * np);
        d.ab = devAlloc<double>(2 * np);
        d.E = devAlloc<double>(np * sab * hab);
        d.Et = devAlloc<double>(np * sab * hab);
        if (with_f32)
        {
            d.Ef = devAlloc<float>(np * sab * hab);
            d.Etf = devAlloc<float>(np * sab * hab);
            d.pPf = devAlloc<float>(8 * np);
        }
        if (with_d1)
        {
            d.E1 = devAlloc<double>(3 * np * sab * hab);
            d.E1t = devAlloc<double>(3 * np * sab * hab);
        }
        if (pc.n_ppairs == 0)
            return;
        DevPtr<double> exps(devUpload(pc.exps, stream_)), coeffs(devUpload(pc.coeffs, stream_)),
            na(devUpload(pc.norms_a, stream_)), nb(devUpload(pc.norms_b, stream_));
        EArgs ea{};
        ea.la = pc.la;
        ea.lb = pc.lb;
        ea.n_pairs = pc.n_pairs;
        ea.n_ppairs = pc.n_ppairs;
        ea.exps = exps.get();
        ea.coeffs = coeffs.get();
        ea.coords = d.coords;
        ea.norms_a = na.get();
        ea.norms_b = nb.get();
        ea.pofs = d.pofs;
        ea.sph.rc = sph_rc_;
        ea.sph.val = sph_val_;
        for (int l = 0; l <= kMaxL + 1; l++)
            ea.sph.ofs[l] = sph_ofs_[l];
        ea.pP = d.pP;
        ea.ab = d.ab;
        ea.E = d.E;
        ea.Et = d.Et;
        ea.Ef = d.Ef;
        ea.Etf = d.Etf;
        ea.pPf = d.pPf;
        ea.E1 = d.E1;
        ea.E1t = d.E1t;
        const int bs = 64;
        ecoeffKernel<<<(unsigned)((pc.n_ppairs + bs - 1) / bs), bs, 0, stream_>>>(ea);
        cudaCheck(cudaGetLastError(), "ecoeffKernel");
        {
            // padded ket tiles for the bulk copies of the DMMA class kernels
            const int hcd = nherm(pc.la + pc.lb), scd = nsph(pc.la) * nsph(pc.lb);
            const int rows = (hcd + 3) / 4 * 4, pitch = kPitch(scd);
            const long long tot = (long long)pc.n_ppairs * rows * pitch;
            d.EtP = devAlloc<double>((size_t)std::max<long long>(tot, 1));
            padEtKernel<<<(unsigned)std::min<long long>((tot + 255) / 256, 65535), 256, 0, stream_>>>(
                d.Et, (long long)pc.n_ppairs, hcd, scd, rows, pitch, d.EtP);
            cudaCheck(cudaGetLastError(), "padEtKernel");
        }
        cudaCheck(cudaStreamSynchronize(stream_), "ecoeffKernel");
    }

    // Reference class order: la = 0..lmax, lb = 0..la (symmetric) or lb = 0..lmax (no symmetry)
    // (src/lible/ints/utils.cpp:49-73, shell_pair_data.cpp:294-309).
    Engine::ClassSet &Engine::mainSet(bool use_symm)
    {
        requireStructure();
        ClassSet &cs = use_symm ? symm_ : nosymm_;
        if (!cs.host.empty() || cs.built)
            return cs;
        for (int la = 0; la <= max_l_; la++)
            for (int lb = 0; lb <= (use_symm ? la : max_l_); lb++)
            {
                PairClass pc;
                if (batch_)
                {
                    // pairs only within a molecule, tagged with the molecule's packed block
                    for (size_t m = 0; m < mol_shells_.size(); m++)
                        appendPairClass(pc, buildPairClass(use_symm, la, lb, shellsL(mol_shells_[m], la),
                                                           shellsL(mol_shells_[m], lb)),
                                        (int32_t)mol_base_[m], (int32_t)mol_nao_[m]);
                    if (pc.pofs.empty())
                    {
                        pc.la = la;
                        pc.lb = lb;
                        pc.pofs.push_back(0);
                    }
                }
                else
                    pc = buildPairClass(use_symm, la, lb, shellsL(shells_, la), shellsL(shells_, lb));
                bool swapped = false;
                if (lb > la)
                {
                    // store with the higher angular momentum first; the caller's orientation is
                    // restored by the epilogue
                    swapped = true;
                    for (size_t i = 0; i < pc.n_ppairs; i++)
                    {
                        std::swap(pc.exps[2 * i], pc.exps[2 * i + 1]);
                        std::swap(pc.coeffs[2 * i], pc.coeffs[2 * i + 1]);
                    }
                    for (size_t i = 0; i < pc.n_pairs; i++)
                        for (int k = 0; k < 3; k++)
                            std::swap(pc.coords[6 * i + k], pc.coords[6 * i + 3 + k]);
                    std::swap(pc.ao_a, pc.ao_b);
                    std::swap(pc.atom_a, pc.atom_b);
                    std::swap(pc.shell_a, pc.shell_b);
                    std::swap(pc.norms_a, pc.norms_b);
                    std::swap(pc.la, pc.lb);
                }
                cs.host.push_back(std::move(pc));
                cs.swapped.push_back(swapped);
                cs.req_l.push_back({la, lb});
            }
        cs.dev.resize(cs.host.size());
        for (size_t c = 0; c < cs.host.size(); c++)
            uploadClass(cs.host[c], true, use_symm, cs.dev[c]);
        cs.built = true;
        return cs;
    }

    Engine::ClassSet &Engine::auxSet()
    {
        requireStructure();
        if (!has_aux_)
            throw EngineError(kStatusNoAux, "RI approximation is not enabled (no auxiliary basis)");
        if (aux_.built)
            return aux_;
        for (int l = 0; l <= max_l_aux_; l++)
        {
            aux_.host.push_back(buildSingleClass(l, shellsL(aux_shells_, l)));
            aux_.swapped.push_back(false);
            aux_.req_l.push_back({l, 0});
        }
        aux_.dev.resize(aux_.host.size());
        for (size_t c = 0; c < aux_.host.size(); c++)
            uploadClass(aux_.host[c], true, false, aux_.dev[c]);
        aux_.built = true;
        return aux_;
    }

    void Engine::requireStructure() const
    {
        if (!has_structure_)
            throw EngineError(kStatusNoStructure, "no structure has been set");
    }

    void Engine::requireSingle() const
    {
        requireStructure();
        if (batch_)
            throw EngineError(kStatusUnsupported, "this call takes a single structure, not a batch");
    }

    PairView Engine::view(const DevPairClass &d)
    {
        return PairView{d.pP, d.ab, d.pofs, d.info, d.E, d.Et, d.Ef, d.Etf, d.E1, d.E1t, d.pPf};
    }

    // Runs one class pair over an explicit task list in store mode.  `bra` and `ket` are in the
    // caller's orientation; the class is launched with the larger pair type in the bra.
    void Engine::runStore(const DevPairClass &bra, bool bra_swapped, const DevPairClass &ket, bool ket_swapped,
                          const uint32_t *d_list, long long n, bool d1, double *d_out, bool same_class)
    {
        const int inject = wait_inject_;
        wait_inject_ = 0;
        if (n == 0)
            return;
        const int tb = pairType(bra.la, bra.lb), tk = pairType(ket.la, ket.lb);
        const bool swap = tb < tk;
        QuartetArgs a{};
        a.bra = view(swap ? ket : bra);
        a.ket = view(swap ? bra : ket);
        a.ket_EtP = (swap ? bra : ket).EtP;
        a.boys = boys_;
        a.boys_f = boys_f_;
        a.status = d_status_;
        a.wait_inject = inject;
        cudaCheck(cudaMemsetAsync(d_status_, 0, sizeof(int), stream_), "memset");
        a.n_tasks = n;
        a.same_class = same_class ? 1 : 0;
        a.flags = (bra_swapped ? 1 : 0) | (ket_swapped ? 2 : 0) | (swap ? 4 : 0);
        if (swap)
            a.flags = (ket_swapped ? 1 : 0) | (bra_swapped ? 2 : 0) | 4;
        uint32_t *list = const_cast<uint32_t *>(d_list);
        DevPtr<uint32_t> swapped_list;
        if (swap)
        {
            // swap the (bra, ket) columns of the task list
            std::vector<uint32_t> h(2 * n);
            cudaCheck(cudaMemcpyAsync(h.data(), d_list, 2 * n * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_), "list");
            cudaCheck(cudaStreamSynchronize(stream_), "list");
            for (long long i = 0; i < n; i++)
                std::swap(h[2 * i], h[2 * i + 1]);
            swapped_list.reset(devUpload(h, stream_));
            list = swapped_list.get();
        }
        a.list = list;
        if (!d1)
        {
            a.mode = kStore;
            a.out = d_out;
            LaunchFn fn = lookupFwd64(swap ? tk : tb, swap ? tb : tk);
            if (!fn)
                throw EngineError(kStatusUnsupported, "quartet class not instantiated");
            cudaCheck(fn(a, stream_, num_sms_), "eri kernel");
        }
        else
        {
            const long long blk = (long long)nsph(bra.la) * nsph(bra.lb) * nsph(ket.la) * nsph(ket.lb);
            DevPtr<double> tmp(devAlloc<double>(n * 12 * blk));
            a.mode = kD1Store;
            a.out = tmp.get();
            const int flags = a.flags;
            a.flags = 0;
            LaunchFn fn = lookupD1(swap ? tk : tb, swap ? tb : tk);
            if (!fn)
                throw EngineError(kStatusUnsupported, "quartet class not instantiated");
            cudaCheck(fn(a, stream_, num_sms_), "eri d1 kernel");
            // caller slots of the internal centres (A, B | C, D)
            int s[4] = {0, 1, 2, 3};
            if (flags & 1)
                std::swap(s[0], s[1]);
            if (flags & 2)
                std::swap(s[2], s[3]);
            if (flags & 4)
                for (int &x : s)
                    x = (x + 2) % 4;
            // drop the derivative blocks of auxiliary dummy centres; compact the remaining slots
            const DevPairClass &ib = swap ? ket : bra, &ik = swap ? bra : ket;
            bool dummy[4] = {false, ib.single, false, ik.single};
            int callerDummy[4] = {0, 0, 0, 0};
            for (int c = 0; c < 4; c++)
                if (dummy[c])
                    callerDummy[s[c]] = 1;
            int remap[4], k = 0;
            for (int c = 0; c < 4; c++)
                remap[c] = callerDummy[c] ? -1 : k++;
            int4 slot = make_int4(remap[s[0]], remap[s[1]], remap[s[2]], remap[s[3]]);
            if (ib.single)
                slot.y = -1;
            if (ik.single)
                slot.w = -1;
            const int nb = 3 * k;
            const auto &sb = swap ? ket : bra;
            const auto &sk = swap ? bra : ket;
            reorderD1Kernel<<<std::max(1, num_sms_ * 8), 256, 0, stream_>>>(
                tmp.get(), n, nsph(sb.la), nsph(sb.lb), nsph(sk.la), nsph(sk.lb), flags, slot, nb, d_out);
            cudaCheck(cudaGetLastError(), "reorder");
            cudaCheck(cudaStreamSynchronize(stream_), "reorder");
        }
        // a bounded wait that gave up makes the call fail (synchronises, so the swapped list stays
        // alive until the kernel is done)
        checkStatus();
    }

    // ------------------------------------------------------------------------------------------
    // Full tensors

    void Engine::eri4(double *out_dev)
    {
        requireSingle();
        ClassSet &cs = mainSet(true);
        const long long n = (long long)nao_;
        cudaCheck(cudaMemsetAsync(out_dev, 0, (size_t)n * n * n * n * sizeof(double), stream_), "memset");
        for (size_t cb = 0; cb < cs.dev.size(); cb++)
            for (size_t ck = 0; ck <= cb; ck++)
            {
                const auto &B = cs.dev[cb], &K = cs.dev[ck];
                std::vector<uint32_t> list;
                for (uint32_t i = 0; i < B.n_pairs; i++)
                    for (uint32_t j = 0; j < (cb == ck ? i + 1 : K.n_pairs); j++)
                    {
                        list.push_back(i);
                        list.push_back(j);
                    }
                const long long nt = (long long)list.size() / 2;
                if (nt == 0)
                    continue;
                DevPtr<uint32_t> dl(devUpload(list, stream_));
                const int sa = nsph(B.la), sb = nsph(B.lb), sc = nsph(K.la), sd = nsph(K.lb);
                DevPtr<double> tmp(devAlloc<double>((size_t)nt * sa * sb * sc * sd));
                runStore(B, false, K, false, dl.get(), nt, false, tmp.get(), cb == ck);
                scatter4Kernel<<<num_sms_ * 8, 256, 0, stream_>>>(tmp.get(), dl.get(), nt, B.info, K.info, sa, sb, sc,
                                                                   sd, n, out_dev);
                cudaCheck(cudaGetLastError(), "scatter4");
                cudaCheck(cudaStreamSynchronize(stream_), "eri4");
            }
    }

    // Diagonal batches (ab|ab) of every pair of every class (the eri4Diagonal analogue).
    std::vector<std::vector<double>> Engine::diagonalBatches(ClassSet &cs)
    {
        std::vector<std::vector<double>> out(cs.dev.size());
        for (size_t c = 0; c < cs.dev.size(); c++)
        {
            const auto &B = cs.dev[c];
            if (B.n_pairs == 0)
                continue;
            std::vector<uint32_t> list;
            for (uint32_t i = 0; i < B.n_pairs; i++)
            {
                list.push_back(i);
                list.push_back(i);
            }
            DevPtr<uint32_t> dl(devUpload(list, stream_));
            const size_t sab = (size_t)nsph(B.la) * nsph(B.lb);
            DevPtr<double> tmp(devAlloc<double>(B.n_pairs * sab * sab));
            runStore(B, false, B, false, dl.get(), (long long)B.n_pairs, false, tmp.get(), true);
            out[c].resize(B.n_pairs * sab * sab);
            cudaCheck(cudaMemcpyAsync(out[c].data(), tmp.get(), out[c].size() * sizeof(double),
                                      cudaMemcpyDeviceToHost, stream_), "diag");
            cudaCheck(cudaStreamSynchronize(stream_), "diag");
        }
        return out;
    }

    void Engine::eri4Diagonal(double *out_host)
    {
        requireSingle();
        ClassSet &cs = mainSet(true);
        auto batches = diagonalBatches(cs);
        const size_t n = nao_;
        std::fill(out_host, out_host + n * n, 0.0);
        for (size_t c = 0; c < cs.host.size(); c++)
        {
            const auto &pc = cs.host[c];
            const int sa = nsph(pc.la), sb = nsph(pc.lb), sab = sa * sb;
            for (size_t i = 0; i < pc.n_pairs; i++)
                for (int x = 0; x < sa; x++)
                    for (int y = 0; y < sb; y++)
                    {
                        const int e = x * sb + y;
                        const double v = batches[c][(i * sab + e) * sab + e];
                        const size_t mu = pc.ao_a[i] + x, nu = pc.ao_b[i] + y;
                        out_host[mu * n + nu] = v;
                        out_host[nu * n + mu] = v;
                    }
        }
    }

    void Engine::eri3(double *out_dev)
    {
        requireSingle();
        ClassSet &ms = mainSet(true);
        ClassSet &xs = auxSet();
        const long long n = (long long)nao_, na = (long long)naux_;
        cudaCheck(cudaMemsetAsync(out_dev, 0, (size_t)n * n * na * sizeof(double), stream_), "memset");
        for (size_t cb = 0; cb < ms.dev.size(); cb++)
            for (size_t cx = 0; cx < xs.dev.size(); cx++)
            {
                const auto &B = ms.dev[cb], &X = xs.dev[cx];
                std::vector<uint32_t> list;
                for (uint32_t i = 0; i < B.n_pairs; i++)
                    for (uint32_t j = 0; j < X.n_pairs; j++)
                    {
                        list.push_back(i);
                        list.push_back(j);
                    }
                const long long nt = (long long)list.size() / 2;
                if (nt == 0)
                    continue;
                DevPtr<uint32_t> dl(devUpload(list, stream_));
                const int sa = nsph(B.la), sb = nsph(B.lb), sc = nsph(X.la);
                DevPtr<double> tmp(devAlloc<double>((size_t)nt * sa * sb * sc));
                runStore(B, false, X, false, dl.get(), nt, false, tmp.get(), false);
                scatter3Kernel<<<num_sms_ * 8, 256, 0, stream_>>>(tmp.get(), dl.get(), nt, B.info, X.info, 0, sa, sb,
                                                                   sc, n, na, out_dev);
                cudaCheck(cudaGetLastError(), "scatter3");
                cudaCheck(cudaStreamSynchronize(stream_), "eri3");
            }
    }

    void Engine::eri2(double *out_dev)
    {
        requireSingle();
        ClassSet &xs = auxSet();
        const long long na = (long long)naux_;
        cudaCheck(cudaMemsetAsync(out_dev, 0, (size_t)na * na * sizeof(double), stream_), "memset");
        for (size_t ca = 0; ca < xs.dev.size(); ca++)
            for (size_t cb = 0; cb <= ca; cb++)
            {
                const auto &A = xs.dev[ca], &B = xs.dev[cb];
                std::vector<uint32_t> list;
                for (uint32_t i = 0; i < A.n_pairs; i++)
                    for (uint32_t j = 0; j < (ca == cb ? i + 1 : B.n_pairs); j++)
                    {
                        list.push_back(i);
                        list.push_back(j);
                    }
                const long long nt = (long long)list.size() / 2;
                if (nt == 0)
                    continue;
                DevPtr<uint32_t> dl(devUpload(list, stream_));
                const int sa = nsph(A.la), sb = nsph(B.la);
                DevPtr<double> tmp(devAlloc<double>((size_t)nt * sa * sb));
                runStore(A, false, B, false, dl.get(), nt, false, tmp.get(), ca == cb);
                scatter2Kernel<<<num_sms_ * 8, 256, 0, stream_>>>(tmp.get(), dl.get(), nt, A.info, B.info, 0, sa, sb, na,
                                                                   out_dev);
                cudaCheck(cudaGetLastError(), "scatter2");
                cudaCheck(cudaStreamSynchronize(stream_), "eri2");
            }
    }

    void Engine::eri2Diagonal(double *out_host)
    {
        requireSingle();
        ClassSet &xs = auxSet();
        auto batches = diagonalBatches(xs);
        std::fill(out_host, out_host + naux_, 0.0);
        for (size_t c = 0; c < xs.host.size(); c++)
        {
            const auto &pc = xs.host[c];
            const int s = nsph(pc.la);
            for (size_t i = 0; i < pc.n_pairs; i++)
                for (int x = 0; x < s; x++)
                    out_host[pc.ao_a[i] + x] = batches[c][(i * s + x) * s + x];
        }
    }

    // ------------------------------------------------------------------------------------------
    // Kernel-API batches: the caller's classes follow shellPairData(use_symm) / shellDataAux.

    void Engine::eri4Batch(bool use_symm, int cab, int ccd, long long n, const uint32_t *pairs_host, double *out_dev,
                           bool d1)
    {
        requireSingle();
        ClassSet &cs = mainSet(use_symm);
        if (cab < 0 || ccd < 0 || cab >= (int)cs.dev.size() || ccd >= (int)cs.dev.size())
            throw EngineError(kStatusInvalid, "class index out of range");
        const auto &B = cs.dev[cab], &K = cs.dev[ccd];
        for (long long i = 0; i < n; i++)
            if (pairs_host[2 * i] >= B.n_pairs || pairs_host[2 * i + 1] >= K.n_pairs)
                throw EngineError(kStatusInvalid, "pair index out of range");
        std::vector<uint32_t> list(pairs_host, pairs_host + 2 * n);
        DevPtr<uint32_t> dl(devUpload(list, stream_));
        runStore(B, cs.swapped[cab], K, cs.swapped[ccd], dl.get(), n, d1, out_dev, use_symm && cab == ccd);
        cudaCheck(cudaStreamSynchronize(stream_), "batch");
    }

    void Engine::eri3Batch(bool use_symm, int cab, int cx, long long n, const uint32_t *idx_host, double *out_dev,
                           bool d1)
    {
        requireSingle();
        ClassSet &cs = mainSet(use_symm);
        ClassSet &xs = auxSet();
        if (cab < 0 || cx < 0 || cab >= (int)cs.dev.size() || cx >= (int)xs.dev.size())
            throw EngineError(kStatusInvalid, "class index out of range");
        const auto &B = cs.dev[cab], &X = xs.dev[cx];
        for (long long i = 0; i < n; i++)
            if (idx_host[2 * i] >= B.n_pairs || idx_host[2 * i + 1] >= X.n_pairs)
                throw EngineError(kStatusInvalid, "index out of range");
        std::vector<uint32_t> list(idx_host, idx_host + 2 * n);
        DevPtr<uint32_t> dl(devUpload(list, stream_));
        runStore(B, cs.swapped[cab], X, false, dl.get(), n, d1, out_dev, false);
        cudaCheck(cudaStreamSynchronize(stream_), "batch");
    }

    void Engine::eri2Batch(int ca, int cb, long long n, const uint32_t *idx_host, double *out_dev, bool d1)
    {
        requireSingle();
        ClassSet &xs = auxSet();
        if (ca < 0 || cb < 0 || ca >= (int)xs.dev.size() || cb >= (int)xs.dev.size())
            throw EngineError(kStatusInvalid, "class index out of range");
        const auto &A = xs.dev[ca], &B = xs.dev[cb];
        for (long long i = 0; i < n; i++)
            if (idx_host[2 * i] >= A.n_pairs || idx_host[2 * i + 1] >= B.n_pairs)
                throw EngineError(kStatusInvalid, "index out of range");
        std::vector<uint32_t> list(idx_host, idx_host + 2 * n);
        DevPtr<uint32_t> dl(devUpload(list, stream_));
        runStore(A, false, B, false, dl.get(), n, d1, out_dev, false);
        cudaCheck(cudaStreamSynchronize(stream_), "batch");
    }

    // ------------------------------------------------------------------------------------------
    // Schwarz screening and the direct J/K build

    // Schwarz factors Q_ab = max sqrt|(mn|mn)| of every pair, and the per-class Schwarz order:
    // pairs grouped by their number of primitive pairs K, decreasing Q inside a group.
    void Engine::ensureSchwarz(ClassSet &cs)
    {
        if (cs.schwarz_done)
            return;
        auto batches = diagonalBatches(cs);
        cs.orders.resize(cs.dev.size());
        for (size_t c = 0; c < cs.dev.size(); c++)
        {
            auto &d = cs.dev[c];
            const int sab = nsph(d.la) * nsph(d.lb);
            d.Qh.assign(d.n_pairs, 0.0);
            for (size_t i = 0; i < d.n_pairs; i++)
            {
                double m = 0.0;
                for (int e = 0; e < sab; e++)
                    m = std::max(m, std::fabs(batches[c][(i * sab + e) * sab + e]));
                d.Qh[i] = std::sqrt(m);
            }
            d.Q = devUpload(d.Qh, stream_);
            const auto &Q = d.Qh;
            const auto &pofs = cs.host[c].pofs;
            const auto &mb = cs.host[c].mat_base;
            auto K = [&](uint32_t x) { return pofs[x + 1] - pofs[x]; };
            auto M = [&](uint32_t x) { return mb.empty() ? 0 : mb[x]; };
            // Q buckets of a factor 4: pairs of one bucket survive or fail against most kets together
            auto bucket = [&](uint32_t x) { return Q[x] > 0 ? (int)std::floor(0.5 * std::log2(Q[x])) : INT_MIN; };
            const auto &hc0 = cs.host[c];
            ClassOrder &o = cs.orders[c];
            o.order.resize(Q.size());
            std::iota(o.order.begin(), o.order.end(), 0u);
            // (molecule, K, bucket descending, AO of a, AO of b): inside a bucket, consecutive pairs
            // share shells and neighbouring AOs, so a warp's digestion touches few rows of D, J, K
            std::stable_sort(o.order.begin(), o.order.end(), [&](uint32_t x, uint32_t y) {
                if (M(x) != M(y))
                    return M(x) < M(y);
                if (K(x) != K(y))
                    return K(x) < K(y);
                if (bucket(x) != bucket(y))
                    return bucket(x) > bucket(y);
                if (hc0.ao_a[x] != hc0.ao_a[y])
                    return hc0.ao_a[x] < hc0.ao_a[y];
                return hc0.ao_b[x] < hc0.ao_b[y];
            });
            o.q.resize(Q.size());
            for (size_t i = 0; i < Q.size(); i++)
            {
                const uint32_t x = o.order[i];
                o.q[i] = Q[x];
                if (o.groups.empty() || o.groups.back().k != K(x) || o.groups.back().mol != M(x) ||
                    o.groups.back().bucket != bucket(x))
                    o.groups.push_back({K(x), (uint32_t)i, (uint32_t)i, M(x), bucket(x), Q[x], Q[x]});
                auto &g = o.groups.back();
                g.end = (uint32_t)i + 1;
                g.qmax = std::max(g.qmax, Q[x]);
                g.qmin = std::min(g.qmin, Q[x]);
            }
            o.qs = o.q;
            for (const auto &g : o.groups)
                std::sort(o.qs.begin() + g.start, o.qs.begin() + g.end, std::greater<double>());
            o.d_order = devUpload(o.order, stream_);
            o.d_q = devUpload(o.q, stream_);
            // bra-side structure-of-arrays copies in this order
            const int sabhab = nsph(d.la) * nsph(d.lb) * nherm(d.la + d.lb);
            std::vector<uint4> soa(Q.size());
            size_t base_p = 0, base_e = 0, base_f = 0;
            for (const auto &g : o.groups)
            {
                const uint32_t ng = g.end - g.start;
                for (uint32_t i = 0; i < ng; i++)
                    soa[g.start + i] =
                        make_uint4((unsigned)(base_p + i), (unsigned)(base_e + i), ng, (unsigned)(base_f + i));
                base_p += (size_t)g.k * 5 * ng;
                base_e += (size_t)g.k * sabhab * ng;
                base_f += (size_t)g.k * 8 * ng;
            }
            if (base_e >= (1ULL << 32) || base_p >= (1ULL << 32))
                throw EngineError(kStatusInvalid, "pair class too large for 32-bit structure-of-arrays offsets");
            // per-position bra fields for the J/K digestion
            std::vector<int4> soa2(Q.size());
            const auto &hc = cs.host[c];
            for (size_t j = 0; j < Q.size(); j++)
            {
                const uint32_t x = o.order[j];
                const int mn = hc.mat_n.empty() ? (int)nao_ : hc.mat_n[x];
                const int kk = (int)K(x);
                if (mn >= (1 << 16) || kk >= (1 << 15))
                    throw EngineError(kStatusInvalid, "molecule or contraction too large for the packed pair fields");
                const bool same = hc.shell_a[x] == hc.shell_b[x];
                soa2[j] = make_int4(hc.ao_a[x], hc.ao_b[x], hc.mat_base.empty() ? 0 : hc.mat_base[x],
                                    (int)((unsigned)mn | ((unsigned)kk << 16) | (same ? 0x80000000u : 0u)));
            }
            if (!soa.empty())
            {
                d.soa = devUpload(soa, stream_);
                d.soa2 = devUpload(soa2, stream_);
                d.Dab = devAlloc<double>(soa.size() * nsph(d.la) * nsph(d.lb));
                d.pPs = devAlloc<double>(std::max<size_t>(base_p, 1));
                d.Es = devAlloc<double>(std::max<size_t>(base_e, 1));
                if (d.Ef)
                {
                    d.Efs = devAlloc<float>(std::max<size_t>(base_e, 1));
                    d.pPfs = devAlloc<float>(std::max<size_t>(base_f, 1));
                }
                soaGatherKernel<<<(unsigned)std::min<size_t>(soa.size(), 65535), 128, 0, stream_>>>(
                    d.E, d.Ef, d.pP, d.pPf, d.pofs, o.d_order, d.soa, (long long)soa.size(), sabhab, d.Es, d.Efs,
                    d.pPs, d.pPfs);
                cudaCheck(cudaGetLastError(), "soaGatherKernel");
            }
        }
        cudaCheck(cudaStreamSynchronize(stream_), "schwarz");
        cs.schwarz_done = true;
    }

    void Engine::freePlan(JKPlan &p)
    {
        for (auto &cp : p.pairs)
            for (void *x : {(void *)cp.prefix64, (void *)cp.prefix32, (void *)cp.begin64, (void *)cp.begin32,
                            (void *)cp.majors, (void *)cp.chunks64, (void *)cp.chunks32, (void *)cp.chunksD1})
                cudaFree(x);
        cudaFree(p.counters);
        p = JKPlan();
    }

    // Cuts a task sequence into work-queue chunks.  Tasks come in runs (major entries) of n[i] tasks
    // costing c[i] each (primitive quartets plus a fixed per-quartet overhead).  A chunk closes once
    // it holds the cost of `unit` tasks of the most expensive run (one full worker step of the
    // heaviest quartets) or `max_tasks` tasks, whichever comes first; with the heaviest runs first
    // in the task order and chunks claimed dynamically, the last chunks to finish are cheap ones.
    static std::vector<unsigned long long> costChunks(const std::vector<unsigned long long> &n,
                                                      const std::vector<double> &c, int unit, int max_tasks)
    {
        double cmax = 0;
        for (size_t i = 0; i < n.size(); i++)
            if (n[i])
                cmax = std::max(cmax, c[i]);
        const double C = (double)std::max(unit, 1) * cmax;
        std::vector<unsigned long long> ch(1, 0);
        unsigned long long pos = 0, cnt = 0;
        double acc = 0;
        for (size_t i = 0; i < n.size(); i++)
        {
            unsigned long long left = n[i];
            while (left > 0)
            {
                const unsigned long long by_cost =
                    std::max<unsigned long long>(1, (unsigned long long)std::ceil((C - acc) / c[i]));
                const unsigned long long by_count = (unsigned long long)max_tasks - cnt;
                const unsigned long long k = std::min(by_cost, by_count);
                if (k > left)
                {
                    acc += (double)left * c[i];
                    cnt += left;
                    pos += left;
                    left = 0;
                }
                else
                {
                    pos += k;
                    left -= k;
                    ch.push_back(pos);
                    acc = 0;
                    cnt = 0;
                }
            }
        }
        if (ch.back() != pos)
            ch.push_back(pos);
        return ch;
    }

    // Surviving quartets of one class pair, kept iff Q_bra Q_ket >= thr (and, with `triangle`, only
    // the unique ones of a class paired with itself).  Both classes are in their Schwarz order, so the
    // surviving bras of a ket are a prefix of each bra group.  Tasks are enumerated ket-major per
    // (bra group, ket group) segment: "major" entries m = (ket pair, bra group) own the task range
    // [prefix[m], prefix[m+1]) whose bras are minor_order[minor_begin[m] + (t - prefix[m])].  All
    // quartets of a segment have the same K_ab and K_cd, so a warp's primitive loops run in lock
    // step.  With mixed precision a second (prefix, begin) pair covers the FP32 part of each range
    // (Q_bra Q_ket < thr32).  Segments are visited heaviest first (decreasing K_ab K_cd) and each task
    // sequence is cut into work-queue chunks (costChunks) that the kernels claim dynamically.
    // Whether a mixed-precision plan keeps every quartet of the class (la lb | lc ld) in FP64: when
    // its FP64 kernel is the DMMA group path, its ket has at least 15 spherical functions and its
    // total angular momentum is at least 8.  Measured per class on (H2O)_8 cc-pVTZ, the FP32
    // register or group kernels of those classes plus the FP64 launch of their large quartets took
    // longer than the DMMA kernel running all of their quartets ((fd|dp) 5.3 against 3.6 ms, (fp|dd)
    // 3.5 against 2.0 ms, (fd|fp) 2.5 against 1.4 ms).
    static bool fp32InFp64(int la, int lb, int lc, int ld)
    {
        const int sab = nsph(la) * nsph(lb), scd = nsph(lc) * nsph(ld);
        const int hab = nherm(la + lb), nr = nherm(la + lb + lc + ld);
        return pickRegGroup<double>(sab, scd, hab, nr) == 0 && scd >= 15 && la + lb + lc + ld >= 8;
    }

    Engine::JKClassPair Engine::buildClassPair(const ClassSet &bs, int cb, const ClassSet &ks, int ck, bool triangle,
                                               double thr, double thr32, bool mixed)
    {
        const ClassOrder &ob = bs.orders[cb], &ok = ks.orders[ck];
        // survivors of the predicate q_b * qj >= t in a group: a prefix of its Q values in decreasing
        // order (the kernels evaluate the same product)
        auto countGroup = [&](const ClassOrder::Group &g, double qj, double t) -> long long {
            if (t <= 0)
                return g.end - g.start;
            return std::partition_point(ob.qs.begin() + g.start, ob.qs.begin() + g.end,
                                        [&](double q) { return q * qj >= t; }) -
                   (ob.qs.begin() + g.start);
        };
        JKClassPair cp;
        cp.cb = cb;
        cp.ck = ck;
        cp.all64 = mixed && fp32InFp64(bs.host[cb].la, bs.host[cb].lb, ks.host[ck].la, ks.host[ck].lb);
        if (cp.all64)
            mixed = false;  // one FP64 task sequence over every surviving quartet
        std::vector<uint32_t> majors, b64, b32;
        std::vector<unsigned long long> p64(1, 0), p32(1, 0);
        auto &run64 = cp.run64, &run32 = cp.run32;  // tasks per major entry
        auto &cost = cp.cost;                       // primitive quartets (+ overhead) per task
        double bra_prims64 = 0, bra_prims32 = 0;
        const double lo64 = mixed ? thr32 : thr;
        // segments (bra group, ket group) of the same molecule, heaviest (largest K_b K_k) first
        std::vector<std::pair<uint32_t, uint32_t>> segs;
        for (uint32_t gb = 0; gb < (uint32_t)ob.groups.size(); gb++)
            for (uint32_t gc = 0; gc < (uint32_t)ok.groups.size(); gc++)
                if (!(triangle && gb < gc) && ob.groups[gb].mol == ok.groups[gc].mol)
                    segs.push_back({gb, gc});
        std::stable_sort(segs.begin(), segs.end(), [&](const auto &x, const auto &y) {
            return (double)ob.groups[x.first].k * ok.groups[x.second].k >
                   (double)ob.groups[y.first].k * ok.groups[y.second].k;
        });
        std::vector<int> fen;  // Fenwick tree over Q ranks (diagonal segments)
        for (const auto &sg : segs)
        {
            const size_t gb = sg.first, gc = sg.second;
            const auto &B = ob.groups[gb], &C = ok.groups[gc];
            const bool diag = triangle && gb == gc;
            const uint32_t nb = B.end - B.start;
            // diagonal segment: a ket at group offset r pairs with the bras at offsets >= r; the
            // survivors among them are counted with a Fenwick tree over the ranks of their Q values,
            // filled from the last offset down
            std::vector<uint32_t> rank;
            if (diag)
            {
                fen.assign(nb + 1, 0);
                std::vector<uint32_t> idx(nb);
                std::iota(idx.begin(), idx.end(), 0u);
                std::stable_sort(idx.begin(), idx.end(),
                                 [&](uint32_t x, uint32_t y) { return ob.q[B.start + x] > ob.q[B.start + y]; });
                rank.resize(nb);
                for (uint32_t r = 0; r < nb; r++)
                    rank[idx[r]] = r;
            }
            auto fenAdd = [&](uint32_t r) {
                for (uint32_t i = r + 1; i <= nb; i += i & (0u - i))
                    fen[i]++;
            };
            auto fenSum = [&](uint32_t r) {  // entries with rank < r
                long long v = 0;
                for (uint32_t i = r; i > 0; i -= i & (0u - i))
                    v += fen[i];
                return v;
            };
            auto countDiag = [&](double qj, double t) -> long long {
                if (t <= 0)
                    return fenSum(nb);
                const uint32_t r = (uint32_t)(std::partition_point(ob.qs.begin() + B.start, ob.qs.begin() + B.end,
                                                                   [&](double q) { return q * qj >= t; }) -
                                              (ob.qs.begin() + B.start));
                return fenSum(r);
            };
            struct Entry
            {
                uint32_t major, lo;
                long long c64, c32;
            };
            std::vector<Entry> entries;
            for (uint32_t jr = C.end; jr-- > C.start;)
            {
                const uint32_t j = jr;
                const double qj = ok.q[j];
                const uint32_t lo = diag ? j - C.start : 0u;
                if (diag)
                    fenAdd(rank[lo]);
                if (thr > 0 && B.qmax * qj < thr)
                    continue;
                const long long call = diag ? countDiag(qj, thr) : countGroup(B, qj, thr);
                if (call == 0)
                    continue;
                const long long c64 = mixed ? (diag ? countDiag(qj, lo64) : countGroup(B, qj, lo64)) : call;
                entries.push_back({j, lo, c64, call - c64});
            }
            // kets in increasing position (the diagonal walk above ran backwards)
            for (size_t e = entries.size(); e-- > 0;)
            {
                const Entry &en = entries[e];
                const uint32_t r = nb - en.lo;
                majors.push_back(ok.order[en.major]);
                b64.push_back(B.start + en.lo);
                b32.push_back(B.start + en.lo);
                const unsigned long long t64 = en.c64 > 0 ? r : 0, t32 = en.c32 > 0 ? r : 0;
                p64.push_back(p64.back() + t64);
                p32.push_back(p32.back() + t32);
                run64.push_back(t64);
                run32.push_back(t32);
                cost.push_back((double)C.k * B.k + 4.0);
                cp.n64 += en.c64;
                cp.n32 += en.c32;
                cp.prim64 += (double)en.c64 * B.k * C.k;
                cp.prim32 += (double)en.c32 * B.k * C.k;
                // bra-side work is counted per (bra primitive, ket pair)
                bra_prims64 += (double)en.c64 * B.k;
                bra_prims32 += (double)en.c32 * B.k;
            }
        }
        cp.t64 = (long long)p64.back();
        cp.t32 = (long long)p32.back();
        const auto &B = bs.host[cb], &K = ks.host[ck];
        cp.tb = pairType(B.la, B.lb);
        cp.tk = pairType(K.la, K.lb);
        const int L = B.la + B.lb + K.la + K.lb;
        const double hab = nherm(B.la + B.lb), hcd = nherm(K.la + K.lb);
        const double sab = nsph(B.la) * nsph(B.lb), scd = nsph(K.la) * nsph(K.lb);
        const double per_prim =
            (20 + 4 * L) + 3.0 * (L + 1) * (L + 2) * (L + 3) * (L + 4) / 24 + hab * hcd + 2 * hab * hcd * scd;
        const double per_bra = 2 * sab * hab * scd;
        cp.flops64 = cp.prim64 * per_prim + bra_prims64 * per_bra;
        cp.flops32 = cp.prim32 * per_prim + bra_prims32 * per_bra;
        cp.n_bra = (int)majors.size();
        if (cp.n64 + cp.n32 == 0)
            return cp;
        cp.majors = devUpload(majors, stream_);
        cp.prefix64 = devUpload(p64, stream_);
        cp.prefix32 = devUpload(p32, stream_);
        cp.begin64 = devUpload(b64, stream_);
        cp.begin32 = devUpload(b32, stream_);
        rebuildChunks(cp, false, cp.chunk_mult64);
        rebuildChunks(cp, true, cp.chunk_mult32);
        return cp;
    }

    // (Re)cuts the FP64 or FP32 task sequence of a class pair into work-queue chunks of at most
    // `mult` work units.
    void Engine::rebuildChunks(JKClassPair &cp, bool fp32, int mult)
    {
        const long long n = fp32 ? cp.t32 : cp.t64;
        unsigned long long *&dev = fp32 ? cp.chunks32 : cp.chunks64;
        cudaFree(dev);
        dev = nullptr;
        (fp32 ? cp.n_chunks32 : cp.n_chunks64) = 0;
        (fp32 ? cp.chunk_mult32 : cp.chunk_mult64) = mult;
        if (n == 0)
            return;
        // bra / ket classes of the launch: the bra set is the auxiliary one for swapped RI pairs
        const int tb = cp.tb, tk = cp.tk;
        const int unit = unitFwd(tb, tk, fp32, fp32 ? cp.shape32 : cp.shape64);
        if (unit == 0)
            return;
        auto ch = costChunks(fp32 ? cp.run32 : cp.run64, cp.cost, unit, mult * unit);
        (fp32 ? cp.n_chunks32 : cp.n_chunks64) = (long long)ch.size() - 1;
        dev = devUpload(ch, stream_);
    }

    // Unique quartets (ab|cd), class cd <= class ab, kept iff Q_ab Q_cd >= thr.
    Engine::JKPlan &Engine::jkPlan(double thr, double thr32, bool mixed)
    {
        ClassSet &cs = mainSet(true);
        ensureSchwarz(cs);
        char key[128];
        snprintf(key, sizeof(key), "%.6e/%.6e/%d", thr, thr32, mixed ? 1 : 0);
        auto it = plans_.find(key);
        if (it != plans_.end())
            return it->second;
        JKPlan plan;
        const size_t nc = cs.dev.size();
        for (size_t cb = 0; cb < nc; cb++)
            for (size_t ck = 0; ck <= cb; ck++)
            {
                JKClassPair cp = buildClassPair(cs, (int)cb, cs, (int)ck, cb == ck, thr, thr32, mixed);
                if (cp.n64 + cp.n32 == 0)
                    continue;
                plan.n_quartets += cp.n64 + cp.n32;
                plan.n_fp32 += cp.n32;
                plan.n_prim += cp.prim64 + cp.prim32;
                plan.flops64 += cp.flops64;
                plan.flops32 += cp.flops32;
                plan.pairs.push_back(cp);
            }
        // most expensive class pairs first
        std::stable_sort(plan.pairs.begin(), plan.pairs.end(), [](const JKClassPair &x, const JKClassPair &y) {
            return x.flops64 + x.flops32 > y.flops64 + y.flops32;
        });
        plan.counters = devAlloc<unsigned long long>(2 * std::max<size_t>(plan.pairs.size(), 1));
        plan.key = key;
        applyTuneCache(plan);
        assignBranches(plan);
        cudaCheck(cudaStreamSynchronize(stream_), "plan");
        plan.thr = thr;
        plan.thr32 = thr32;
        return plans_.emplace(key, std::move(plan)).first->second;
    }

    // Longest-processing-time assignment of the class pairs (already in decreasing cost) to the
    // stream branches of the fork/join launch sequence, so the tail of one class kernel overlaps
    // the next ones.
    void Engine::assignBranches(JKPlan &plan)
    {
        double load[kBranches] = {};
        for (auto &cp : plan.pairs)
        {
            int b = 0;
            for (int i = 1; i < kBranches; i++)
                if (load[i] < load[b])
                    b = i;
            cp.branch = b;
            load[b] += cp.flops64 + 0.5 * cp.flops32 + 1e6;
        }
    }

    // D_ab of every pair of the main classes, in Schwarz order, for the coalesced J_cd digestion.
    void Engine::gatherDab(const double *D)
    {
        for (const auto &d : mainSet(true).dev)
            if (d.Dab && d.n_pairs)
            {
                const long long tot = (long long)d.n_pairs * nsph(d.la) * nsph(d.lb);
                dabGatherKernel<<<(unsigned)std::min<long long>((tot + 255) / 256, num_sms_ * 8), 256, 0, stream_>>>(
                    D, d.soa2, (long long)d.n_pairs, nsph(d.la), nsph(d.lb), d.Dab);
            }
        cudaCheck(cudaGetLastError(), "dabGatherKernel");
    }

    // Event pairs around each class launch of a profiled build.
    struct Engine::LaunchTimer
    {
        std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
        std::vector<LaunchTime> info;
        void before(cudaStream_t s)
        {
            cudaEvent_t a, b;
            cudaCheck(cudaEventCreate(&a), "event");
            cudaCheck(cudaEventCreate(&b), "event");
            ev.push_back({a, b});
            cudaCheck(cudaEventRecord(a, s), "event");
        }
        void after(cudaStream_t s) { cudaCheck(cudaEventRecord(ev.back().second, s), "event"); }
        ~LaunchTimer()
        {
            for (auto &e : ev)
            {
                cudaEventDestroy(e.first);
                cudaEventDestroy(e.second);
            }
        }
    };

    // Shape 2 runs a J/K class pair in the other orientation: the kernel's bra is the plan's ket class
    // and its ket the plan's bra class, (cd|ab) for (ab|cd), which the final A + A^T of J and K makes
    // equivalent.  The plan's tasks stay as they are (major = ket pair, minor = bra pair) and are
    // decoded with major_ket = 0; the bra-side copies in Schwarz order and the per-position Q of the
    // minor list belong to the plan's bra class and are left unused.
    static void flipOrientation(QuartetArgs &a, const double *bra_etp)
    {
        std::swap(a.bra, a.ket);
        std::swap(a.bra_qpair, a.ket_qpair);
        a.major_ket = 0;
        a.bra_qpos = nullptr;
        a.bra_soa = nullptr;
        a.bra_pPs = nullptr;
        a.bra_Es = nullptr;
        a.bra_Efs = nullptr;
        a.bra_pPfs = nullptr;
        a.bra_soa2 = nullptr;
        a.bra_Dab = nullptr;
        a.bra_npos = 0;
        a.ket_EtP = bra_etp;
    }

    // Launches one J/K build of `plan` (memsets, class kernels over the stream branches, block
    // symmetrisation) on stream_; usable inside a stream capture.  With a timer every class launch
    // goes to stream_ itself, bracketed by events.
    void Engine::enqueueJK(JKPlan &plan, const double *D, double *J, double *K, bool mixed, LaunchTimer *timer)
    {
        ClassSet &cs = mainSet(true);
        const size_t n = (size_t)packed_;
        cudaCheck(cudaMemsetAsync(J, 0, n * sizeof(double), stream_), "memset");
        cudaCheck(cudaMemsetAsync(K, 0, n * sizeof(double), stream_), "memset");
        cudaCheck(cudaMemsetAsync(plan.counters, 0, 2 * plan.pairs.size() * sizeof(unsigned long long), stream_),
                  "memset");
        gatherDab(D);
        cudaCheck(cudaMemsetAsync(d_status_, 0, sizeof(int), stream_), "memset");
        cudaCheck(cudaEventRecord(fork_, stream_), "fork");
        bool used[kBranches] = {};
        if (!timer)
            for (const auto &cp : plan.pairs)
                used[cp.branch] = true;
        for (int b = 0; b < kBranches; b++)
            if (used[b])
                cudaCheck(cudaStreamWaitEvent(branch_[b], fork_, 0), "fork");
        for (size_t ip = 0; ip < plan.pairs.size(); ip++)
        {
            const auto &cp = plan.pairs[ip];
            const auto &B = cs.dev[cp.cb], &Kc = cs.dev[cp.ck];
            cudaStream_t st = timer ? stream_ : branch_[cp.branch];
            const auto &Bh = cs.host[cp.cb], &Kh = cs.host[cp.ck];
            QuartetArgs a{};
            a.bra = view(B);
            a.ket = view(Kc);
            a.boys = boys_;
            a.boys_f = boys_f_;
            a.list = nullptr;
            a.major_ket = 1;
            a.major_order = cp.majors;
            a.minor_order = cs.orders[cp.cb].d_order;
            a.n_major = cp.n_bra;
            a.same_class = cp.cb == cp.ck;
            a.mode = kJK;
            a.D = D;
            a.J = J;
            a.K = K;
            a.nao = (int)nao_;
            a.n_tasks = cp.t64;
            a.prefix = cp.prefix64;
            a.minor_begin = cp.begin64;
            a.chunks = cp.chunks64;
            a.n_chunks = cp.n_chunks64;
            a.counter = plan.counters + 2 * ip;
            a.grid_div = cp.grid_div64;
            a.bra_qpos = cs.orders[cp.cb].d_q;
            a.bra_qpair = B.Q;
            a.ket_qpair = Kc.Q;
            a.q_lo = (mixed && !cp.all64) ? plan.thr32 : plan.thr;
            a.q_hi = HUGE_VAL;
            a.bra_soa = B.soa;
            a.bra_pPs = B.pPs;
            a.bra_Es = B.Es;
            a.bra_Efs = B.Efs;
            a.bra_pPfs = B.pPfs;
            a.bra_soa2 = B.soa2;
            a.bra_Dab = B.Dab;
            a.bra_npos = (int)B.n_pairs;
            a.ket_EtP = Kc.EtP;
            a.status = d_status_;
            LaunchFn f64 = lookupFwd64(cp.tb, cp.tk, cp.shape64);
            if (!f64)
                throw EngineError(kStatusUnsupported, "quartet class not instantiated");
            if (timer && cp.t64 > 0)
            {
                timer->before(st);
                timer->info.push_back({{Bh.la, Bh.lb, Kh.la, Kh.lb}, 2 * cp.shape64, 0.0, cp.flops64, cp.n64});
            }
            {
                QuartetArgs a64 = a;
                if (cp.shape64 == 2)
                    flipOrientation(a64, B.EtP);
                cudaCheck(f64(a64, st, num_sms_), "jk kernel");
            }
            if (timer && cp.t64 > 0)
                timer->after(st);
            if (mixed && cp.t32 > 0)
            {
                a.q_lo = plan.thr;
                a.q_hi = plan.thr32;
                a.n_tasks = cp.t32;
                a.prefix = cp.prefix32;
                a.minor_begin = cp.begin32;
                a.chunks = cp.chunks32;
                a.n_chunks = cp.n_chunks32;
                a.counter = plan.counters + 2 * ip + 1;
                a.grid_div = cp.grid_div32;
                LaunchFn f32 = lookupFwd32(cp.tb, cp.tk, cp.shape32);
                if (!f32)
                    throw EngineError(kStatusUnsupported, "FP32 quartet class not instantiated");
                if (timer)
                {
                    timer->before(st);
                    timer->info.push_back({{Bh.la, Bh.lb, Kh.la, Kh.lb}, 1 + 2 * cp.shape32, 0.0, cp.flops32, cp.n32});
                }
                QuartetArgs a32 = a;
                if (cp.shape32 == 2)
                    flipOrientation(a32, B.EtP);
                cudaCheck(f32(a32, st, num_sms_), "jk kernel fp32");
                if (timer)
                    timer->after(st);
            }
        }
        for (int b = 0; b < kBranches; b++)
            if (used[b])
            {
                cudaCheck(cudaEventRecord(join_[b], branch_[b]), "join");
                cudaCheck(cudaStreamWaitEvent(stream_, join_[b], 0), "join");
            }
        const dim3 grid((unsigned)std::max(1, num_sms_ * 4 / (int)std::max<size_t>(mol_nao_.size(), 1)),
                        (unsigned)mol_nao_.size());
        symmetrizeBlocksKernel<<<grid, 256, 0, stream_>>>(J, d_blocks_);
        symmetrizeBlocksKernel<<<grid, 256, 0, stream_>>>(K, d_blocks_);
        cudaCheck(cudaGetLastError(), "symmetrize");
    }

    // Three-centre (mn|P) quartets of every main pair class with every auxiliary shell class, kept iff
    // Q_mn Q_P >= thr; the larger pair type is the bra (`swap` when that is the auxiliary class).
    Engine::JKPlan &Engine::riPlan(double thr)
    {
        ClassSet &ms = mainSet(true);
        ClassSet &xs = auxSet();
        ensureSchwarz(ms);
        ensureSchwarz(xs);
        char key[64];
        snprintf(key, sizeof(key), "%.6e", thr);
        auto it = ri_plans_.find(key);
        if (it != ri_plans_.end())
            return it->second;
        JKPlan plan;
        for (size_t cb = 0; cb < ms.dev.size(); cb++)
            for (size_t cx = 0; cx < xs.dev.size(); cx++)
            {
                const auto &B = ms.dev[cb], &X = xs.dev[cx];
                const bool swap = pairType(B.la, B.lb) < pairType(X.la, X.lb);
                JKClassPair cp = swap ? buildClassPair(xs, (int)cx, ms, (int)cb, false, thr, 0.0, false)
                                      : buildClassPair(ms, (int)cb, xs, (int)cx, false, thr, 0.0, false);
                cp.swap = swap;
                if (cp.n64 == 0)
                    continue;
                plan.n_quartets += cp.n64;
                plan.n_prim += cp.prim64;
                plan.flops64 += cp.flops64;
                plan.pairs.push_back(cp);
            }
        plan.counters = devAlloc<unsigned long long>(2 * std::max<size_t>(plan.pairs.size(), 1));
        cudaCheck(cudaStreamSynchronize(stream_), "plan");
        plan.thr = thr;
        return ri_plans_.emplace(key, std::move(plan)).first->second;
    }

    void Engine::jk(const double *D_dev, double *J_dev, double *K_dev, const JKOptions &opt, JKStats *stats)
    {
        const bool mixed = opt.precision == 1;
        JKPlan &plan = jkPlan(opt.schwarz, opt.fp32_threshold, mixed);
        if (opt.use_graph)
        {
            char key[256];
            snprintf(key, sizeof(key), "%s|%p|%p|%p", plan.key.c_str(), (const void *)D_dev, (void *)J_dev,
                     (void *)K_dev);
            if (!graph_exec_ || graph_key_ != key)
            {
                releaseGraph();
                cudaGraph_t g = nullptr;
                cudaCheck(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "capture");
                try
                {
                    enqueueJK(plan, D_dev, J_dev, K_dev, mixed);
                }
                catch (...)
                {
                    cudaStreamEndCapture(stream_, &g);
                    if (g)
                        cudaGraphDestroy(g);
                    throw;
                }
                cudaCheck(cudaStreamEndCapture(stream_, &g), "capture");
                cudaError_t e = cudaGraphInstantiate(&graph_exec_, g, 0);
                cudaGraphDestroy(g);
                cudaCheck(e, "cudaGraphInstantiate");
                graph_key_ = key;
            }
            cudaCheck(cudaGraphLaunch(graph_exec_, stream_), "cudaGraphLaunch");
        }
        else
            enqueueJK(plan, D_dev, J_dev, K_dev, mixed);
        if (stats)
        {
            stats->n_quartets = plan.n_quartets;
            stats->n_fp32 = plan.n_fp32;
            stats->n_launches = 2;
            for (const auto &cp : plan.pairs)
                stats->n_launches += 1 + (cp.t32 > 0 ? 1 : 0);
        }
    }

    // ------------------------------------------------------------------------------------------
    // Autotuning of the class-pair launches.  The tunable "tile" of a persistent class kernel is
    // its occupancy (resident blocks per SM divided by grid_div) and the granularity of its work
    // queue (chunks of at most chunk_mult work units); every candidate is timed on the caller's
    // buffers with CUDA events and the fastest is kept.  Results are keyed by GPU name, quartet
    // class and the size bucket floor(log2(tasks)), and appended to a plain-text cache:
    //     <gpu>|<la> <lb> <lc> <ld>|<fp32>|<bucket>|<grid_div> <chunk_mult>

    static int sizeBucket(long long n)
    {
        int b = 0;
        while ((1LL << (b + 1)) <= n)
            b++;
        return b;
    }

    void Engine::applyTuneCache(JKPlan &plan)
    {
        if (tune_cache_.empty())
            return;
        FILE *f = fopen(tune_cache_.c_str(), "r");
        if (!f)
            return;
        struct Choice
        {
            int gd, cm, shape;
        };
        std::map<std::string, Choice> entries;
        char line[512];
        while (fgets(line, sizeof(line), f))
        {
            std::string l(line);
            const size_t bar = l.rfind('|');
            if (bar == std::string::npos)
                continue;
            int gd = 0, cm = 0, shape = 0;  // lines without the shape field are the default shape
            const int got = sscanf(l.c_str() + bar + 1, "%d %d %d", &gd, &cm, &shape);
            if (got >= 2 && gd > 0 && cm > 0 && shape >= 0 && shape <= 2)
                entries[l.substr(0, bar)] = {gd, cm, got == 3 ? shape : 0};
        }
        fclose(f);
        ClassSet &cs = mainSet(true);
        for (auto &cp : plan.pairs)
            for (int fp32 = 0; fp32 < 2; fp32++)
            {
                const long long n = fp32 ? cp.t32 : cp.t64;
                if (n == 0)
                    continue;
                const auto &B = cs.host[cp.cb], &K = cs.host[cp.ck];
                char key[256];
                snprintf(key, sizeof(key), "%s|%d %d %d %d|%d|%d", gpu_name_.c_str(), B.la, B.lb, K.la, K.lb, fp32,
                         sizeBucket(n));
                auto it = entries.find(key);
                if (it == entries.end())
                    continue;
                const Choice &ch = it->second;
                const int shape = (ch.shape >= 1 && hasFwdVariant(cp.tb, cp.tk, fp32 == 1, ch.shape)) ? ch.shape : 0;
                (fp32 ? cp.grid_div32 : cp.grid_div64) = ch.gd;
                (fp32 ? cp.shape32 : cp.shape64) = shape;
                rebuildChunks(cp, fp32 == 1, ch.cm);
                plan.tuned = true;
            }
    }

    std::string Engine::jkAutotune(const double *D, double *J, double *K, const JKOptions &opt,
                                   const std::string &cache)
    {
        const bool mixed = opt.precision == 1;
        if (!cache.empty())
            tune_cache_ = cache;
        JKPlan &plan = jkPlan(opt.schwarz, opt.fp32_threshold, mixed);
        releaseGraph();
        ClassSet &cs = mainSet(true);
        cudaEvent_t e0, e1;
        cudaCheck(cudaEventCreate(&e0), "event");
        cudaCheck(cudaEventCreate(&e1), "event");
        std::string summary;
        gatherDab(D);
        FILE *out = cache.empty() ? nullptr : fopen(cache.c_str(), "a");
        const int grid_divs[] = {1, 2};
        const int mults[] = {2, 8, 32};
        for (size_t ip = 0; ip < plan.pairs.size(); ip++)
        {
            JKClassPair &cp = plan.pairs[ip];
            const auto &B = cs.dev[cp.cb], &Kc = cs.dev[cp.ck];
            for (int fp32 = 0; fp32 < (mixed ? 2 : 1); fp32++)
            {
                const long long n = fp32 ? cp.t32 : cp.t64;
                if (n == 0)
                    continue;
                // shapes: the default, the alternative tile shape, the other orientation
                int shapes[3] = {0, 0, 0}, n_shapes = 1;
                for (int s2 = 1; s2 <= 2; s2++)
                    if (hasFwdVariant(cp.tb, cp.tk, fp32 == 1, s2))
                        shapes[n_shapes++] = s2;
                float best = 1e30f;
                int best_gd = 1, best_cm = 8, best_shape = 0;
                for (int si = 0; si < n_shapes; si++)
                for (int cm : mults)
                {
                    const int shape = shapes[si];
                    LaunchFn fn = fp32 ? lookupFwd32(cp.tb, cp.tk, shape) : lookupFwd64(cp.tb, cp.tk, shape);
                    if (!fn)
                        throw EngineError(kStatusUnsupported, "quartet class not instantiated");
                    (fp32 ? cp.shape32 : cp.shape64) = shape;
                    rebuildChunks(cp, fp32 == 1, cm);  // the work unit depends on the shape
                    for (int gd : grid_divs)
                    {
                        QuartetArgs a{};
                        a.bra = view(B);
                        a.ket = view(Kc);
                        a.boys = boys_;
                        a.boys_f = boys_f_;
                        a.major_ket = 1;
                        a.major_order = cp.majors;
                        a.minor_order = cs.orders[cp.cb].d_order;
                        a.n_major = cp.n_bra;
                        a.same_class = cp.cb == cp.ck;
                        a.mode = kJK;
                        a.D = D;
                        a.J = J;
                        a.K = K;
                        a.nao = (int)nao_;
                        a.n_tasks = n;
                        a.prefix = fp32 ? cp.prefix32 : cp.prefix64;
                        a.minor_begin = fp32 ? cp.begin32 : cp.begin64;
                        a.chunks = fp32 ? cp.chunks32 : cp.chunks64;
                        a.n_chunks = fp32 ? cp.n_chunks32 : cp.n_chunks64;
                        a.counter = plan.counters + 2 * ip + fp32;
                        a.grid_div = gd;
                        a.bra_qpos = cs.orders[cp.cb].d_q;
                        a.bra_qpair = B.Q;
                        a.ket_qpair = Kc.Q;
                        a.q_lo = fp32 ? plan.thr : ((mixed && !cp.all64) ? plan.thr32 : plan.thr);
                        a.q_hi = fp32 ? plan.thr32 : HUGE_VAL;
                        a.bra_soa = B.soa;
                        a.bra_pPs = B.pPs;
                        a.bra_Es = B.Es;
                        a.bra_Efs = B.Efs;
                        a.bra_pPfs = B.pPfs;
                        a.bra_soa2 = B.soa2;
                        a.bra_Dab = B.Dab;
                        a.bra_npos = (int)B.n_pairs;
                        a.ket_EtP = Kc.EtP;
                        a.status = d_status_;
                        if (shape == 2)
                            flipOrientation(a, B.EtP);
                        // a second timing only for short launches, where one sample is noisy
                        float t_min = 1e30f;
                        for (int rep = 0; rep < 2 && (rep == 0 || t_min < 2.0f); rep++)
                        {
                            cudaCheck(cudaMemsetAsync(a.counter, 0, sizeof(unsigned long long), stream_), "memset");
                            cudaCheck(cudaEventRecord(e0, stream_), "event");
                            cudaCheck(fn(a, stream_, num_sms_), "autotune kernel");
                            cudaCheck(cudaEventRecord(e1, stream_), "event");
                            cudaCheck(cudaEventSynchronize(e1), "event");
                            float ms = 0;
                            cudaCheck(cudaEventElapsedTime(&ms, e0, e1), "event");
                            t_min = std::min(t_min, ms);
                        }
                        if (t_min < best)
                        {
                            best = t_min;
                            best_gd = gd;
                            best_cm = cm;
                            best_shape = shape;
                        }
                    }
                }
                (fp32 ? cp.shape32 : cp.shape64) = best_shape;
                rebuildChunks(cp, fp32 == 1, best_cm);
                (fp32 ? cp.grid_div32 : cp.grid_div64) = best_gd;
                const auto &Bh = cs.host[cp.cb], &Kh = cs.host[cp.ck];
                char line[320];
                snprintf(line, sizeof(line), "%s|%d %d %d %d|%d|%d|%d %d %d\n", gpu_name_.c_str(), Bh.la, Bh.lb, Kh.la,
                         Kh.lb, fp32, sizeBucket(n), best_gd, best_cm, best_shape);
                if (out)
                    fputs(line, out);
                char info[200];
                snprintf(info, sizeof(info), "(%d%d|%d%d) %s tasks=%lld shape=%d grid_div=%d chunk_mult=%d %.3f ms\n",
                         Bh.la, Bh.lb, Kh.la, Kh.lb, fp32 ? "fp32" : "fp64", n, best_shape, best_gd, best_cm, best);
                summary += info;
            }
        }
        if (out)
            fclose(out);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaCheck(cudaStreamSynchronize(stream_), "autotune");
        plan.tuned = true;
        return summary;
    }

    std::vector<Engine::LaunchTime> Engine::jkProfile(const double *D, double *J, double *K, const JKOptions &opt)
    {
        const bool mixed = opt.precision == 1;
        JKPlan &plan = jkPlan(opt.schwarz, opt.fp32_threshold, mixed);
        LaunchTimer timer;
        enqueueJK(plan, D, J, K, mixed, &timer);
        cudaCheck(cudaStreamSynchronize(stream_), "profile");
        for (size_t i = 0; i < timer.ev.size(); i++)
        {
            float ms = 0;
            cudaCheck(cudaEventElapsedTime(&ms, timer.ev[i].first, timer.ev[i].second), "event");
            timer.info[i].ms = ms;
        }
        return timer.info;
    }

    long long Engine::jkLaunchCount(const JKOptions &opt)
    {
        JKPlan &plan = jkPlan(opt.schwarz, opt.fp32_threshold, opt.precision == 1);
        long long c = 2;
        for (const auto &cp : plan.pairs)
            c += 1 + (cp.t32 > 0 ? 1 : 0);
        return c;
    }

    JKPlanInfo Engine::jkPlanInfo(const JKOptions &opt)
    {
        JKPlan &plan = jkPlan(opt.schwarz, opt.fp32_threshold, opt.precision == 1);
        JKPlanInfo info;
        info.n_quartets = plan.n_quartets;
        info.n_fp32 = plan.n_fp32;
        info.n_prim_quartets = (long long)plan.n_prim;
        info.flops_fp64 = plan.flops64;
        info.flops_fp32 = plan.flops32;
        info.n_launches = jkLaunchCount(opt);
        return info;
    }

    std::vector<Engine::JKClassInfo> Engine::jkPlanClasses(const JKOptions &opt)
    {
        JKPlan &plan = jkPlan(opt.schwarz, opt.fp32_threshold, opt.precision == 1);
        ClassSet &cs = mainSet(true);
        std::vector<JKClassInfo> v;
        for (const auto &cp : plan.pairs)
        {
            const auto &B = cs.dev[cp.cb], &K = cs.dev[cp.ck];
            v.push_back({{B.la, B.lb, K.la, K.lb}, cp.n64, cp.n32, cp.prim64 + cp.prim32, cp.flops64 + cp.flops32});
        }
        return v;
    }

    // ------------------------------------------------------------------------------------------
    // J/K energy gradient (adjoint of the J/K build): dE/dR over all unique quartets.

    // The quartets are those of the FP64 J/K plan with the same Schwarz threshold, so the gradient
    // is the exact derivative of the energy lible_gpu_jk_energy_forward computes with that threshold.
    void Engine::jkGradient(const double *D_dev, double *grad_dev, double schwarz)
    {
        requireSingle();
        ClassSet &cs = mainSet(true);
        JKPlan &plan = jkPlan(schwarz, 0.0, false);
        const size_t n = nao_;
        cudaCheck(cudaMemsetAsync(grad_dev, 0, 3 * n_atoms_ * sizeof(double), stream_), "memset");
        cudaCheck(cudaMemsetAsync(plan.counters, 0, 2 * plan.pairs.size() * sizeof(unsigned long long), stream_),
                  "memset");
        for (size_t ip = 0; ip < plan.pairs.size(); ip++)
        {
            auto &cp = plan.pairs[ip];
            const auto &B = cs.dev[cp.cb], &K = cs.dev[cp.ck];
            if (!cp.chunksD1 && cp.t64 > 0)
            {
                // one quartet per block at a time: chunks of the heaviest quartet up to 8 tasks; the
                // register classes take 32 quartets per warp step
                const int gt = d1RegisterGroup(B.la, B.lb, K.la, K.lb);
                const int unit = gt ? 32 / gt : 1;
                auto ch = costChunks(cp.run64, cp.cost, unit, 8 * unit);
                cp.n_chunksD1 = (long long)ch.size() - 1;
                cp.chunksD1 = devUpload(ch, stream_);
            }
            QuartetArgs a{};
            a.bra = view(B);
            a.ket = view(K);
            a.boys = boys_;
            a.boys_f = boys_f_;
            a.list = nullptr;
            a.major_ket = 1;
            a.major_order = cp.majors;
            a.minor_order = cs.orders[cp.cb].d_order;
            a.minor_begin = cp.begin64;
            a.prefix = cp.prefix64;
            a.n_major = cp.n_bra;
            a.n_tasks = cp.t64;
            a.bra_qpair = B.Q;
            a.ket_qpair = K.Q;
            a.q_lo = plan.thr;
            a.q_hi = HUGE_VAL;
            a.same_class = cp.cb == cp.ck;
            a.mode = kD1Grad;
            a.D = D_dev;
            a.nao = (int)n;
            a.grad = grad_dev;
            a.n_atoms = n_atoms_;
            a.chunks = cp.chunksD1;
            a.n_chunks = cp.n_chunksD1;
            a.counter = plan.counters + 2 * ip;
            cudaCheck(lookupD1(pairType(B.la, B.lb), pairType(K.la, K.lb))(a, stream_, num_sms_), "grad kernel");
        }
        cudaCheck(cudaStreamSynchronize(stream_), "grad");
    }

    // ------------------------------------------------------------------------------------------
    // RI-J pieces: gamma_P = sum_mn (mn|P) D_mn and J_mn = sum_P (mn|P) d_P.

    // Launch arguments of RI plan entry `ip` (epilogue fields left to the caller).
    QuartetArgs Engine::riArgs(const JKPlan &plan, size_t ip)
    {
        ClassSet &ms = mainSet(true);
        ClassSet &xs = auxSet();
        const auto &cp = plan.pairs[ip];
        // cp.cb / cp.ck index the bra / ket sets: (aux, main) when cp.swap, else (main, aux)
        const ClassSet &bs = cp.swap ? xs : ms;
        const auto &B = bs.dev[cp.cb];
        const auto &K = (cp.swap ? ms : xs).dev[cp.ck];
        QuartetArgs a{};
        a.bra = view(B);
        a.ket = view(K);
        a.boys = boys_;
        a.boys_f = boys_f_;
        a.list = nullptr;
        a.major_ket = 1;
        a.major_order = cp.majors;
        a.minor_order = bs.orders[cp.cb].d_order;
        a.minor_begin = cp.begin64;
        a.prefix = cp.prefix64;
        a.n_major = cp.n_bra;
        a.n_tasks = cp.t64;
        a.bra_qpos = bs.orders[cp.cb].d_q;
        a.bra_qpair = B.Q;
        a.ket_qpair = K.Q;
        a.ket_EtP = K.EtP;
        a.status = d_status_;
        a.q_lo = plan.thr;
        a.q_hi = HUGE_VAL;
        a.aux_side = cp.swap ? 1 : 0;
        a.nao = (int)nao_;
        a.bra_soa = B.soa;
        a.bra_pPs = B.pPs;
        a.bra_Es = B.Es;
        a.bra_Efs = B.Efs;
        a.bra_pPfs = B.pPfs;
        a.chunks = cp.chunks64;
        a.n_chunks = cp.n_chunks64;
        return a;
    }

    LaunchFn Engine::riLaunchFn(const JKPlan &plan, size_t ip)
    {
        const auto &cp = plan.pairs[ip];
        const auto &B = (cp.swap ? auxSet() : mainSet(true)).dev[cp.cb];
        const auto &K = (cp.swap ? mainSet(true) : auxSet()).dev[cp.ck];
        return lookupFwd64(pairType(B.la, B.lb), pairType(K.la, K.lb));
    }

    void Engine::riContract(const double *D_dev, const double *dcoef_dev, double *gamma_dev, double *J_dev,
                            double schwarz)
    {
        requireSingle();
        JKPlan &plan = riPlan(schwarz);
        const size_t n = nao_;
        if (gamma_dev)
            cudaCheck(cudaMemsetAsync(gamma_dev, 0, naux_ * sizeof(double), stream_), "memset");
        if (J_dev)
            cudaCheck(cudaMemsetAsync(J_dev, 0, n * n * sizeof(double), stream_), "memset");
        cudaCheck(cudaMemsetAsync(d_status_, 0, sizeof(int), stream_), "memset");
        cudaCheck(cudaMemsetAsync(plan.counters, 0, 2 * plan.pairs.size() * sizeof(unsigned long long), stream_),
                  "memset");
        for (size_t ip = 0; ip < plan.pairs.size(); ip++)
        {
            QuartetArgs a = riArgs(plan, ip);
            a.D = D_dev;
            a.dcoef = dcoef_dev;
            a.gamma = gamma_dev;
            a.J = J_dev;
            const LaunchFn fn = riLaunchFn(plan, ip);
            if (gamma_dev)
            {
                a.counter = plan.counters + 2 * ip;
                a.mode = kRIGamma;
                cudaCheck(fn(a, stream_, num_sms_), "ri gamma");
            }
            if (J_dev)
            {
                a.counter = plan.counters + 2 * ip + 1;
                a.mode = kRIJ;
                cudaCheck(fn(a, stream_, num_sms_), "ri J");
            }
        }
        if (J_dev)
        {
            symmetrizeKernel<<<num_sms_ * 4, 256, 0, stream_>>>(J_dev, (long long)n);
            cudaCheck(cudaGetLastError(), "symmetrize");
        }
        cudaCheck(cudaStreamSynchronize(stream_), "ri");
        checkStatus();
    }

    // Unique auxiliary shell pairs (P|Q) with the RI plan's Schwarz test, for the two-centre part of
    // the RI-J gradient.
    Engine::JKPlan &Engine::ri2Plan(double thr)
    {
        ClassSet &xs = auxSet();
        ensureSchwarz(xs);
        char key[64];
        snprintf(key, sizeof(key), "2c %.6e", thr);
        auto it = ri_plans_.find(key);
        if (it != ri_plans_.end())
            return it->second;
        JKPlan plan;
        for (size_t ca = 0; ca < xs.dev.size(); ca++)
            for (size_t cb = 0; cb <= ca; cb++)
            {
                // the larger pair type in the bra, as the class kernels are instantiated
                const bool swap = pairType(xs.dev[ca].la, 0) < pairType(xs.dev[cb].la, 0);
                const int b = swap ? (int)cb : (int)ca, k = swap ? (int)ca : (int)cb;
                JKClassPair cp = buildClassPair(xs, b, xs, k, ca == cb, thr, 0.0, false);
                if (cp.n64 == 0)
                    continue;
                plan.n_quartets += cp.n64;
                plan.pairs.push_back(cp);
            }
        plan.counters = devAlloc<unsigned long long>(2 * std::max<size_t>(plan.pairs.size(), 1));
        cudaCheck(cudaStreamSynchronize(stream_), "plan");
        plan.thr = thr;
        return ri_plans_.emplace(key, std::move(plan)).first->second;
    }

    void Engine::riGradient(const double *D_dev, const double *dcoef_dev, double *grad_dev, double schwarz)
    {
        requireSingle();
        ClassSet &ms = mainSet(true);
        ClassSet &xs = auxSet();
        JKPlan &p3 = riPlan(schwarz);
        JKPlan &p2 = ri2Plan(schwarz);
        cudaCheck(cudaMemsetAsync(grad_dev, 0, 3 * n_atoms_ * sizeof(double), stream_), "memset");
        cudaCheck(cudaMemsetAsync(d_status_, 0, sizeof(int), stream_), "memset");
        for (JKPlan *plan : {&p3, &p2})
        {
            const bool two = plan == &p2;
            cudaCheck(cudaMemsetAsync(plan->counters, 0, 2 * plan->pairs.size() * sizeof(unsigned long long), stream_),
                      "memset");
            for (size_t ip = 0; ip < plan->pairs.size(); ip++)
            {
                auto &cp = plan->pairs[ip];
                const ClassSet &bs = two ? xs : (cp.swap ? xs : ms);
                const ClassSet &ks = two ? xs : (cp.swap ? ms : xs);
                const auto &B = bs.dev[cp.cb], &K = ks.dev[cp.ck];
                if (!cp.chunksD1 && cp.t64 > 0)
                {
                    const int gt = d1RegisterGroup(B.la, B.lb, K.la, K.lb);
                    const int unit = gt ? 32 / gt : 1;
                    auto ch = costChunks(cp.run64, cp.cost, unit, 8 * unit);
                    cp.n_chunksD1 = (long long)ch.size() - 1;
                    cp.chunksD1 = devUpload(ch, stream_);
                }
                QuartetArgs a{};
                a.bra = view(B);
                a.ket = view(K);
                a.boys = boys_;
                a.boys_f = boys_f_;
                a.list = nullptr;
                a.major_ket = 1;
                a.major_order = cp.majors;
                a.minor_order = bs.orders[cp.cb].d_order;
                a.minor_begin = cp.begin64;
                a.prefix = cp.prefix64;
                a.n_major = cp.n_bra;
                a.n_tasks = cp.t64;
                a.bra_qpair = B.Q;
                a.ket_qpair = K.Q;
                a.q_lo = plan->thr;
                a.q_hi = HUGE_VAL;
                a.same_class = two && cp.cb == cp.ck;
                a.aux_side = two ? 2 : (cp.swap ? 1 : 0);
                a.mode = kD1GradRI;
                a.D = D_dev;
                a.dcoef = dcoef_dev;
                a.nao = (int)nao_;
                a.grad = grad_dev;
                a.n_atoms = n_atoms_;
                a.status = d_status_;
                a.chunks = cp.chunksD1;
                a.n_chunks = cp.n_chunksD1;
                a.counter = plan->counters + 2 * ip;
                cudaCheck(lookupD1(pairType(B.la, B.lb), pairType(K.la, K.lb))(a, stream_, num_sms_), "ri grad");
            }
        }
        cudaCheck(cudaStreamSynchronize(stream_), "ri grad");
        checkStatus();
    }

    std::vector<int> Engine::auxShellStarts()
    {
        requireStructure();
        if (!has_aux_)
            throw EngineError(kStatusNoAux, "RI approximation is not enabled");
        std::vector<int> v;
        for (const Shell &sh : aux_shells_)
            v.push_back((int)sh.ofs_sph);
        v.push_back((int)naux_);
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
        return v;
    }

    void Engine::riStore(int P_lo, int P_hi, double *T_dev, double schwarz, bool packed)
    {
        requireSingle();
        JKPlan &plan = riPlan(schwarz);
        const size_t n = nao_, row = packed ? n * (n + 1) / 2 : n * n;
        cudaCheck(cudaMemsetAsync(T_dev, 0, (size_t)(P_hi - P_lo) * row * sizeof(double), stream_), "memset");
        cudaCheck(cudaMemsetAsync(plan.counters, 0, 2 * plan.pairs.size() * sizeof(unsigned long long), stream_),
                  "memset");
        for (size_t ip = 0; ip < plan.pairs.size(); ip++)
        {
            QuartetArgs a = riArgs(plan, ip);
            a.out = T_dev;
            a.ri_lo = P_lo;
            a.ri_hi = P_hi;
            a.flags = packed ? kRIPacked : 0;
            a.counter = plan.counters + 2 * ip;
            a.mode = kRIStore;
            cudaCheck(riLaunchFn(plan, ip)(a, stream_, num_sms_), "ri store");
        }
    }

    // Reads the device status word of the last calls (bounded waits that gave up set it).
    void Engine::checkStatus()
    {
        int st = 0;
        cudaCheck(cudaMemcpyAsync(&st, d_status_, sizeof(int), cudaMemcpyDeviceToHost, stream_), "status");
        cudaCheck(cudaStreamSynchronize(stream_), "status");
        if (st != 0)
        {
            cudaCheck(cudaMemsetAsync(d_status_, 0, sizeof(int), stream_), "memset");
            cudaCheck(cudaStreamSynchronize(stream_), "status");
            throw EngineError(kStatusTimeout, "a bounded device wait gave up (bulk copy did not complete)");
        }
    }

    // One thread waits on a freshly initialised shared-memory barrier that expects one arrival
    // and gets none: the wait runs out after `polls` polls and records the timeout status, exactly
    // as a stalled bulk copy would.  Nothing is in flight when the block exits.
    __global__ void boundedWaitKernel(int *status, int polls)
    {
        __shared__ __align__(8) uint64_t mbar;
        if (threadIdx.x == 0)
        {
            mbarInit(&mbar);
            mbarWait(&mbar, 0, status, polls);
        }
    }

    void Engine::injectWaitTimeout(int polls)
    {
        if (polls < 0 || polls > kWaitPolls)
            throw EngineError(kStatusInvalid, "polls must be in [0, 2^20]");
        wait_inject_ = polls;
    }

    void Engine::checkBoundedWait(int polls)
    {
        if (polls < 1 || polls > (1 << 20))
            throw EngineError(kStatusInvalid, "polls must be in [1, 2^20]");
        cudaCheck(cudaMemsetAsync(d_status_, 0, sizeof(int), stream_), "memset");
        boundedWaitKernel<<<1, 32, 0, stream_>>>(d_status_, polls);
        cudaCheck(cudaGetLastError(), "boundedWaitKernel");
        checkStatus();
    }

    double *Engine::staging(int slot, size_t n)
    {
        if (slot < 0 || slot >= 4)
            throw EngineError(kStatusInternal, "bad staging slot");
        if (staging_n_[slot] < n)
        {
            releaseGraph();  // a captured graph may refer to the old buffer
            cudaCheck(cudaStreamSynchronize(stream_), "staging");
            cudaFree(staging_[slot]);
            staging_[slot] = nullptr;
            staging_n_[slot] = 0;
            cudaCheck(cudaMalloc(&staging_[slot], n * sizeof(double)), "cudaMalloc");
            staging_n_[slot] = n;
        }
        return staging_[slot];
    }

    void Engine::sync()
    {
        cudaCheck(cudaStreamSynchronize(stream_), "sync");
    }
}
