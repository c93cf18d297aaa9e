// RI metric factorisation (shared by RI-J and RI-K), the cached three-centre tensor of RI-J and the
// RI exchange build
//     K_mn = sum_{PQ} (m l|P) [(P|Q)^{-1}]_{PQ} (Q|n s) D_ls,   D = C C^T.
// The reference exposes the three- and two-centre kernels this builds on (ERI3Kernel / eri2,
// src/lible/ints/twoel/eri_kernels.cpp:1122-1162) but no RI exchange driver.
//
// Pipeline, all on the device:
//   1. (P|Q) -> Cholesky factor L (or G = V w^{-1/2} from an eigendecomposition, see MetricFactor);
//   2. per block of auxiliary functions: T[P][m][n] = (mn|P) by the class kernels (kRIStore), then
//      Z[P][m][i] = sum_n T[P][m][n] C[n][i] as one DGEMM over the whole block;
//   3. W = L^{-1} Z along P: one DTRSM with nao*occ right-hand sides (or W = Z G);
//   4. K = sum_R W_R W_R^T: W is re-laid out as A[m][R][i] block by block and each block is one
//      symmetric rank-k product with k = R_block * occ (syrkUpper, this file's split-K FP64 DMMA
//      kernel; cuBLAS DSYRK when k is odd).
// The three-centre tensor is never held in full: only Z (naux x nao x occ) and one block of T.
// When the fitted tensor B = L^{-1} (mn|P) fits in device memory it is instead built once per
// structure (buildFitted) and every call is one strided-batched DGEMM and one syrkUpper
// (riExchangeFitted): no integrals and no triangular solve per call.
// RI-J keeps the packed lower triangle of (mn|P) instead (buildT3, t3Gamma, t3Coulomb).
#include "ri_solve.hpp"

#include <cmath>
#include <string>
#include <vector>

namespace lible_b200
{
    void blasCheck(cublasStatus_t s, const char *what)
    {
        if (s != CUBLAS_STATUS_SUCCESS)
            throw EngineError(kStatusCuda, std::string("cuBLAS ") + what + " failed (status " + std::to_string((int)s) +
                                               ")");
    }

    namespace
    {
        // A[(m * rb + r) * occ + i] = W[((r0 + r) * n + m) * occ + i] for r < rb.
        __global__ void relayoutKernel(const double *__restrict__ W, long long n, long long occ, long long r0,
                                       long long rb, double *__restrict__ A)
        {
            const long long total = n * rb * occ;
            for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
                 g += (long long)gridDim.x * blockDim.x)
            {
                const long long i = g % occ, mr = g / occ;
                const long long r = mr % rb, m = mr / rb;
                A[g] = W[((r0 + r) * n + m) * occ + i];
            }
        }

        __global__ void mirrorUpperKernel(double *K, long long n)
        {
            for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < n * n;
                 g += (long long)gridDim.x * blockDim.x)
            {
                const long long r = g / n, c = g % n;
                if (r > c)
                    K[r * n + c] = K[c * n + r];
            }
        }

        // C[m * k + j] = U[m + idx[j] * n] * scale[j]  (U column-major n x n, C row-major n x k).
        __global__ void factorColumnsKernel(const double *__restrict__ U, long long n, const int *__restrict__ idx,
                                            const double *__restrict__ scale, long long k, double *__restrict__ C)
        {
            for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < n * k;
                 g += (long long)gridDim.x * blockDim.x)
            {
                const long long m = g / k, j = g % k;
                C[g] = U[m + (long long)idx[j] * n] * scale[j];
            }
        }

        struct EventPair
        {
            cudaEvent_t a = nullptr, b = nullptr;
            EventPair()
            {
                cudaCheck(cudaEventCreate(&a), "event");
                cudaCheck(cudaEventCreate(&b), "event");
            }
            ~EventPair()
            {
                cudaEventDestroy(a);
                cudaEventDestroy(b);
            }
            double seconds() const
            {
                float ms = 0;
                cudaCheck(cudaEventElapsedTime(&ms, a, b), "event");
                return 1e-3 * ms;
            }
        };

        int gridFor(long long total)
        {
            return (int)std::max<long long>(1, std::min<long long>((total + 255) / 256, 148LL * 16));
        }

        // ---- symmetric rank-k update on the DMMA pipe -------------------------------------------
        // K[r][c] += sign * sum_j Z[r][j] Z[c][j] for c >= r (the row-major upper triangle; callers
        // mirror it), Z row-major n x k with an even row pitch ldz, so every row starts on 16 bytes.
        // A block owns one 128 x 128 output tile on or above the diagonal and one slice of k; its 16
        // warps own 32 x 32 sub-tiles as 4 x 4 mma.m8n8k4.f64 tiles.  The two 128-row operand panels
        // stream through a 4-stage cp.async pipeline in 16-column steps (row pitch 20 doubles, so the
        // fragment reads of a warp spread over all banks), and each partial sum reaches K by one FP64
        // atomic per element and slice.  Algorithmic FLOPs: n (n + 1) k.
        constexpr int kSyrkBM = 128, kSyrkKB = 16, kSyrkP = 20, kSyrkStages = 4, kSyrkThreads = 512;
        constexpr int kSyrkStageDoubles = 2 * kSyrkBM * kSyrkP;
        constexpr size_t kSyrkSmem = (size_t)kSyrkStages * kSyrkStageDoubles * sizeof(double);

        __device__ __forceinline__ void cpAsync16(double *dst, const double *src, int bytes)
        {
            const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(bytes) : "memory");
        }
        __device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
        template <int N>
        __device__ __forceinline__ void cpAsyncWait()
        {
            asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
        }
        __device__ __forceinline__ void dmmaF64(double &d0, double &d1, double a, double b)
        {
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                         : "+d"(d0), "+d"(d1)
                         : "d"(a), "d"(b));
        }

        __global__ void __launch_bounds__(kSyrkThreads, 1)
            syrkUpperKernel(const double *__restrict__ Z, long long n, long long k, long long ldz, long long kslice,
                            int tiles_per_side, double sign, double *__restrict__ K)
        {
            extern __shared__ __align__(16) double sm[];
            // tile (bi, bj), bj >= bi, numbered row by row
            int t = (int)blockIdx.x, bi = 0;
            while (t >= tiles_per_side - bi)
            {
                t -= tiles_per_side - bi;
                bi++;
            }
            const int bj = bi + t;
            const long long r0 = (long long)bi * kSyrkBM, c0 = (long long)bj * kSyrkBM;
            const long long kb = (long long)blockIdx.y * kslice;
            const long long ke = kb + kslice < k ? kb + kslice : k;
            if (kb >= ke)
                return;
            const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, r8 = lane >> 2, k4 = lane & 3;
            const int wm = warp >> 2, wn = warp & 3;
            const long long nsteps = (ke - kb + kSyrkKB - 1) / kSyrkKB;

            // one step: 2 panels x 128 rows x 16 doubles = 2048 chunks of 16 bytes, 4 per thread;
            // rows past n and columns past the slice are zero-filled
            auto load = [&](long long step, int buf) {
                double *base = sm + (size_t)buf * kSyrkStageDoubles;
                const long long k0 = kb + step * kSyrkKB;
#pragma unroll
                for (int i = 0; i < 4; i++)
                {
                    const int ch = tid + i * kSyrkThreads;
                    const int which = ch >> 10, row = (ch >> 3) & (kSyrkBM - 1), col = (ch & 7) * 2;
                    const long long grow = (which ? c0 : r0) + row, gcol = k0 + col;
                    int bytes = 0;
                    if (grow < n && gcol < ke)
                        bytes = gcol + 1 < ke ? 16 : 8;
                    const double *src = bytes ? Z + grow * ldz + gcol : Z;
                    cpAsync16(base + which * kSyrkBM * kSyrkP + row * kSyrkP + col, src, bytes);
                }
            };

            double acc[4][4][2];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++)
                    acc[i][j][0] = acc[i][j][1] = 0.0;
#pragma unroll
            for (int s = 0; s < kSyrkStages - 1; s++)
            {
                if (s < nsteps)
                    load(s, s);
                cpAsyncCommit();
            }
            for (long long step = 0; step < nsteps; step++)
            {
                // step's copies have landed, and every warp is done with the buffer refilled next
                cpAsyncWait<kSyrkStages - 2>();
                __syncthreads();
                const long long nx = step + kSyrkStages - 1;
                if (nx < nsteps)
                    load(nx, (int)(nx % kSyrkStages));
                cpAsyncCommit();
                const double *As = sm + (size_t)(step % kSyrkStages) * kSyrkStageDoubles;
                const double *Bs = As + kSyrkBM * kSyrkP;
#pragma unroll
                for (int kk = 0; kk < kSyrkKB; kk += 4)
                {
                    double af[4], bf[4];
#pragma unroll
                    for (int i = 0; i < 4; i++)
                    {
                        af[i] = As[(wm * 32 + i * 8 + r8) * kSyrkP + kk + k4];
                        bf[i] = Bs[(wn * 32 + i * 8 + r8) * kSyrkP + kk + k4];
                    }
#pragma unroll
                    for (int i = 0; i < 4; i++)
#pragma unroll
                        for (int j = 0; j < 4; j++)
                            dmmaF64(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
                }
            }
            cpAsyncWait<0>();
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++)
#pragma unroll
                    for (int h = 0; h < 2; h++)
                    {
                        const long long r = r0 + wm * 32 + i * 8 + r8;
                        const long long c = c0 + wn * 32 + j * 8 + 2 * k4 + h;
                        if (r < n && c < n && c >= r)
                            atomicAdd(K + r * n + c, sign * acc[i][j][h]);
                    }
        }
    }

    void syrkUpper(const double *Z, long long n, long long k, long long ldz, double sign, double *K, cudaStream_t s)
    {
        if (n <= 0 || k <= 0)
            return;
        if ((ldz & 1) || (reinterpret_cast<uintptr_t>(Z) & 15))
            throw EngineError(kStatusInternal, "syrkUpper: operand rows must start on 16 bytes");
        cudaCheck(cudaFuncSetAttribute(syrkUpperKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSyrkSmem),
                  "syrk attribute");
        int dev = 0, sms = 148;
        cudaCheck(cudaGetDevice(&dev), "device");
        cudaCheck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "sm count");
        const long long T = (n + kSyrkBM - 1) / kSyrkBM;
        const long long tiles = T * (T + 1) / 2;
        // one block per SM: split k so that tiles x slices fills the SMs once
        long long slices = std::max<long long>(1, sms / tiles);
        long long kslice = (k + slices - 1) / slices;
        kslice = (kslice + kSyrkKB - 1) / kSyrkKB * kSyrkKB;
        slices = (k + kslice - 1) / kslice;
        if (tiles > INT32_MAX || slices > 65535)
            throw EngineError(kStatusUnsupported, "syrkUpper: problem too large for one launch");
        syrkUpperKernel<<<dim3((unsigned)tiles, (unsigned)slices), kSyrkThreads, kSyrkSmem, s>>>(Z, n, k, ldz, kslice,
                                                                                               (int)T, sign, K);
        cudaCheck(cudaGetLastError(), "syrk");
    }

    void mirrorUpper(double *K_dev, long long n, cudaStream_t s)
    {
        mirrorUpperKernel<<<gridFor(n * n), 256, 0, s>>>(K_dev, n);
        cudaCheck(cudaGetLastError(), "mirror");
    }

    void factorMetric(Engine &e, MetricFactor &mf)
    {
        const size_t na = e.naux();
        const cudaStream_t s = e.stream();
        mf.method = -1;
        mf.lo = mf.hi = mf.shift = 0;
        mf.dropped = 0;
        mf.naux = na;
        mf.fac.reset(na * na);
        double *metric = mf.fac.p;
        e.eri2(metric);
        e.sync();
        // keep a copy: a failed Cholesky overwrites the matrix
        DevBuf<double> copy(na * na), work;
        DevBuf<int> info(1);
        cudaCheck(cudaMemcpyAsync(copy.p, metric, na * na * sizeof(double), cudaMemcpyDeviceToDevice, s), "copy");
        SolverHandle sh(s);
        int lwork = 0;
        cusolverDnDpotrf_bufferSize(sh.h, CUBLAS_FILL_MODE_LOWER, (int)na, metric, (int)na, &lwork);
        work.reset((size_t)std::max(lwork, 1));
        cusolverDnDpotrf(sh.h, CUBLAS_FILL_MODE_LOWER, (int)na, metric, (int)na, work.p, lwork, info.p);
        int hinfo = 0;
        cudaCheck(cudaMemcpyAsync(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost, s), "info");
        cudaCheck(cudaStreamSynchronize(s), "potrf");
        double shift = 0.0;
        if (hinfo != 0)
        {
            // not numerically positive definite: retry with the diagonal raised by 1e-11 of its largest
            // element (Tikhonov regularisation) before resorting to an eigendecomposition
            std::vector<double> dg(na);
            cudaCheck(cudaMemcpy2DAsync(dg.data(), sizeof(double), copy.p, (na + 1) * sizeof(double), sizeof(double),
                                        na, cudaMemcpyDeviceToHost, s),
                      "diag");
            cudaCheck(cudaStreamSynchronize(s), "diag");
            shift = 1e-11 * *std::max_element(dg.begin(), dg.end());
            for (double &v : dg)
                v += shift;
            cudaCheck(cudaMemcpyAsync(metric, copy.p, na * na * sizeof(double), cudaMemcpyDeviceToDevice, s), "copy");
            cudaCheck(cudaMemcpy2DAsync(metric, (na + 1) * sizeof(double), dg.data(), sizeof(double), sizeof(double),
                                        na, cudaMemcpyHostToDevice, s),
                      "diag");
            cusolverDnDpotrf(sh.h, CUBLAS_FILL_MODE_LOWER, (int)na, metric, (int)na, work.p, lwork, info.p);
            cudaCheck(cudaMemcpyAsync(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost, s), "info");
            cudaCheck(cudaStreamSynchronize(s), "potrf");
        }
        if (hinfo == 0)
        {
            std::vector<double> dg(na);
            cudaCheck(cudaMemcpy2DAsync(dg.data(), sizeof(double), metric, (na + 1) * sizeof(double), sizeof(double),
                                        na, cudaMemcpyDeviceToHost, s),
                      "diag");
            cudaCheck(cudaStreamSynchronize(s), "diag");
            double lo = 1e300, hi = 0;
            for (double v : dg)
            {
                lo = std::min(lo, v * v);
                hi = std::max(hi, v * v);
            }
            mf.method = shift > 0 ? 2 : 0;
            mf.lo = lo;
            mf.hi = hi;
            mf.shift = shift;
            return;
        }
        // eigendecomposition of the unmodified metric (in `copy`; eigenvectors overwrite it)
        DevBuf<double> w(na);
        int lw2 = 0;
        cusolverDnDsyevd_bufferSize(sh.h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, (int)na, copy.p, (int)na,
                                    w.p, &lw2);
        work.reset((size_t)std::max(lw2, 1));
        cusolverDnDsyevd(sh.h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, (int)na, copy.p, (int)na, w.p, work.p,
                         lw2, info.p);
        std::vector<double> hw(na);
        cudaCheck(cudaMemcpyAsync(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost, s), "info");
        cudaCheck(cudaMemcpyAsync(hw.data(), w.p, na * sizeof(double), cudaMemcpyDeviceToHost, s), "w");
        cudaCheck(cudaStreamSynchronize(s), "syevd");
        if (hinfo != 0)
            throw EngineError(kStatusInternal,
                              "eigendecomposition of the RI metric failed (info " + std::to_string(hinfo) + ")");
        const double wmax = *std::max_element(hw.begin(), hw.end());
        std::vector<double> scale(na, 0.0);
        int dropped = 0;
        double lo = 1e300;
        for (size_t k = 0; k < na; k++)
            if (hw[k] > 1e-12 * wmax)
            {
                scale[k] = 1.0 / std::sqrt(hw[k]);
                lo = std::min(lo, hw[k]);
            }
            else
                dropped++;
        DevBuf<double> dscale(na);
        cudaCheck(cudaMemcpyAsync(dscale.p, scale.data(), na * sizeof(double), cudaMemcpyHostToDevice, s), "copy");
        BlasHandle bh(s);
        // G = V diag(scale): column k of the column-major eigenvector matrix times scale_k
        blasCheck(cublasDdgmm(bh.h, CUBLAS_SIDE_RIGHT, (int)na, (int)na, copy.p, (int)na, dscale.p, 1, mf.fac.p,
                              (int)na),
                  "dgmm");
        cudaCheck(cudaStreamSynchronize(s), "metric factor");
        mf.method = 1;
        mf.lo = lo;
        mf.hi = wmax;
        mf.dropped = dropped;
    }

    void solveMetric(Engine &e, const MetricFactor &mf, double *rhs)
    {
        const int na = (int)mf.naux;
        const cudaStream_t s = e.stream();
        if (!mf.solver)
            mf.solver = std::make_unique<SolverHandle>(s);
        if (mf.method == 2)
        {
            DevBuf<int> info(1);
            cusolverDnDpotrs(mf.solver->h, CUBLAS_FILL_MODE_LOWER, na, 1, mf.fac.p, na, rhs, na, info.p);
            cudaCheck(cudaStreamSynchronize(s), "potrs");
            return;
        }
        if (mf.method == 0)
        {
            // M^{-1} from the factor once (potri), then per solve one DSYMV and one step of iterative
            // refinement against the factor (two DTRMV and a second DSYMV) instead of two
            // triangular solves with a single right-hand side: matrix-vector products stream the
            // triangle at HBM rate, and the refinement brings the explicit inverse's error (~cond(M)
            // eps, cond up to 1e10 for even-tempered fitting sets) back to the level of the
            // triangular solves
            if (!mf.inv.p)
            {
                mf.inv.reset((size_t)na * na);
                cudaCheck(cudaMemcpyAsync(mf.inv.p, mf.fac.p, (size_t)na * na * sizeof(double),
                                          cudaMemcpyDeviceToDevice, s),
                          "copy");
                DevBuf<int> info(1);
                DevBuf<double> work;
                int lwork = 0;
                cusolverDnDpotri_bufferSize(mf.solver->h, CUBLAS_FILL_MODE_LOWER, na, mf.inv.p, na, &lwork);
                work.reset((size_t)std::max(lwork, 1));
                cusolverDnDpotri(mf.solver->h, CUBLAS_FILL_MODE_LOWER, na, mf.inv.p, na, work.p, lwork, info.p);
                int hinfo = 0;
                cudaCheck(cudaMemcpyAsync(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost, s), "info");
                cudaCheck(cudaStreamSynchronize(s), "potri");
                if (hinfo != 0)
                {
                    mf.inv.clear();
                    throw EngineError(kStatusInternal, "inverse of the RI metric failed (info " +
                                                           std::to_string(hinfo) + ")");
                }
            }
            if (!mf.blas)
                mf.blas = std::make_unique<BlasHandle>(s);
            const cublasHandle_t h = mf.blas->h;
            DevBuf<double> x(mf.naux), t(mf.naux);
            const double one = 1.0, zero = 0.0, mone = -1.0;
            // x0 = M^{-1} b
            blasCheck(cublasDsymv(h, CUBLAS_FILL_MODE_LOWER, na, &one, mf.inv.p, na, rhs, 1, &zero, x.p, 1), "symv");
            // r = b - L L^T x0 (in place of b), then x = x0 + M^{-1} r
            cudaCheck(cudaMemcpyAsync(t.p, x.p, mf.naux * sizeof(double), cudaMemcpyDeviceToDevice, s), "copy");
            blasCheck(cublasDtrmv(h, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, CUBLAS_DIAG_NON_UNIT, na, mf.fac.p, na, t.p, 1),
                      "trmv");
            blasCheck(cublasDtrmv(h, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, na, mf.fac.p, na, t.p, 1),
                      "trmv");
            blasCheck(cublasDaxpy(h, na, &mone, t.p, 1, rhs, 1), "axpy");
            blasCheck(cublasDsymv(h, CUBLAS_FILL_MODE_LOWER, na, &one, mf.inv.p, na, rhs, 1, &one, x.p, 1), "symv");
            cudaCheck(cudaMemcpyAsync(rhs, x.p, mf.naux * sizeof(double), cudaMemcpyDeviceToDevice, s), "copy");
            cudaCheck(cudaStreamSynchronize(s), "symv");
            return;
        }
        // d = G (G^T gamma)
        BlasHandle bh(s);
        DevBuf<double> c(mf.naux);
        const double one = 1.0, zero = 0.0;
        blasCheck(cublasDgemv(bh.h, CUBLAS_OP_T, na, na, &one, mf.fac.p, na, rhs, 1, &zero, c.p, 1), "gemv");
        blasCheck(cublasDgemv(bh.h, CUBLAS_OP_N, na, na, &one, mf.fac.p, na, c.p, 1, &zero, rhs, 1), "gemv");
        cudaCheck(cudaStreamSynchronize(s), "eigen solve");
    }

    void riExchange(Engine &e, BlasHandle &bh, const MetricFactor &mf, const double *C_dev, long long occ,
                    double schwarz, double sign, double *K_dev, size_t block_bytes, RIKStats *stats)
    {
        if (occ <= 0)
            return;
        const long long n = (long long)e.nao(), na = (long long)e.naux();
        const cudaStream_t s = e.stream();
        const long long m = n * occ;  // rows of the column-major view of Z: (m, i) fused
        if (m > INT32_MAX || na > INT32_MAX)
            throw EngineError(kStatusUnsupported, "RI-K: nao * occ exceeds the 32-bit cuBLAS dimension range");

        // auxiliary blocks: whole shells, at most block_bytes of T (one shell at least)
        const std::vector<int> starts = e.auxShellStarts();
        const long long per_fn = n * n * (long long)sizeof(double);
        const long long cap = std::max<long long>(1, (long long)block_bytes / per_fn);
        std::vector<std::pair<int, int>> blocks;
        for (size_t i = 0; i + 1 < starts.size();)
        {
            size_t j = i + 1;
            while (j + 1 < starts.size() && starts[j + 1] - starts[i] <= cap)
                j++;
            blocks.push_back({starts[i], starts[j]});
            i = j;
        }
        long long pb_max = 0;
        for (auto &b : blocks)
            pb_max = std::max<long long>(pb_max, b.second - b.first);

        // T also serves as the scratch of the eigen-path product (na per row) and of the re-laid-out
        // W blocks (m per auxiliary function)
        DevBuf<double> Z((size_t)(na * m)), T((size_t)std::max({pb_max * n * n, na, m}));
        EventPair ev_int, ev_gemm, ev_solve, ev_syrk;
        double t_int = 0, t_gemm = 0;
        const double one = 1.0, zero = 0.0;
        for (auto &b : blocks)
        {
            const long long pb = b.second - b.first;
            cudaCheck(cudaEventRecord(ev_int.a, s), "event");
            e.riStore(b.first, b.second, T.p, schwarz);
            cudaCheck(cudaEventRecord(ev_int.b, s), "event");
            // Z_cm (occ x pb*n) = C_cm (occ x n) . T_cm (n x pb*n): row-major Z[P][m][i] = T[P][m][:] . C
            cudaCheck(cudaEventRecord(ev_gemm.a, s), "event");
            blasCheck(cublasDgemm(bh.h, CUBLAS_OP_N, CUBLAS_OP_N, (int)occ, (int)(pb * n), (int)n, &one, C_dev,
                                  (int)occ, T.p, (int)n, &zero, Z.p + (size_t)b.first * m, (int)occ),
                      "dgemm");
            cudaCheck(cudaEventRecord(ev_gemm.b, s), "event");
            cudaCheck(cudaEventSynchronize(ev_gemm.b), "ri block");
            t_int += ev_int.seconds();
            t_gemm += ev_gemm.seconds();
        }
        e.checkStatus();

        // W = L^{-1} Z along P.  Column-major view: Z_cm (m x na), W_cm L^T = Z_cm.
        cudaCheck(cudaEventRecord(ev_solve.a, s), "event");
        if (mf.method == 0 || mf.method == 2)
        {
            blasCheck(cublasDtrsm(bh.h, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, CUBLAS_DIAG_NON_UNIT,
                                  (int)m, (int)na, &one, mf.fac.p, (int)na, Z.p, (int)m),
                      "dtrsm");
        }
        else
        {
            // W_cm = Z_cm G, by row blocks of Z_cm through a scratch of at most T's size
            const long long mb = std::max<long long>(1, std::min<long long>(m, (long long)T.n / na));
            for (long long r0 = 0; r0 < m; r0 += mb)
            {
                const long long rows = std::min(mb, m - r0);
                blasCheck(cublasDgemm(bh.h, CUBLAS_OP_N, CUBLAS_OP_N, (int)rows, (int)na, (int)na, &one, Z.p + r0,
                                      (int)m, mf.fac.p, (int)na, &zero, T.p, (int)rows),
                          "dgemm");
                cudaCheck(cudaMemcpy2DAsync(Z.p + r0, (size_t)m * sizeof(double), T.p, (size_t)rows * sizeof(double),
                                            (size_t)rows * sizeof(double), (size_t)na, cudaMemcpyDeviceToDevice, s),
                          "copy");
            }
        }
        cudaCheck(cudaEventRecord(ev_solve.b, s), "event");

        // K += sign * sum_R W_R W_R^T, R in blocks laid out as A[m][R][i] (T reused as A)
        cudaCheck(cudaEventRecord(ev_syrk.a, s), "event");
        const long long rb = std::max<long long>(1, std::min<long long>(na, (long long)T.n / m));
        for (long long r0 = 0; r0 < na; r0 += rb)
        {
            const long long rows = std::min(rb, na - r0);
            relayoutKernel<<<gridFor(n * rows * occ), 256, 0, s>>>(Z.p, n, occ, r0, rows, T.p);
            cudaCheck(cudaGetLastError(), "relayout");
            // the DMMA SYRK on even row lengths (rows start on 16 bytes), else cuBLAS
            if ((rows * occ) % 2 == 0)
                syrkUpper(T.p, n, rows * occ, rows * occ, sign, K_dev, s);
            else
                blasCheck(cublasDsyrk(bh.h, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, (int)n, (int)(rows * occ), &sign,
                                      T.p, (int)(rows * occ), &one, K_dev, (int)n),
                          "dsyrk");
        }
        cudaCheck(cudaEventRecord(ev_syrk.b, s), "event");
        cudaCheck(cudaEventSynchronize(ev_syrk.b), "ri exchange");
        if (stats)
        {
            stats->t_ints += t_int;
            stats->t_gemm += t_gemm;
            stats->t_solve += ev_solve.seconds();
            stats->t_syrk += ev_syrk.seconds();
            stats->n_blocks += (int)blocks.size();
            stats->flops_gemm += 2.0 * (double)na * (double)n * (double)n * (double)occ;
            stats->flops_solve += (mf.method == 1 ? 2.0 : 1.0) * (double)na * (double)na * (double)m;
            stats->flops_syrk += (double)n * (double)(n + 1) * (double)na * (double)occ;
        }
    }

    void buildFitted(Engine &e, BlasHandle &bh, const MetricFactor &mf, double schwarz, FittedTensor &ft)
    {
        const long long n = (long long)e.nao(), na = (long long)e.naux();
        const cudaStream_t s = e.stream();
        const long long rows = n * n;  // column-major view of T[P][m][n]: rows (m, n), columns P
        if (rows > INT32_MAX || na > INT32_MAX)
            throw EngineError(kStatusUnsupported, "RI-K: nao^2 exceeds the 32-bit cuBLAS dimension range");
        ft.B.reset((size_t)(na * rows));
        EventPair ev;
        cudaCheck(cudaEventRecord(ev.a, s), "event");
        // all auxiliary functions in one store launch sequence: T[P][m][n] = (mn|P)
        e.riStore(0, (int)na, ft.B.p, schwarz);
        e.checkStatus();
        const double one = 1.0, zero = 0.0;
        if (mf.method == 0 || mf.method == 2)
        {
            // B_cm L^T = T_cm  (B_cm = T_cm L^{-T}: column R of B is sum_P T_P (L^{-T})_PR)
            blasCheck(cublasDtrsm(bh.h, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, CUBLAS_DIAG_NON_UNIT,
                                  (int)rows, (int)na, &one, mf.fac.p, (int)na, ft.B.p, (int)rows),
                      "dtrsm");
        }
        else
        {
            // B_cm = T_cm G by row blocks through a scratch of at most 1 GiB
            const long long mb = std::max<long long>(1, std::min<long long>(rows, (1LL << 27) / std::max(na, 1LL)));
            DevBuf<double> tmp((size_t)(mb * na));
            for (long long r0 = 0; r0 < rows; r0 += mb)
            {
                const long long rr = std::min(mb, rows - r0);
                blasCheck(cublasDgemm(bh.h, CUBLAS_OP_N, CUBLAS_OP_N, (int)rr, (int)na, (int)na, &one, ft.B.p + r0,
                                      (int)rows, mf.fac.p, (int)na, &zero, tmp.p, (int)rr),
                          "dgemm");
                cudaCheck(cudaMemcpy2DAsync(ft.B.p + r0, (size_t)rows * sizeof(double), tmp.p,
                                            (size_t)rr * sizeof(double), (size_t)rr * sizeof(double), (size_t)na,
                                            cudaMemcpyDeviceToDevice, s),
                          "copy");
            }
        }
        cudaCheck(cudaEventRecord(ev.b, s), "event");
        cudaCheck(cudaEventSynchronize(ev.b), "fitted tensor");
        ft.schwarz = schwarz;
        ft.naux = (size_t)na;
        ft.nao = (size_t)n;
        ft.t_build = ev.seconds();
    }

    void riExchangeFitted(Engine &e, BlasHandle &bh, const FittedTensor &ft, const double *C_dev, long long occ,
                          double sign, double *K_dev, RIKStats *stats)
    {
        if (occ <= 0)
            return;
        const long long n = (long long)ft.nao, na = (long long)ft.naux;
        const cudaStream_t s = e.stream();
        const long long k = na * occ;
        if (k > INT32_MAX)
            throw EngineError(kStatusUnsupported, "RI-K: naux * occ exceeds the 32-bit cuBLAS dimension range");
        // Z[m][R][i] = sum_n B[R][m][n] C[n][i], written straight in the layout of the final product:
        // per R one GEMM, in column-major terms Z_R,cm (occ x n, ld = naux*occ) = C_cm (occ x n) B_R,cm
        // (B_R symmetric in (m, n)); all R as one strided batch
        // rows of Z padded to an even length, so each starts on 16 bytes for the SYRK's copies
        const long long ldz = k + (k & 1);
        if (ldz > INT32_MAX)
            throw EngineError(kStatusUnsupported, "RI-K: naux * occ exceeds the 32-bit cuBLAS dimension range");
        if (ft.Z.n < (size_t)(n * ldz))
        {
            ft.Z.clear();
            ft.Z.reset((size_t)(n * ldz));
        }
        DevBuf<double> &Z = ft.Z;
        EventPair ev_gemm, ev_syrk;
        const double one = 1.0, zero = 0.0;
        cudaCheck(cudaEventRecord(ev_gemm.a, s), "event");
        blasCheck(cublasDgemmStridedBatched(bh.h, CUBLAS_OP_N, CUBLAS_OP_N, (int)occ, (int)n, (int)n, &one, C_dev,
                                            (int)occ, 0, ft.B.p, (int)n, n * n, &zero, Z.p, (int)ldz, occ, (int)na),
                  "dgemm batched");
        cudaCheck(cudaEventRecord(ev_gemm.b, s), "event");
        // K += sign Z Z^T over (R, i), the upper triangle by the DMMA kernel
        cudaCheck(cudaEventRecord(ev_syrk.a, s), "event");
        syrkUpper(Z.p, n, k, ldz, sign, K_dev, s);
        cudaCheck(cudaEventRecord(ev_syrk.b, s), "event");
        cudaCheck(cudaEventSynchronize(ev_syrk.b), "ri exchange");
        if (stats)
        {
            stats->t_gemm += ev_gemm.seconds();
            stats->t_syrk += ev_syrk.seconds();
            stats->flops_gemm += 2.0 * (double)na * (double)n * (double)n * (double)occ;
            stats->flops_syrk += (double)n * (double)(n + 1) * (double)na * (double)occ;
        }
    }

    namespace
    {
        // gamma[P] = sum_e T[P][e] D[e], e over the n2 elements of a row: one block per row P (rows
        // streamed once from HBM, D read from L2), a block reduction of 256 partial sums.  Rows are
        // read as double2 when n2 is even (every row then starts on 16 bytes).
        template <bool VEC>
        __global__ void __launch_bounds__(256) t3GammaKernel(const double *__restrict__ T, const double *__restrict__ D,
                                                             long long n2, long long naux, double *__restrict__ gamma)
        {
            __shared__ double red[8];
            for (long long P = blockIdx.x; P < naux; P += gridDim.x)
            {
                double s0 = 0.0, s1 = 0.0;
                if constexpr (VEC)
                {
                    const double2 *row = reinterpret_cast<const double2 *>(T + P * n2);
                    const double2 *d2 = reinterpret_cast<const double2 *>(D);
                    for (long long e = threadIdx.x; e < n2 / 2; e += 256)
                    {
                        const double2 t = __ldcs(row + e);  // streamed once: no reuse in L2
                        const double2 d = __ldg(d2 + e);
                        s0 = fma(t.x, d.x, s0);
                        s1 = fma(t.y, d.y, s1);
                    }
                }
                else
                {
                    for (long long e = threadIdx.x; e < n2; e += 256)
                        s0 = fma(__ldcs(T + P * n2 + e), __ldg(D + e), s0);
                }
                double v = s0 + s1;
                for (int o = 16; o > 0; o >>= 1)
                    v += __shfl_down_sync(0xffffffffu, v, o);
                if ((threadIdx.x & 31) == 0)
                    red[threadIdx.x >> 5] = v;
                __syncthreads();
                if (threadIdx.x == 0)
                {
                    double t = 0.0;
                    for (int w = 0; w < 8; w++)
                        t += red[w];
                    gamma[P] = t;
                }
                __syncthreads();
            }
        }

        // J[e] += sum_{P in the block's range} d[P] T[P][e]: blocks tile the n2 elements (a double2
        // per thread when n2 is even, else one double) and split the auxiliary range in slices of
        // `per`; each element of T is read once, two rows in flight per step.
        template <bool VEC>
        __global__ void __launch_bounds__(256) t3CoulombKernel(const double *__restrict__ T, const double *__restrict__ dcoef,
                                                               long long n2, long long naux, long long per,
                                                               double *__restrict__ J)
        {
            const long long e = (long long)blockIdx.x * 256 + threadIdx.x;
            const long long P0 = (long long)blockIdx.y * per, P1 = P0 + per < naux ? P0 + per : naux;
            if constexpr (VEC)
            {
                if (2 * e >= n2)
                    return;
                double a0 = 0.0, a1 = 0.0, b0 = 0.0, b1 = 0.0;
                long long P = P0;
                for (; P + 1 < P1; P += 2)
                {
                    const double2 t0 = __ldcs(reinterpret_cast<const double2 *>(T + P * n2) + e);
                    const double2 t1 = __ldcs(reinterpret_cast<const double2 *>(T + (P + 1) * n2) + e);
                    const double d0 = __ldg(dcoef + P), d1 = __ldg(dcoef + P + 1);
                    a0 = fma(t0.x, d0, a0);
                    a1 = fma(t0.y, d0, a1);
                    b0 = fma(t1.x, d1, b0);
                    b1 = fma(t1.y, d1, b1);
                }
                if (P < P1)
                {
                    const double2 t0 = __ldcs(reinterpret_cast<const double2 *>(T + P * n2) + e);
                    const double d0 = __ldg(dcoef + P);
                    a0 = fma(t0.x, d0, a0);
                    a1 = fma(t0.y, d0, a1);
                }
                atomicAdd(J + 2 * e, a0 + b0);
                atomicAdd(J + 2 * e + 1, a1 + b1);
            }
            else
            {
                if (e >= n2)
                    return;
                double a0 = 0.0;
                for (long long P = P0; P < P1; P++)
                    a0 = fma(__ldcs(T + P * n2 + e), __ldg(dcoef + P), a0);
                atomicAdd(J + e, a0);
            }
        }

        // Dp[i (i + 1) / 2 + j] = D_ij + D_ji for j < i, D_ii for j = i (one thread per element).
        __global__ void packDensityKernel(const double *__restrict__ D, long long n, double *__restrict__ Dp)
        {
            const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
            if (e >= n * n)
                return;
            const long long i = e / n, j = e % n;
            if (j > i)
                return;
            Dp[i * (i + 1) / 2 + j] = i == j ? D[e] : D[e] + D[j * n + i];
        }

        // J_ij = J_ji = Jp[max (max + 1) / 2 + min] (one thread per element of J).
        __global__ void unpackTriangleKernel(const double *__restrict__ Jp, long long n, double *__restrict__ J)
        {
            const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
            if (e >= n * n)
                return;
            const long long i = e / n, j = e % n;
            J[e] = i >= j ? Jp[i * (i + 1) / 2 + j] : Jp[j * (j + 1) / 2 + i];
        }
    }

    void buildT3(Engine &e, double schwarz, CachedT3 &t3)
    {
        const size_t n = e.nao(), na = e.naux();
        t3.T.reset(na * CachedT3::rowLength(n));
        EventPair ev;
        cudaCheck(cudaEventRecord(ev.a, e.stream()), "event");
        e.riStore(0, (int)na, t3.T.p, schwarz, true);
        e.checkStatus();
        cudaCheck(cudaEventRecord(ev.b, e.stream()), "event");
        cudaCheck(cudaEventSynchronize(ev.b), "three-centre tensor");
        t3.schwarz = schwarz;
        t3.naux = na;
        t3.nao = n;
        t3.t_build = ev.seconds();
    }

    void t3Gamma(Engine &e, const CachedT3 &t3, const double *D_dev, double *gamma_dev)
    {
        const long long n = (long long)t3.nao, n2 = (long long)CachedT3::rowLength(t3.nao), na = (long long)t3.naux;
        if (t3.Dp.n < (size_t)n2)
            t3.Dp.reset((size_t)n2);
        packDensityKernel<<<(unsigned)((n * n + 255) / 256), 256, 0, e.stream()>>>(D_dev, n, t3.Dp.p);
        cudaCheck(cudaGetLastError(), "t3 pack");
        const int grid = (int)std::min<long long>(na, 148LL * 8);
        if (n2 % 2 == 0)
            t3GammaKernel<true><<<grid, 256, 0, e.stream()>>>(t3.T.p, t3.Dp.p, n2, na, gamma_dev);
        else
            t3GammaKernel<false><<<grid, 256, 0, e.stream()>>>(t3.T.p, t3.Dp.p, n2, na, gamma_dev);
        cudaCheck(cudaGetLastError(), "t3 gamma");
    }

    void t3Coulomb(Engine &e, const CachedT3 &t3, const double *d_dev, double *J_out)
    {
        const long long n = (long long)t3.nao, n2 = (long long)CachedT3::rowLength(t3.nao), na = (long long)t3.naux;
        if (t3.Jp.n < (size_t)n2)
            t3.Jp.reset((size_t)n2);
        double *J_dev = t3.Jp.p;
        cudaCheck(cudaMemsetAsync(J_dev, 0, (size_t)n2 * sizeof(double), e.stream()), "memset");
        const bool vec = n2 % 2 == 0;
        const long long blocks = ((vec ? n2 / 2 : n2) + 255) / 256;
        // enough auxiliary slices to give every SM several blocks
        const long long ps = std::max<long long>(1, std::min<long long>(na, (148LL * 16 + blocks - 1) / blocks));
        const long long per = (na + ps - 1) / ps;
        const dim3 grid((unsigned)blocks, (unsigned)((na + per - 1) / per));
        if (vec)
            t3CoulombKernel<true><<<grid, 256, 0, e.stream()>>>(t3.T.p, d_dev, n2, na, per, J_dev);
        else
            t3CoulombKernel<false><<<grid, 256, 0, e.stream()>>>(t3.T.p, d_dev, n2, na, per, J_dev);
        cudaCheck(cudaGetLastError(), "t3 coulomb");
        unpackTriangleKernel<<<(unsigned)((n * n + 255) / 256), 256, 0, e.stream()>>>(J_dev, n, J_out);
        cudaCheck(cudaGetLastError(), "t3 unpack");
    }

    void splitDensity(Engine &e, const double *D_dev, long long n, DevBuf<double> &Cp, long long &n_pos,
                      DevBuf<double> &Cm, long long &n_neg)
    {
        const cudaStream_t s = e.stream();
        // D is symmetric, so its row-major layout is also its column-major one
        DevBuf<double> U((size_t)(n * n)), w((size_t)n), work;
        DevBuf<int> info(1);
        cudaCheck(cudaMemcpyAsync(U.p, D_dev, (size_t)(n * n) * sizeof(double), cudaMemcpyDeviceToDevice, s), "copy");
        SolverHandle sh(s);
        int lw = 0;
        cusolverDnDsyevd_bufferSize(sh.h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, (int)n, U.p, (int)n, w.p,
                                    &lw);
        work.reset((size_t)std::max(lw, 1));
        cusolverDnDsyevd(sh.h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, (int)n, U.p, (int)n, w.p, work.p, lw,
                         info.p);
        int hinfo = 0;
        std::vector<double> hw((size_t)n);
        cudaCheck(cudaMemcpyAsync(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost, s), "info");
        cudaCheck(cudaMemcpyAsync(hw.data(), w.p, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, s), "w");
        cudaCheck(cudaStreamSynchronize(s), "syevd");
        if (hinfo != 0)
            throw EngineError(kStatusInternal, "eigendecomposition of D failed (info " + std::to_string(hinfo) + ")");
        double wmax = 0;
        for (double v : hw)
            wmax = std::max(wmax, std::fabs(v));
        std::vector<int> ip, im;
        std::vector<double> sp, sm;
        for (long long k = 0; k < n; k++)
        {
            if (!(std::fabs(hw[k]) > 1e-12 * wmax))
                continue;
            if (hw[k] > 0)
            {
                ip.push_back((int)k);
                sp.push_back(std::sqrt(hw[k]));
            }
            else
            {
                im.push_back((int)k);
                sm.push_back(std::sqrt(-hw[k]));
            }
        }
        auto build = [&](const std::vector<int> &idx, const std::vector<double> &sc, DevBuf<double> &C) {
            const long long k = (long long)idx.size();
            C.reset((size_t)std::max<long long>(n * k, 1));
            if (k == 0)
                return;
            DevBuf<int> didx(idx.size());
            DevBuf<double> dsc(sc.size());
            cudaCheck(cudaMemcpyAsync(didx.p, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice, s), "copy");
            cudaCheck(cudaMemcpyAsync(dsc.p, sc.data(), sc.size() * sizeof(double), cudaMemcpyHostToDevice, s), "copy");
            factorColumnsKernel<<<gridFor(n * k), 256, 0, s>>>(U.p, n, didx.p, dsc.p, k, C.p);
            cudaCheck(cudaGetLastError(), "factor");
            cudaCheck(cudaStreamSynchronize(s), "factor");
        };
        build(ip, sp, Cp);
        build(im, sm, Cm);
        n_pos = (long long)ip.size();
        n_neg = (long long)im.size();
    }
}
