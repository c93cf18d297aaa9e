// RI building blocks shared by the RI-J and RI-K entry points: owning device buffers and library
// handles, the factorised metric (P|Q), and the RI exchange build.
#pragma once

#include "engine_api.hpp"

#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <algorithm>
#include <memory>

namespace lible_b200
{
    // Owning device buffer (freed on scope exit, also when a check throws).
    template <class T>
    struct DevBuf
    {
        T *p = nullptr;
        size_t n = 0;
        DevBuf() = default;
        explicit DevBuf(size_t count) { reset(count); }
        void reset(size_t count)
        {
            cudaFree(p);
            p = nullptr;
            n = 0;
            cudaCheck(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)), "cudaMalloc");
            n = count;
        }
        void clear()
        {
            cudaFree(p);
            p = nullptr;
            n = 0;
        }
        ~DevBuf() { cudaFree(p); }
        DevBuf(const DevBuf &) = delete;
        DevBuf &operator=(const DevBuf &) = delete;
    };

    struct SolverHandle
    {
        cusolverDnHandle_t h = nullptr;
        explicit SolverHandle(cudaStream_t s = nullptr)
        {
            if (cusolverDnCreate(&h) != CUSOLVER_STATUS_SUCCESS)
                throw EngineError(kStatusCuda, "cusolverDnCreate failed");
            cusolverDnSetStream(h, s);
        }
        ~SolverHandle() { cusolverDnDestroy(h); }
        SolverHandle(const SolverHandle &) = delete;
        SolverHandle &operator=(const SolverHandle &) = delete;
    };

    struct BlasHandle
    {
        cublasHandle_t h = nullptr;
        explicit BlasHandle(cudaStream_t s = nullptr)
        {
            if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS)
                throw EngineError(kStatusCuda, "cublasCreate failed");
            cublasSetStream(h, s);
        }
        ~BlasHandle() { cublasDestroy(h); }
        BlasHandle(const BlasHandle &) = delete;
        BlasHandle &operator=(const BlasHandle &) = delete;
    };

    void blasCheck(cublasStatus_t s, const char *what);

    // The RI metric M = (P|Q) of the engine's auxiliary basis, factorised on the device.
    //  * method 0: Cholesky M = L L^T (`fac` = L, lower triangle, column-major);
    //  * method 2: the same after raising the diagonal by `shift` (1e-11 of its largest element),
    //    when M is not numerically positive definite;
    //  * method 1: eigendecomposition M = V diag(w) V^T when the shifted Cholesky fails too; `fac` =
    //    G = V diag(w^{-1/2}) with the columns of w < 1e-12 max(w) set to zero (`dropped` of them),
    //    so M^{-1} is replaced by G G^T.
    // lo / hi: the squared range of the Cholesky diagonal (a bound on the conditioning), or the
    // range of the kept eigenvalues.
    struct MetricFactor
    {
        int method = -1;
        double lo = 0, hi = 0, shift = 0;
        int dropped = 0;
        size_t naux = 0;
        DevBuf<double> fac;
        // M^{-1} (lower triangle, column-major), formed from the Cholesky factor by the first solve
        // of method 0 (a positive definite metric), so that every solve is one symmetric
        // matrix-vector product; the shifted and eigen methods keep their solves
        mutable DevBuf<double> inv;
        // solver and cuBLAS handles of the solves, created once
        mutable std::unique_ptr<SolverHandle> solver;
        mutable std::unique_ptr<BlasHandle> blas;
    };
    void factorMetric(Engine &e, MetricFactor &mf);

    // rhs <- M^{-1} rhs (device vector of naux doubles).
    void solveMetric(Engine &e, const MetricFactor &mf, double *rhs);

    // K += sign * sum_{PQ} (m l|P) M^{-1}_{PQ} (Q|n s) (C C^T)_{ls} for the device factor C
    // ([nao][occ] row-major), into the lower-stored device K (column-major lower triangle = the
    // row-major upper triangle; the caller mirrors it).  The three-centre integrals are built in
    // blocks of auxiliary functions of at most `block_bytes` and contracted with C at once, so
    // only Z = (mn|P) C (naux x nao x occ doubles) is held in full.
    struct RIKStats
    {
        double t_ints = 0, t_gemm = 0, t_solve = 0, t_syrk = 0;  // seconds (CUDA events)
        int n_blocks = 0;
        double flops_gemm = 0, flops_solve = 0, flops_syrk = 0;
    };
    void riExchange(Engine &e, BlasHandle &bh, const MetricFactor &mf, const double *C_dev, long long occ,
                    double schwarz, double sign, double *K_dev, size_t block_bytes, RIKStats *stats);

    // The fitted three-centre tensor B[R][m][n] = sum_P F_PR (mn|P), F = L^{-T} (Cholesky) or G
    // (eigendecomposition), so that sum_R B_R,mn B_R,ls = sum_PQ (mn|P) M^{-1}_PQ (Q|ls).  Built once
    // per structure and Schwarz threshold (naux * nao^2 doubles) and kept in HBM; every later
    // exchange build is then one strided-batched DGEMM and one symmetric rank-k product.
    struct FittedTensor
    {
        DevBuf<double> B;
        double schwarz = -1;
        size_t naux = 0, nao = 0;
        double t_build = 0;  // seconds of the build (integrals + fit)
        // the exchange operand Z of the last call, kept so that later calls with at most as many
        // occupied columns reuse it instead of allocating and freeing naux * nao * occ doubles
        mutable DevBuf<double> Z;
    };
    void buildFitted(Engine &e, BlasHandle &bh, const MetricFactor &mf, double schwarz, FittedTensor &ft);
    // K += sign * sum_R (B_R C)(B_R C)^T with the cached tensor (same contract as riExchange).
    void riExchangeFitted(Engine &e, BlasHandle &bh, const FittedTensor &ft, const double *C_dev, long long occ,
                          double sign, double *K_dev, RIKStats *stats);

    // The raw three-centre tensor (mn|P) (Schwarz screened), kept in HBM by the RI-J calls when it
    // fits; each RI-J is then two passes over it.  (mn|P) is symmetric in m, n, so only the lower
    // triangle is kept: T[P][i (i + 1) / 2 + j] = (ij|P), j <= i, naux * nao (nao + 1) / 2 doubles.
    struct CachedT3
    {
        DevBuf<double> T;
        double schwarz = -1;
        size_t naux = 0, nao = 0;
        double t_build = 0;  // seconds of the build
        // packed operands of the two passes: D_ij + D_ji (D_ii on the diagonal), and J's triangle
        mutable DevBuf<double> Dp, Jp;
        static size_t rowLength(size_t nao) { return nao * (nao + 1) / 2; }
    };
    void buildT3(Engine &e, double schwarz, CachedT3 &t3);
    // gamma_P = sum_mn (mn|P) D_mn (full sum over both triangles; D need not be symmetric).
    void t3Gamma(Engine &e, const CachedT3 &t3, const double *D_dev, double *gamma_dev);
    // J_mn = sum_P (mn|P) d_P (symmetric by construction).
    void t3Coulomb(Engine &e, const CachedT3 &t3, const double *d_dev, double *J_dev);

    // Mirrors the row-major upper triangle of the n x n matrix into the lower one.
    void mirrorUpper(double *K_dev, long long n, cudaStream_t s);

    // Factor of a symmetric device matrix D (n x n): D = C+ C+^T - C- C-^T from its eigenpairs with
    // |w| > 1e-12 max|w|; C+ / C- are allocated here ([n][n_pos] / [n][n_neg] row-major).
    void splitDensity(Engine &e, const double *D_dev, long long n, DevBuf<double> &Cp, long long &n_pos,
                      DevBuf<double> &Cm, long long &n_neg);
}
