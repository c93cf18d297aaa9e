// The C ABI (include/lible_b200.h) over the Engine.  Converts exceptions to status codes and
// stages host arrays through device memory.
#include "../../include/lible_b200.h"
#include "engine_api.hpp"
#include "ri_solve.hpp"

#include <cuda_runtime.h>
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <map>
#include <mutex>
#include <string>

using namespace lible_b200;

namespace lible_b200
{
    // noalloc.cu: device address of the allocation-free call's staging buffer on the current device.
    uint32_t *noAllocScratch(long long *max_pairs);
    // peak.cu: measured FP32 throughput {FFMA, packed FFMA2} in TFLOP/s.
    std::pair<double, double> measureFp32Peak(int device, cudaStream_t s);
}

struct lible_gpu_ctx
{
    std::unique_ptr<Engine> eng;
    // serialises the calls on this context (every entry point that touches it holds the lock)
    std::recursive_mutex mu;
    // last RI-J metric solve: 0 Cholesky, 1 eigendecomposition with cutoff; eigenvalue range (or
    // the squared range of the Cholesky diagonal, a lower bound of the condition number); dropped
    int rij_method = -1;
    double rij_lo = 0, rij_hi = 0;
    int rij_dropped = 0;
    double rij_shift = 0;
    // factorised RI metric of the current structure (built by the first RI-J / RI-K call) and the
    // cuBLAS handle of the RI calls; both dropped when the structure changes
    std::unique_ptr<MetricFactor> metric;
    std::unique_ptr<BlasHandle> blas;
    // fitted three-centre tensor of the RI-K calls (built by the first call that has the room);
    // rik_fitted_mode 0 = never build it (stream the integrals on every call), 1 = when it fits
    std::unique_ptr<FittedTensor> fitted;
    int rik_fitted_mode = 1;
    // three-centre tensor (mn|P) of the RI-J calls, kept when it fits (rij_cached_mode 1) so that
    // every later RI-J is two streaming passes over it instead of two integral evaluations
    std::unique_ptr<CachedT3> t3;
    int rij_cached_mode = 1;

    void structureChanged()
    {
        metric.reset();
        fitted.reset();
        t3.reset();
    }
    const MetricFactor &metricFactor(Engine &e)
    {
        if (!metric)
        {
            auto m = std::make_unique<MetricFactor>();
            factorMetric(e, *m);
            metric = std::move(m);
        }
        rij_method = metric->method;
        rij_lo = metric->lo;
        rij_hi = metric->hi;
        rij_dropped = metric->dropped;
        rij_shift = metric->shift;
        return *metric;
    }
    BlasHandle &blasHandle(Engine &e)
    {
        if (!blas)
            blas = std::make_unique<BlasHandle>(e.stream());
        return *blas;
    }
};

namespace
{
    // The calling thread's last error message per context: a call that succeeds on another thread
    // in the meantime does not clear it.
    thread_local std::map<const lible_gpu_ctx *, std::string> t_errors;

    int fail(lible_gpu_ctx *ctx, int code, const std::string &msg)
    {
        if (ctx)
            t_errors[ctx] = msg;
        return code;
    }

    template <class F>
    int guard(lible_gpu_ctx *ctx, F &&f)
    {
        if (!ctx || !ctx->eng)
            return LIBLE_GPU_EINVAL;
        std::lock_guard<std::recursive_mutex> lock(ctx->mu);
        try
        {
            cudaSetDevice(ctx->eng->device());
            f(*ctx->eng);
            t_errors.erase(ctx);
            return LIBLE_GPU_OK;
        }
        catch (const EngineError &e)
        {
            return fail(ctx, e.code, e.what());
        }
        catch (const std::exception &e)
        {
            return fail(ctx, LIBLE_GPU_EINTERNAL, e.what());
        }
    }

    bool isDevice(const void *p)
    {
        if (!p)
            return false;
        cudaPointerAttributes at{};
        if (cudaPointerGetAttributes(&at, p) != cudaSuccess)
        {
            cudaGetLastError();
            return false;
        }
        return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
    }

    // Device view of a caller array: the array itself if it is device memory, else a staged copy.
    // With an engine and a slot, host arrays are staged in the context's cached buffer of that slot
    // (grow-only, kept until the context is destroyed), so repeated calls allocate nothing and the
    // device addresses stay stable (which keeps captured CUDA graphs valid).
    struct DevArray
    {
        double *ptr = nullptr;
        double *user = nullptr;
        size_t n = 0;
        bool owned = false, staged = false;
        cudaStream_t s = nullptr;

        DevArray(const double *p, size_t count, bool copy_in, cudaStream_t stream, Engine *eng = nullptr,
                 int slot = -1)
            : user(const_cast<double *>(p)), n(count), s(stream)
        {
            if (!p)
                return;
            if (isDevice(p))
            {
                ptr = const_cast<double *>(p);
                return;
            }
            staged = true;
            if (eng && slot >= 0)
                ptr = eng->staging(slot, std::max<size_t>(n, 1));
            else
            {
                cudaCheck(cudaMalloc(&ptr, std::max<size_t>(n, 1) * sizeof(double)), "cudaMalloc");
                owned = true;
            }
            if (copy_in)
                cudaCheck(cudaMemcpyAsync(ptr, p, n * sizeof(double), cudaMemcpyHostToDevice, s), "H2D");
        }
        void copyOut()
        {
            if (staged && user)
            {
                cudaCheck(cudaMemcpyAsync(user, ptr, n * sizeof(double), cudaMemcpyDeviceToHost, s), "D2H");
                cudaCheck(cudaStreamSynchronize(s), "D2H");
            }
            else
                cudaCheck(cudaStreamSynchronize(s), "sync");
        }
        ~DevArray()
        {
            if (owned)
                cudaFree(ptr);
        }
    };

    std::vector<std::array<double, 3>> coords(int n_atoms, const double *xyz, int units)
    {
        std::vector<std::array<double, 3>> c(n_atoms);
        const double f = units == 0 ? kAngstromToBohr : 1.0;
        for (int a = 0; a < n_atoms; a++)
            for (int k = 0; k < 3; k++)
                c[a][k] = xyz[3 * a + k] * f;
        return c;
    }

    std::vector<BasisAtom> atomsFromArrays(int n_atoms, const int *Z, const int *nsh, const int *l,
                                           const int *np, const double *exps, const double *coeffs)
    {
        std::vector<BasisAtom> atoms(n_atoms);
        size_t is = 0, ip = 0;
        for (int a = 0; a < n_atoms; a++)
        {
            atoms[a].z = Z[a];
            for (int k = 0; k < nsh[a]; k++, is++)
            {
                BasisShell s;
                s.l = l[is];
                if (np[is] <= 0)
                    throw EngineError(kStatusInvalid, "shell with no primitives");
                for (int p = 0; p < np[is]; p++, ip++)
                {
                    s.exps.push_back(exps[ip]);
                    s.coeffs.push_back(coeffs[ip]);
                }
                atoms[a].shells.push_back(s);
            }
        }
        return atoms;
    }
}

extern "C" {

int lible_host_spherical_trafo(int l, int *n, int *rows, int *carts, double *vals)
{
    if (!n || l < 0 || l > 8)
        return LIBLE_GPU_EINVAL;
    auto t = sphericalTrafo(l);
    const int cap = *n;
    *n = (int)t.size();
    if (rows && carts && vals)
        for (int i = 0; i < (int)t.size() && i < cap; i++)
        {
            rows[i] = t[i].row;
            carts[i] = t[i].cart;
            vals[i] = t[i].val;
        }
    return LIBLE_GPU_OK;
}

int lible_host_shell_norms(int l, int n_prim, const double *exps, const double *coeffs, double *norms)
{
    if (l < 0 || l > kMaxL || n_prim <= 0 || !exps || !coeffs || !norms)
        return LIBLE_GPU_EINVAL;
    std::vector<double> e(exps, exps + n_prim), c(coeffs, coeffs + n_prim), pn;
    for (double x : e)
        pn.push_back(purePrimitiveNorm(l, x));
    auto v = shellNorms(l, e, c, pn);
    std::copy(v.begin(), v.end(), norms);
    return LIBLE_GPU_OK;
}

int lible_host_pair_classes(const char *basis_root, const char *basis, int n_atoms, const int *atomic_nrs,
                            const double *xyz, int units, int use_symm, int *n_classes, int *ls, long long *n_pairs,
                            long long *n_ppairs)
{
    if (!basis_root || !basis || n_atoms <= 0 || !atomic_nrs || !xyz || !n_classes)
        return LIBLE_GPU_EINVAL;
    try
    {
        std::string path = findBasisFile(basis_root, basis);
        std::vector<BasisAtom> atoms;
        for (int a = 0; a < n_atoms; a++)
            atoms.push_back(readBasisAtom(path, atomic_nrs[a]));
        auto shells = constructShells(atoms, coords(n_atoms, xyz, units));
        int lmax = 0;
        for (const auto &s : shells)
            lmax = std::max(lmax, s.l);
        auto byL = [&](int l) {
            std::vector<Shell> v;
            for (const auto &s : shells)
                if (s.l == l)
                    v.push_back(s);
            return v;
        };
        int k = 0;
        for (int la = 0; la <= lmax; la++)
            for (int lb = 0; lb <= (use_symm ? la : lmax); lb++, k++)
            {
                if (ls)
                {
                    PairClass pc = buildPairClass(use_symm != 0, la, lb, byL(la), byL(lb));
                    ls[2 * k] = la;
                    ls[2 * k + 1] = lb;
                    if (n_pairs)
                        n_pairs[k] = (long long)pc.n_pairs;
                    if (n_ppairs)
                        n_ppairs[k] = (long long)pc.n_ppairs;
                }
            }
        *n_classes = k;
        return LIBLE_GPU_OK;
    }
    catch (const EngineError &e)
    {
        return e.code;
    }
    catch (const std::exception &)
    {
        return LIBLE_GPU_EINVAL;
    }
}

int lible_host_boys(int n, double x, double *F)
{
    if (n < 0 || n > kBoysMaxN || !F || !(x >= 0))
        return LIBLE_GPU_EINVAL;
    static const std::vector<double> grid = boysGrid();
    boysHost(n, x, grid, F);
    return LIBLE_GPU_OK;
}

int lible_gpu_create(int device, lible_gpu_ctx **ctx)
{
    if (!ctx)
        return LIBLE_GPU_EINVAL;
    *ctx = nullptr;
    auto *c = new lible_gpu_ctx;
    try
    {
        c->eng = std::make_unique<Engine>(device);
    }
    catch (const EngineError &e)
    {
        delete c;
        return e.code;
    }
    catch (const std::exception &)
    {
        delete c;
        return LIBLE_GPU_EINTERNAL;
    }
    *ctx = c;
    return LIBLE_GPU_OK;
}

int lible_gpu_destroy(lible_gpu_ctx *ctx)
{
    t_errors.erase(ctx);
    delete ctx;
    return LIBLE_GPU_OK;
}

const char *lible_gpu_last_error(const lible_gpu_ctx *ctx)
{
    if (!ctx)
        return "null context";
    const auto it = t_errors.find(ctx);
    return it == t_errors.end() ? "" : it->second.c_str();
}

int lible_gpu_set_structure_named(lible_gpu_ctx *ctx, const char *basis_root, const char *basis,
                                  const char *aux_root, const char *aux_basis, int n_atoms,
                                  const int *atomic_nrs, const double *xyz, int units)
{
    return guard(ctx, [&](Engine &e) {
        if (!basis_root || !basis || n_atoms <= 0 || !atomic_nrs || !xyz)
            throw EngineError(kStatusInvalid, "invalid structure arguments");
        std::string path = findBasisFile(basis_root, basis);
        std::vector<BasisAtom> main;
        for (int a = 0; a < n_atoms; a++)
            main.push_back(readBasisAtom(path, atomic_nrs[a]));
        std::vector<BasisAtom> aux;
        if (aux_basis && aux_basis[0])
        {
            std::string apath = findBasisFile(aux_root ? aux_root : basis_root, aux_basis);
            for (int a = 0; a < n_atoms; a++)
                aux.push_back(readBasisAtom(apath, atomic_nrs[a]));
        }
        ctx->structureChanged();
        e.setStructure(main, (aux_basis && aux_basis[0]) ? &aux : nullptr, coords(n_atoms, xyz, units));
    });
}

int lible_gpu_set_structure(lible_gpu_ctx *ctx, int n_atoms, const int *atomic_nrs, const double *xyz, int units,
                            const int *shells_per_atom, const int *shell_l, const int *shell_nprim,
                            const double *exps, const double *coeffs, const int *aux_shells_per_atom,
                            const int *aux_shell_l, const int *aux_shell_nprim, const double *aux_exps,
                            const double *aux_coeffs)
{
    return guard(ctx, [&](Engine &e) {
        if (n_atoms <= 0 || !atomic_nrs || !xyz || !shells_per_atom || !shell_l || !shell_nprim || !exps || !coeffs)
            throw EngineError(kStatusInvalid, "invalid structure arguments");
        auto main = atomsFromArrays(n_atoms, atomic_nrs, shells_per_atom, shell_l, shell_nprim, exps, coeffs);
        std::vector<BasisAtom> aux;
        if (aux_shells_per_atom)
            aux = atomsFromArrays(n_atoms, atomic_nrs, aux_shells_per_atom, aux_shell_l, aux_shell_nprim, aux_exps,
                                  aux_coeffs);
        ctx->structureChanged();
        e.setStructure(main, aux_shells_per_atom ? &aux : nullptr, coords(n_atoms, xyz, units));
    });
}

int lible_gpu_dims(lible_gpu_ctx *ctx, long long *nao, long long *naux, int *n_atoms, int *max_l)
{
    return guard(ctx, [&](Engine &e) {
        if (nao)
            *nao = (long long)e.nao();
        if (naux)
            *naux = (long long)e.naux();
        if (n_atoms)
            *n_atoms = e.nAtoms();
        if (max_l)
            *max_l = e.maxL();
    });
}

int lible_gpu_eri4(lible_gpu_ctx *ctx, double *out)
{
    return guard(ctx, [&](Engine &e) {
        const size_t n = e.nao();
        DevArray o(out, n * n * n * n, false, e.stream());
        e.eri4(o.ptr);
        o.copyOut();
    });
}

int lible_gpu_eri4_diagonal(lible_gpu_ctx *ctx, double *out)
{
    return guard(ctx, [&](Engine &e) {
        const size_t n = e.nao();
        std::vector<double> h(n * n);
        e.eri4Diagonal(h.data());
        if (isDevice(out))
            cudaCheck(cudaMemcpy(out, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice), "copy");
        else
            std::memcpy(out, h.data(), h.size() * sizeof(double));
    });
}

int lible_gpu_eri3(lible_gpu_ctx *ctx, double *out)
{
    return guard(ctx, [&](Engine &e) {
        if (!e.hasAux())
            throw EngineError(kStatusNoAux, "RI approximation is not enabled!");
        const size_t n = e.nao();
        DevArray o(out, n * n * e.naux(), false, e.stream());
        e.eri3(o.ptr);
        o.copyOut();
    });
}

int lible_gpu_eri2(lible_gpu_ctx *ctx, double *out)
{
    return guard(ctx, [&](Engine &e) {
        if (!e.hasAux())
            throw EngineError(kStatusNoAux, "eri2(): RI approximation is not enabled");
        DevArray o(out, e.naux() * e.naux(), false, e.stream());
        e.eri2(o.ptr);
        o.copyOut();
    });
}

int lible_gpu_eri2_diagonal(lible_gpu_ctx *ctx, double *out)
{
    return guard(ctx, [&](Engine &e) {
        if (!e.hasAux())
            throw EngineError(kStatusNoAux, "eri2Diagonal(): RI approximation is not enabled");
        std::vector<double> h(e.naux());
        e.eri2Diagonal(h.data());
        if (isDevice(out))
            cudaCheck(cudaMemcpy(out, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice), "copy");
        else
            std::memcpy(out, h.data(), h.size() * sizeof(double));
    });
}

int lible_gpu_pair_classes(lible_gpu_ctx *ctx, int use_symm, int *n_classes, int *ls, long long *n_pairs,
                           long long *n_ppairs)
{
    return guard(ctx, [&](Engine &e) {
        auto ci = e.pairClasses(use_symm != 0);
        if (n_classes)
            *n_classes = (int)ci.size();
        for (size_t i = 0; i < ci.size(); i++)
        {
            if (ls)
            {
                ls[2 * i] = ci[i].la;
                ls[2 * i + 1] = ci[i].lb;
            }
            if (n_pairs)
                n_pairs[i] = ci[i].n_pairs;
            if (n_ppairs)
                n_ppairs[i] = ci[i].n_ppairs;
        }
    });
}

int lible_gpu_aux_classes(lible_gpu_ctx *ctx, int *n_classes, int *ls, long long *n_shells)
{
    return guard(ctx, [&](Engine &e) {
        auto ci = e.auxClasses();
        if (n_classes)
            *n_classes = (int)ci.size();
        for (size_t i = 0; i < ci.size(); i++)
        {
            if (ls)
                ls[i] = ci[i].la;
            if (n_shells)
                n_shells[i] = ci[i].n_pairs;
        }
    });
}

static int batch4(lible_gpu_ctx *ctx, int use_symm, int cab, int ccd, long long n, const unsigned *pairs, double *out,
                  bool d1)
{
    return guard(ctx, [&](Engine &e) {
        if (n < 0 || (n > 0 && (!pairs || !out)))
            throw EngineError(kStatusInvalid, "invalid batch arguments");
        auto ci = e.pairClasses(use_symm != 0);
        if (cab < 0 || ccd < 0 || cab >= (int)ci.size() || ccd >= (int)ci.size())
            throw EngineError(kStatusInvalid, "class index out of range");
        const size_t blk = (size_t)nsph(ci[cab].la) * nsph(ci[cab].lb) * nsph(ci[ccd].la) * nsph(ci[ccd].lb);
        DevArray o(out, (size_t)n * blk * (d1 ? 12 : 1), false, e.stream());
        e.eri4Batch(use_symm != 0, cab, ccd, n, pairs, o.ptr, d1);
        o.copyOut();
    });
}

int lible_gpu_eri4_batch(lible_gpu_ctx *ctx, int use_symm, int class_ab, int class_cd, long long n,
                         const unsigned *pairs, double *out)
{
    return batch4(ctx, use_symm, class_ab, class_cd, n, pairs, out, false);
}

int lible_gpu_eri4d1_batch(lible_gpu_ctx *ctx, int use_symm, int class_ab, int class_cd, long long n,
                           const unsigned *pairs, double *out)
{
    return batch4(ctx, use_symm, class_ab, class_cd, n, pairs, out, true);
}

int lible_gpu_eri4_batch_noalloc(lible_gpu_ctx *ctx, int use_symm, int class_ab, int class_cd, long long n,
                                 const unsigned *pairs, double *out)
{
    return guard(ctx, [&](Engine &e) {
        if (n < 0 || (n > 0 && (!pairs || !out)))
            throw EngineError(kStatusInvalid, "invalid batch arguments");
        long long max_pairs = 0;
        uint32_t *scratch = noAllocScratch(&max_pairs);
        if (n > max_pairs)
            throw EngineError(kStatusInvalid, "eri4 batch without allocation: n = " + std::to_string(n) +
                                                  " exceeds the maximum of " + std::to_string(max_pairs) + " pairs");
        if (n > 0 && !isDevice(out))
            throw EngineError(kStatusInvalid, "eri4 batch without allocation: out must be device memory");
        if (n > 0 && isDevice(pairs))
            throw EngineError(kStatusInvalid, "eri4 batch without allocation: pairs must be host memory");
        e.eri4BatchNoAlloc(use_symm != 0, class_ab, class_cd, n, pairs, out, scratch, max_pairs);
    });
}

static int batch3(lible_gpu_ctx *ctx, int use_symm, int cab, int cx, long long n, const unsigned *idx, double *out,
                  bool d1)
{
    return guard(ctx, [&](Engine &e) {
        if (n < 0 || (n > 0 && (!idx || !out)))
            throw EngineError(kStatusInvalid, "invalid batch arguments");
        auto ci = e.pairClasses(use_symm != 0);
        auto xi = e.auxClasses();
        if (cab < 0 || cx < 0 || cab >= (int)ci.size() || cx >= (int)xi.size())
            throw EngineError(kStatusInvalid, "class index out of range");
        const size_t blk = (size_t)nsph(ci[cab].la) * nsph(ci[cab].lb) * nsph(xi[cx].la);
        DevArray o(out, (size_t)n * blk * (d1 ? 9 : 1), false, e.stream());
        e.eri3Batch(use_symm != 0, cab, cx, n, idx, o.ptr, d1);
        o.copyOut();
    });
}

int lible_gpu_eri3_batch(lible_gpu_ctx *ctx, int use_symm, int class_ab, int aux_class, long long n,
                         const unsigned *idx, double *out)
{
    return batch3(ctx, use_symm, class_ab, aux_class, n, idx, out, false);
}

int lible_gpu_eri3d1_batch(lible_gpu_ctx *ctx, int use_symm, int class_ab, int aux_class, long long n,
                           const unsigned *idx, double *out)
{
    return batch3(ctx, use_symm, class_ab, aux_class, n, idx, out, true);
}

static int batch2(lible_gpu_ctx *ctx, int ca, int cb, long long n, const unsigned *idx, double *out, bool d1)
{
    return guard(ctx, [&](Engine &e) {
        if (n < 0 || (n > 0 && (!idx || !out)))
            throw EngineError(kStatusInvalid, "invalid batch arguments");
        auto xi = e.auxClasses();
        if (ca < 0 || cb < 0 || ca >= (int)xi.size() || cb >= (int)xi.size())
            throw EngineError(kStatusInvalid, "class index out of range");
        const size_t blk = (size_t)nsph(xi[ca].la) * nsph(xi[cb].la);
        DevArray o(out, (size_t)n * blk * (d1 ? 6 : 1), false, e.stream());
        e.eri2Batch(ca, cb, n, idx, o.ptr, d1);
        o.copyOut();
    });
}

int lible_gpu_eri2_batch(lible_gpu_ctx *ctx, int a, int b, long long n, const unsigned *idx, double *out)
{
    return batch2(ctx, a, b, n, idx, out, false);
}

int lible_gpu_eri2d1_batch(lible_gpu_ctx *ctx, int a, int b, long long n, const unsigned *idx, double *out)
{
    return batch2(ctx, a, b, n, idx, out, true);
}

static int specialBatch(lible_gpu_ctx *ctx, int kind, int use_symm, int a, int b, long long n, const unsigned *pairs,
                        double *out)
{
    return guard(ctx, [&](Engine &e) {
        if (n < 0 || (n > 0 && (!pairs || !out)))
            throw EngineError(kStatusInvalid, "bad batch arguments");
        if (kind != 0 && !e.hasAux())
            throw EngineError(kStatusNoAux, "RI approximation is not enabled");
        const auto main = e.pairClasses(use_symm != 0);
        const auto aux = kind == 0 ? std::vector<Engine::ClassInfo>{} : e.auxClasses();
        const auto &ca = kind == 2 ? aux : main;
        const auto &cb = kind == 0 ? main : aux;
        if (a < 0 || a >= (int)ca.size() || b < 0 || b >= (int)cb.size())
            throw EngineError(kStatusInvalid, "class index out of range");
        const size_t blk = (size_t)(2 * ca[a].la + 1) * (2 * ca[a].lb + 1) * (2 * cb[b].la + 1) * (2 * cb[b].lb + 1) *
                           (kind == 2 ? 36 : 3);
        DevArray o(out, (size_t)n * blk, false, e.stream());
        e.specialBatch(kind, use_symm != 0, a, b, n, pairs, o.ptr);
        o.copyOut();
    });
}

int lible_gpu_eri4soc_batch(lible_gpu_ctx *ctx, int use_symm, int class_ab, int class_cd, long long n,
                            const unsigned *pairs, double *out)
{
    return specialBatch(ctx, 0, use_symm, class_ab, class_cd, n, pairs, out);
}

int lible_gpu_eri3soc_batch(lible_gpu_ctx *ctx, int use_symm, int class_ab, int aux_class, long long n,
                            const unsigned *pairs, double *out)
{
    return specialBatch(ctx, 1, use_symm, class_ab, aux_class, n, pairs, out);
}

int lible_gpu_eri2d2_batch(lible_gpu_ctx *ctx, int aux_class_a, int aux_class_b, long long n, const unsigned *pairs,
                           double *out)
{
    return specialBatch(ctx, 2, 0, aux_class_a, aux_class_b, n, pairs, out);
}

static JKOptions toOpts(const lible_gpu_jk_opts *o)
{
    JKOptions j;
    if (o)
    {
        j.schwarz = o->schwarz_threshold;
        j.fp32_threshold = o->fp32_threshold;
        j.precision = o->precision;
        j.use_graph = o->use_graph;
    }
    return j;
}

int lible_gpu_jk(lible_gpu_ctx *ctx, const double *D, double *J, double *K, const lible_gpu_jk_opts *opts,
                 lible_gpu_jk_stats *stats)
{
    return guard(ctx, [&](Engine &e) {
        if (!D || !J || !K)
            throw EngineError(kStatusInvalid, "null D/J/K");
        const size_t n2 = (size_t)e.packedSize();
        DevArray d(D, n2, true, e.stream(), &e, 0);
        DevArray j(J, n2, false, e.stream(), &e, 1);
        DevArray k(K, n2, false, e.stream(), &e, 2);
        JKStats st;
        e.jk(d.ptr, j.ptr, k.ptr, toOpts(opts), &st);
        j.copyOut();
        k.copyOut();
        e.checkStatus();
        if (stats)
        {
            stats->n_quartets = st.n_quartets;
            stats->n_fp32 = st.n_fp32;
            stats->n_launches = st.n_launches;
        }
    });
}

int lible_gpu_set_batch(lible_gpu_ctx *ctx, int n_mol, const char *basis_root, const char *const *basis,
                        const int *n_atoms, const int *atomic_nrs, const double *xyz, int units)
{
    return guard(ctx, [&](Engine &e) {
        if (n_mol <= 0 || !basis_root || !basis || !n_atoms || !atomic_nrs || !xyz)
            throw EngineError(kStatusInvalid, "invalid batch arguments");
        std::vector<std::vector<BasisAtom>> mols;
        std::vector<std::vector<std::array<double, 3>>> xyzs;
        std::map<std::string, std::string> paths;
        long long at = 0;
        for (int m = 0; m < n_mol; m++)
        {
            if (!basis[m] || n_atoms[m] <= 0)
                throw EngineError(kStatusInvalid, "invalid batch molecule " + std::to_string(m));
            auto it = paths.find(basis[m]);
            if (it == paths.end())
                it = paths.emplace(basis[m], findBasisFile(basis_root, basis[m])).first;
            std::vector<BasisAtom> atoms;
            for (int a = 0; a < n_atoms[m]; a++)
                atoms.push_back(readBasisAtom(it->second, atomic_nrs[at + a]));
            mols.push_back(std::move(atoms));
            xyzs.push_back(coords(n_atoms[m], xyz + 3 * at, units));
            at += n_atoms[m];
        }
        ctx->structureChanged();
        e.setBatch(mols, xyzs);
    });
}

int lible_gpu_batch_layout(lible_gpu_ctx *ctx, int *n_mol, long long *nao, long long *base, long long *packed)
{
    return guard(ctx, [&](Engine &e) {
        const auto &na = e.molNao(), &mb = e.molBase();
        if (n_mol)
            *n_mol = (int)na.size();
        for (size_t m = 0; m < na.size(); m++)
        {
            if (nao)
                nao[m] = na[m];
            if (base)
                base[m] = mb[m];
        }
        if (packed)
            *packed = e.packedSize();
    });
}

int lible_gpu_jk_profile(lible_gpu_ctx *ctx, const double *D, double *J, double *K, const lible_gpu_jk_opts *opts,
                         int *n, int *ls, int *fp32, double *ms, double *flops, long long *tasks)
{
    return guard(ctx, [&](Engine &e) {
        if (!D || !J || !K || !n)
            throw EngineError(kStatusInvalid, "null argument");
        const size_t n2 = (size_t)e.packedSize();
        DevArray d(D, n2, true, e.stream(), &e, 0);
        DevArray j(J, n2, false, e.stream(), &e, 1);
        DevArray k(K, n2, false, e.stream(), &e, 2);
        auto v = e.jkProfile(d.ptr, j.ptr, k.ptr, toOpts(opts));
        j.copyOut();
        k.copyOut();
        const int cap = *n;
        *n = (int)v.size();
        if (!ls)
            return;
        for (int i = 0; i < std::min(cap, (int)v.size()); i++)
        {
            for (int q = 0; q < 4; q++)
                ls[4 * i + q] = v[i].l[q];
            if (fp32)
                fp32[i] = v[i].fp32;
            if (ms)
                ms[i] = v[i].ms;
            if (flops)
                flops[i] = v[i].flops;
            if (tasks)
                tasks[i] = v[i].tasks;
        }
    });
}

int lible_gpu_set_tune_cache(lible_gpu_ctx *ctx, const char *path)
{
    return guard(ctx, [&](Engine &e) { e.setTuneCache(path ? path : ""); });
}

int lible_gpu_jk_autotune(lible_gpu_ctx *ctx, const double *D, double *J, double *K, const lible_gpu_jk_opts *opts,
                          const char *cache_path, char *summary, int summary_len)
{
    return guard(ctx, [&](Engine &e) {
        if (!D || !J || !K)
            throw EngineError(kStatusInvalid, "null D/J/K");
        const size_t n2 = (size_t)e.packedSize();
        DevArray d(D, n2, true, e.stream(), &e, 0);
        DevArray j(J, n2, false, e.stream(), &e, 1);
        DevArray k(K, n2, false, e.stream(), &e, 2);
        std::string s = e.jkAutotune(d.ptr, j.ptr, k.ptr, toOpts(opts), cache_path ? cache_path : "");
        j.copyOut();
        k.copyOut();
        if (summary && summary_len > 0)
        {
            const size_t c = std::min<size_t>(s.size(), (size_t)summary_len - 1);
            std::memcpy(summary, s.data(), c);
            summary[c] = 0;
        }
    });
}

int lible_gpu_jk_plan(lible_gpu_ctx *ctx, const lible_gpu_jk_opts *opts, lible_gpu_jk_plan_info *info)
{
    return guard(ctx, [&](Engine &e) {
        if (!info)
            throw EngineError(kStatusInvalid, "null info");
        JKPlanInfo p = e.jkPlanInfo(toOpts(opts));
        info->n_quartets = p.n_quartets;
        info->n_fp32 = p.n_fp32;
        info->n_prim_quartets = p.n_prim_quartets;
        info->n_launches = p.n_launches;
        info->flops_fp64 = p.flops_fp64;
        info->flops_fp32 = p.flops_fp32;
    });
}

int lible_gpu_jk_plan_classes(lible_gpu_ctx *ctx, const lible_gpu_jk_opts *opts, int *n, int *ls, long long *n64,
                              long long *n32, double *n_prim, double *flops)
{
    return guard(ctx, [&](Engine &e) {
        if (!n)
            throw EngineError(kStatusInvalid, "null n");
        auto v = e.jkPlanClasses(toOpts(opts));
        *n = (int)v.size();
        if (!ls)
            return;
        for (size_t i = 0; i < v.size(); i++)
        {
            for (int k = 0; k < 4; k++)
                ls[4 * i + k] = v[i].l[k];
            if (n64)
                n64[i] = v[i].n64;
            if (n32)
                n32[i] = v[i].n32;
            if (n_prim)
                n_prim[i] = v[i].prim;
            if (flops)
                flops[i] = v[i].flops;
        }
    });
}

int lible_gpu_stream(lible_gpu_ctx *ctx, void **stream)
{
    return guard(ctx, [&](Engine &e) {
        if (!stream)
            throw EngineError(kStatusInvalid, "null stream");
        *stream = (void *)e.stream();
    });
}

int lible_gpu_fp64_peak(lible_gpu_ctx *ctx, double *dfma, double *dmma)
{
    return guard(ctx, [&](Engine &e) {
        auto p = measureFp64Peak(e.device(), e.stream());
        if (dfma)
            *dfma = p.first;
        if (dmma)
            *dmma = p.second;
    });
}

int lible_gpu_fp32_peak(lible_gpu_ctx *ctx, double *ffma, double *ffma2)
{
    return guard(ctx, [&](Engine &e) {
        auto p = measureFp32Peak(e.device(), e.stream());
        if (ffma)
            *ffma = p.first;
        if (ffma2)
            *ffma2 = p.second;
    });
}

int lible_gpu_check_bounded_wait(lible_gpu_ctx *ctx, int polls)
{
    return guard(ctx, [&](Engine &e) { e.checkBoundedWait(polls); });
}

int lible_gpu_inject_wait_timeout(lible_gpu_ctx *ctx, int polls)
{
    return guard(ctx, [&](Engine &e) { e.injectWaitTimeout(polls); });
}

int lible_gpu_eval_special(lible_gpu_ctx *ctx, int which, int order, long long n, const double *x, double *out)
{
    return guard(ctx, [&](Engine &e) {
        if (n < 0 || (n > 0 && (!x || !out)) || which < 0 || which > 2)
            throw EngineError(kStatusInvalid, "invalid special-function arguments");
        const size_t per = which == 0 ? 1 : (size_t)std::max(order, 0) + 1;
        DevArray xi(const_cast<double *>(x), (size_t)n, true, e.stream());
        DevArray o(out, (size_t)n * per, false, e.stream());
        e.evalSpecial(which, order, n, xi.ptr, o.ptr);
        o.copyOut();
    });
}

int lible_gpu_jk_energy_forward(lible_gpu_ctx *ctx, const double *D, const lible_gpu_jk_opts *opts, double *energy,
                                double *J, double *K)
{
    return guard(ctx, [&](Engine &e) {
        if (!D || !energy)
            throw EngineError(kStatusInvalid, "null D/energy");
        const size_t nn = (size_t)e.packedSize();
        DevArray d(D, nn, true, e.stream(), &e, 0);
        DevArray j(J, nn, false, e.stream(), &e, 1);
        DevArray k(K, nn, false, e.stream(), &e, 2);
        // without caller J / K the context's staging buffers of those slots hold them
        double *jp = j.ptr ? j.ptr : e.staging(1, nn), *kp = k.ptr ? k.ptr : e.staging(2, nn);
        e.jk(d.ptr, jp, kp, toOpts(opts), nullptr);
        std::vector<double> hd(nn), hj(nn), hk(nn);
        cudaCheck(cudaMemcpyAsync(hd.data(), d.ptr, nn * 8, cudaMemcpyDeviceToHost, e.stream()), "D2H");
        cudaCheck(cudaMemcpyAsync(hj.data(), jp, nn * 8, cudaMemcpyDeviceToHost, e.stream()), "D2H");
        cudaCheck(cudaMemcpyAsync(hk.data(), kp, nn * 8, cudaMemcpyDeviceToHost, e.stream()), "D2H");
        cudaCheck(cudaStreamSynchronize(e.stream()), "sync");
        double s = 0.0;
        for (size_t x = 0; x < nn; x++)
            s += hd[x] * (0.5 * hj[x] - 0.25 * hk[x]);
        *energy = s;
        if (J)
            j.copyOut();
        if (K)
            k.copyOut();
        e.checkStatus();
    });
}

int lible_gpu_jk_energy_backward(lible_gpu_ctx *ctx, const double *D, const lible_gpu_jk_opts *opts, double *grad)
{
    return guard(ctx, [&](Engine &e) {
        if (!D || !grad)
            throw EngineError(kStatusInvalid, "null D/grad");
        const size_t n = e.nao();
        DevArray d(D, n * n, true, e.stream());
        DevArray g(grad, 3 * (size_t)e.nAtoms(), false, e.stream());
        e.jkGradient(d.ptr, g.ptr, toOpts(opts).schwarz);
        g.copyOut();
    });
}

int lible_gpu_rij_last_solve(lible_gpu_ctx *ctx, int *method, double *lo, double *hi, int *dropped, double *shift)
{
    if (!ctx)
        return LIBLE_GPU_EINVAL;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    if (shift)
        *shift = ctx->rij_shift;
    if (method)
        *method = ctx->rij_method;
    if (lo)
        *lo = ctx->rij_lo;
    if (hi)
        *hi = ctx->rij_hi;
    if (dropped)
        *dropped = ctx->rij_dropped;
    return LIBLE_GPU_OK;
}

int lible_gpu_ri_contract(lible_gpu_ctx *ctx, const double *D, const double *dcoef, double schwarz_threshold,
                          double *gamma, double *J)
{
    return guard(ctx, [&](Engine &e) {
        if (!e.hasAux())
            throw EngineError(kStatusNoAux, "RI approximation is not enabled");
        const size_t n = e.nao(), na = e.naux();
        DevArray d(D, n * n, true, e.stream());
        DevArray c(dcoef, na, true, e.stream());
        DevArray g(gamma, na, false, e.stream());
        DevArray j(J, n * n, false, e.stream());
        if ((gamma && !D) || (J && !dcoef))
            throw EngineError(kStatusInvalid, "missing input");
        e.riContract(d.ptr, c.ptr, g.ptr, j.ptr, schwarz_threshold);
        if (gamma)
            g.copyOut();
        if (J)
            j.copyOut();
    });
}

int lible_gpu_rij(lible_gpu_ctx *ctx, const double *D, double schwarz_threshold, double *J, double *gamma,
                  double *dcoef)
{
    return guard(ctx, [&](Engine &e) {
        if (!e.hasAux())
            throw EngineError(kStatusNoAux, "RI approximation is not enabled");
        if (!D || !J)
            throw EngineError(kStatusInvalid, "null D/J");
        const size_t n = e.nao(), na = e.naux();
        DevArray d(D, n * n, true, e.stream());
        DevArray j(J, n * n, false, e.stream());
        DevBuf<double> rhs_b(na);
        double *rhs = rhs_b.p;
        // the tensor (naux * nao (nao + 1) / 2 doubles) is built by the first call when it takes at
        // most 60% of the free memory and kept until the structure, the threshold or the mode changes
        if (ctx->t3 && (ctx->t3->schwarz != schwarz_threshold || ctx->rij_cached_mode == 0))
            ctx->t3.reset();
        if (!ctx->t3 && ctx->rij_cached_mode == 1)
        {
            size_t free_b = 0, total_b = 0;
            cudaCheck(cudaMemGetInfo(&free_b, &total_b), "meminfo");
            if (na * CachedT3::rowLength(n) * sizeof(double) <= (size_t)(0.6 * (double)free_b))
            {
                auto t = std::make_unique<CachedT3>();
                buildT3(e, schwarz_threshold, *t);
                ctx->t3 = std::move(t);
            }
        }
        if (ctx->t3)
        {
            t3Gamma(e, *ctx->t3, d.ptr, rhs);
            e.sync();
        }
        else
            e.riContract(d.ptr, nullptr, rhs, nullptr, schwarz_threshold);
        if (gamma)
        {
            e.sync();
            cudaCheck(cudaMemcpy(gamma, rhs, na * 8, isDevice(gamma) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost),
                      "copy");
        }
        solveMetric(e, ctx->metricFactor(e), rhs);
        if (dcoef)
            cudaCheck(cudaMemcpy(dcoef, rhs, na * 8, isDevice(dcoef) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost),
                      "copy");
        if (ctx->t3)
        {
            t3Coulomb(e, *ctx->t3, rhs, j.ptr);
            e.sync();
        }
        else
            e.riContract(nullptr, rhs, nullptr, j.ptr, schwarz_threshold);
        j.copyOut();
    });
}

int lible_gpu_rij_set_cached(lible_gpu_ctx *ctx, int mode)
{
    return guard(ctx, [&](Engine &) {
        if (mode != 0 && mode != 1)
            throw EngineError(kStatusInvalid, "mode must be 0 (evaluate on every call) or 1 (cache when it fits)");
        ctx->rij_cached_mode = mode;
        if (mode == 0)
            ctx->t3.reset();
    });
}

int lible_gpu_one_electron(lible_gpu_ctx *ctx, const double *charges, int n_charges, double *S, double *T,
                           double *V)
{
    return guard(ctx, [&](Engine &e) {
        if (!S && !T && !V)
            throw EngineError(kStatusInvalid, "no output requested");
        if (charges && n_charges < 0)
            throw EngineError(kStatusInvalid, "negative n_charges");
        const size_t n = e.nao();
        DevArray s(S, n * n, false, e.stream()), t(T, n * n, false, e.stream()), v(V, n * n, false, e.stream());
        e.oneElectron(charges, charges ? n_charges : 0, charges == nullptr, s.ptr, t.ptr, v.ptr);
        e.sync();
        s.copyOut();
        t.copyOut();
        v.copyOut();
    });
}

int lible_gpu_one_electron_batch_ex(lible_gpu_ctx *ctx, int use_symm, int class_ab, int op, long long n,
                                    const unsigned *pairs, const double *charges, const double *omegas, int n_charges,
                                    const double *origin, double *out)
{
    return guard(ctx, [&](Engine &e) {
        if (n < 0 || (n > 0 && (!pairs || !out)) || (charges && n_charges < 0))
            throw EngineError(kStatusInvalid, "bad one-electron batch arguments");
        if (op < 0 || op > 14)
            throw EngineError(kStatusInvalid, "bad one-electron operator");
        const auto cls = e.pairClasses(use_symm != 0);
        if (class_ab < 0 || class_ab >= (int)cls.size())
            throw EngineError(kStatusInvalid, "bad class index");
        const int nblk = op == 14 ? 9 : ((op >= 3 && op <= 5) || op == 10) ? 6 : ((op >= 6 && op <= 8) || op >= 11) ? 3 : 1;
        const size_t blk = (size_t)(2 * cls[class_ab].la + 1) * (2 * cls[class_ab].lb + 1) * nblk;
        DevArray o(out, (size_t)n * blk, false, e.stream());
        e.oneElectronBatch(use_symm != 0, class_ab, op, n, pairs, charges, charges ? n_charges : 0, o.ptr, omegas,
                           origin);
        o.copyOut();
    });
}

int lible_gpu_one_electron_batch(lible_gpu_ctx *ctx, int use_symm, int class_ab, int op, long long n,
                                 const unsigned *pairs, const double *charges, int n_charges, double *out)
{
    if (op > 5)
        return fail(ctx, LIBLE_GPU_EINVAL, "ops 6..9 take lible_gpu_one_electron_batch_ex");
    return lible_gpu_one_electron_batch_ex(ctx, use_symm, class_ab, op, n, pairs, charges, nullptr, n_charges,
                                           nullptr, out);
}

namespace
{
    int oneElectronOperator(lible_gpu_ctx *ctx, int op, const double *charges, const double *omegas, int n_charges,
                            const double *origin, double *out)
    {
        return guard(ctx, [&](Engine &e) {
            if (!out || (charges && n_charges < 0))
                throw EngineError(kStatusInvalid, "bad one-electron operator arguments");
            const size_t n = e.nao();
            const int nblk = op == 9 ? 1 : op == 14 ? 9 : 3;
            DevArray o(out, (size_t)nblk * n * n, false, e.stream());
            e.oneElectronOperator(op, charges, charges ? n_charges : 0, omegas, origin, o.ptr);
            o.copyOut();
        });
    }
}

int lible_gpu_dipole_moment(lible_gpu_ctx *ctx, const double *origin, double *out)
{
    return oneElectronOperator(ctx, 6, nullptr, nullptr, 0, origin, out);
}

int lible_gpu_momentum(lible_gpu_ctx *ctx, double *out)
{
    return oneElectronOperator(ctx, 7, nullptr, nullptr, 0, nullptr, out);
}

int lible_gpu_angular_momentum(lible_gpu_ctx *ctx, const double *origin, double *out)
{
    return oneElectronOperator(ctx, 8, nullptr, nullptr, 0, origin, out);
}

int lible_gpu_pvp_integrals(lible_gpu_ctx *ctx, const double *charges, int n_charges, double *out)
{
    return oneElectronOperator(ctx, 14, charges, nullptr, charges ? n_charges : 0, nullptr, out);
}

int lible_gpu_spin_orbit_coupling_1el(lible_gpu_ctx *ctx, double *out)
{
    return oneElectronOperator(ctx, 13, nullptr, nullptr, 0, nullptr, out);
}

int lible_gpu_nuclear_attraction_erf(lible_gpu_ctx *ctx, const double *omegas, double *out)
{
    return oneElectronOperator(ctx, 9, nullptr, omegas, 0, nullptr, out);
}

int lible_gpu_external_charges_erf(lible_gpu_ctx *ctx, const double *charges, const double *omegas, int n_charges,
                                   double *out)
{
    if (!charges || n_charges < 0)
        return fail(ctx, LIBLE_GPU_EINVAL, "null charges");
    return oneElectronOperator(ctx, 9, charges, omegas, n_charges, nullptr, out);
}

int lible_gpu_one_electron_grad(lible_gpu_ctx *ctx, const double *D, const double *W, double *grad)
{
    return guard(ctx, [&](Engine &e) {
        if (!grad)
            throw EngineError(kStatusInvalid, "null grad");
        const size_t n = e.nao();
        DevArray d(D, n * n, true, e.stream()), w(W, n * n, true, e.stream());
        DevArray g(grad, (size_t)e.nAtoms() * 3, false, e.stream());
        e.oneElectronGrad(d.ptr, w.ptr, g.ptr);
        e.sync();
        g.copyOut();
    });
}

int lible_gpu_overlap(lible_gpu_ctx *ctx, double *out)
{
    return lible_gpu_one_electron(ctx, nullptr, 0, out, nullptr, nullptr);
}

int lible_gpu_kinetic_energy(lible_gpu_ctx *ctx, double *out)
{
    return lible_gpu_one_electron(ctx, nullptr, 0, nullptr, out, nullptr);
}

int lible_gpu_nuclear_attraction(lible_gpu_ctx *ctx, double *out)
{
    return lible_gpu_one_electron(ctx, nullptr, 0, nullptr, nullptr, out);
}

int lible_gpu_external_charges(lible_gpu_ctx *ctx, const double *charges, int n_charges, double *out)
{
    if (!charges && n_charges > 0)
        return fail(ctx, LIBLE_GPU_EINVAL, "null charges");
    static const double none[4] = {0, 0, 0, 0};
    return lible_gpu_one_electron(ctx, charges ? charges : none, charges ? n_charges : 0, nullptr, nullptr, out);
}

int lible_gpu_rij_grad(lible_gpu_ctx *ctx, const double *D, double schwarz_threshold, double *grad, double *energy)
{
    return guard(ctx, [&](Engine &e) {
        if (!e.hasAux())
            throw EngineError(kStatusNoAux, "RI approximation is not enabled");
        if (!D || !grad)
            throw EngineError(kStatusInvalid, "null D/grad");
        const size_t n = e.nao(), na = e.naux();
        DevArray d(D, n * n, true, e.stream());
        DevArray g(grad, (size_t)e.nAtoms() * 3, false, e.stream());
        DevBuf<double> rhs(na);
        e.riContract(d.ptr, nullptr, rhs.p, nullptr, schwarz_threshold);
        std::vector<double> gamma(na), dc(na);
        cudaCheck(cudaMemcpy(gamma.data(), rhs.p, na * 8, cudaMemcpyDeviceToHost), "copy");
        solveMetric(e, ctx->metricFactor(e), rhs.p);
        e.riGradient(d.ptr, rhs.p, g.ptr, schwarz_threshold);
        g.copyOut();
        if (energy)
        {
            cudaCheck(cudaMemcpy(dc.data(), rhs.p, na * 8, cudaMemcpyDeviceToHost), "copy");
            double s = 0.0;
            for (size_t i = 0; i < na; i++)
                s += gamma[i] * dc[i];
            *energy = 0.5 * s;
        }
    });
}

int lible_gpu_rik(lible_gpu_ctx *ctx, const double *D, const double *C, long long n_occ, double schwarz_threshold,
                  double *K, lible_gpu_rik_info *info)
{
    return guard(ctx, [&](Engine &e) {
        if (!e.hasAux())
            throw EngineError(kStatusNoAux, "RI approximation is not enabled");
        if (!K || (!D && !C))
            throw EngineError(kStatusInvalid, "null K, or neither D nor C given");
        if (C && n_occ < 0)
            throw EngineError(kStatusInvalid, "negative n_occ");
        const size_t n = e.nao();
        DevArray k(K, n * n, false, e.stream());
        cudaCheck(cudaMemsetAsync(k.ptr, 0, n * n * sizeof(double), e.stream()), "memset");
        const MetricFactor &mf = ctx->metricFactor(e);
        BlasHandle &bh = ctx->blasHandle(e);
        RIKStats st;
        // one block of (mn|P): a quarter of the free device memory left after Z, 256 MiB .. 16 GiB
        size_t free_b = 0, total_b = 0;
        cudaCheck(cudaMemGetInfo(&free_b, &total_b), "meminfo");
        const size_t z_bytes = e.naux() * n * (size_t)std::max<long long>(n_occ > 0 ? n_occ : (long long)n, 1) * 8;
        const size_t avail = free_b > z_bytes ? free_b - z_bytes : 0;
        const size_t block_bytes = std::min<size_t>(size_t(16) << 30, std::max<size_t>(size_t(256) << 20, avail / 4));
        long long n_pos = n_occ, n_neg = 0;
        // the fitted tensor (naux * nao^2 doubles) is built once and kept when it takes at most
        // 60% of the free memory after Z; otherwise every call streams blocks of integrals
        const size_t fit_bytes = e.naux() * n * n * sizeof(double);
        if (ctx->fitted && ctx->fitted->schwarz != schwarz_threshold)
            ctx->fitted.reset();
        if (ctx->rik_fitted_mode == 0)
            ctx->fitted.reset();
        if (!ctx->fitted && ctx->rik_fitted_mode == 1 && fit_bytes <= (size_t)(0.6 * (double)avail))
        {
            auto ft = std::make_unique<FittedTensor>();
            buildFitted(e, bh, mf, schwarz_threshold, *ft);
            st.t_ints += ft->t_build;
            st.n_blocks += 1;
            ctx->fitted = std::move(ft);
        }
        const FittedTensor *ft = ctx->fitted.get();
        auto exchange = [&](const double *c, long long occ, double sign) {
            if (ft)
                riExchangeFitted(e, bh, *ft, c, occ, sign, k.ptr, &st);
            else
                riExchange(e, bh, mf, c, occ, schwarz_threshold, sign, k.ptr, block_bytes, &st);
        };
        if (C)
        {
            DevArray c(C, n * (size_t)std::max<long long>(n_occ, 1), true, e.stream());
            exchange(c.ptr, n_occ, 1.0);
        }
        else
        {
            DevArray d(D, n * n, true, e.stream());
            DevBuf<double> cp, cm;
            splitDensity(e, d.ptr, (long long)n, cp, n_pos, cm, n_neg);
            exchange(cp.p, n_pos, 1.0);
            exchange(cm.p, n_neg, -1.0);
        }
        mirrorUpper(k.ptr, (long long)n, e.stream());
        e.sync();
        k.copyOut();
        if (info)
        {
            info->n_pos = n_pos;
            info->n_neg = n_neg;
            info->n_blocks = st.n_blocks;
            info->t_ints = st.t_ints;
            info->t_gemm = st.t_gemm;
            info->t_solve = st.t_solve;
            info->t_syrk = st.t_syrk;
            info->flops_gemm = st.flops_gemm;
            info->flops_solve = st.flops_solve;
            info->flops_syrk = st.flops_syrk;
            info->fitted = ft ? 1 : 0;
        }
    });
}

int lible_gpu_rik_set_fitted(lible_gpu_ctx *ctx, int mode)
{
    return guard(ctx, [&](Engine &) {
        if (mode != 0 && mode != 1)
            throw EngineError(kStatusInvalid, "mode must be 0 (stream) or 1 (cache when it fits)");
        ctx->rik_fitted_mode = mode;
        if (mode == 0)
            ctx->fitted.reset();
    });
}

} // extern "C"
