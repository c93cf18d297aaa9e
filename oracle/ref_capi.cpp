// Test infrastructure only: a flat C ABI over the reference's own `lible::ints` code, compiled
// from the reference sources by oracle/Makefile into oracle/_ref/liblible_ref.so.
//
// It exists so that the Python tests and the reference arm of bench.py can call the unmodified
// reference path.  Nothing in the product links or loads it.
//
// What it wraps (reference paths are relative to the reference project root):
//   Structure ctors                     src/lible/ints/structure.hpp:18-62
//   eri4 / eri4Diagonal                 src/lible/ints/twoel/eri4.cpp:38-95, 152-174
//   eri3                                src/lible/ints/twoel/eri3.cpp:7-48
//   eri2 / eri2Diagonal                 src/lible/ints/twoel/eri2.cpp:27-96
//   ERI4Kernel / ERI3Kernel / ERI2Kernel and the D1 kernels   src/lible/ints/twoel/eri_kernels.hpp:60-169
//   shellPairData / shellDataAux        src/lible/ints/shell_pair_data.cpp:280-309
//   the kernel-API golden sums          test/tests_ints.cpp:873-1053
// The reference has no J/K, gradient or RI-J driver.  ref_jk, ref_jk_grad and ref_rij_* below
// digest the reference's own ERI4Kernel / ERI4D1Kernel / ERI3Kernel batches on the CPU; that
// digestion (Schwarz screening, 8-fold symmetry weights) is this project's restatement and is
// the CPU baseline for those paths.

#include <lible/ints/ints.hpp>
#include <lible/ints/twoel/eri_kernels.hpp>

#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace lints = lible::ints;

namespace
{
    thread_local std::string g_err;

    struct RefStructure
    {
        std::unique_ptr<lints::Structure> s;
    };

    template <class F>
    int guarded(F &&f)
    {
        try
        {
            f();
            return 0;
        }
        catch (const std::exception &e)
        {
            g_err = e.what();
            return 1;
        }
    }

    lints::basis_atoms_t makeBasisAtoms(int n_atoms, const int *Z, const int *nshell_per_atom,
                                        const int *shell_l, const int *shell_nprim,
                                        const double *exps, const double *coeffs)
    {
        lints::basis_atoms_t atoms;
        size_t ish = 0, iprim = 0;
        for (int a = 0; a < n_atoms; a++)
        {
            lints::BasisAtom atom;
            atom.atomic_nr_ = Z[a];
            for (int k = 0; k < nshell_per_atom[a]; k++, ish++)
            {
                lints::BasisShell sh;
                sh.l_ = shell_l[ish];
                for (int p = 0; p < shell_nprim[ish]; p++, iprim++)
                {
                    sh.exps_.push_back(exps[iprim]);
                    sh.coeffs_.push_back(coeffs[iprim]);
                }
                atom.basis_shells_.push_back(sh);
            }
            atoms.push_back(atom);
        }
        return atoms;
    }

    // Shell-level degeneracy factor of a unique quartet (1/2 for a==b, c==d, ab==cd).
    inline double quartetWeight(const lints::ShellPairData &ab, size_t i, const lints::ShellPairData &cd,
                                size_t j, bool same_class)
    {
        double f = 1.0;
        if (ab.shell_idxs_[2 * i] == ab.shell_idxs_[2 * i + 1])
            f *= 0.5;
        if (cd.shell_idxs_[2 * j] == cd.shell_idxs_[2 * j + 1])
            f *= 0.5;
        if (same_class && i == j)
            f *= 0.5;
        return f;
    }

    // Schwarz factor per shell pair: max over the pair's functions of sqrt|(mn|mn)|.
    std::vector<double> schwarzFactors(const lints::ShellPairData &sp)
    {
        std::vector<double> q(sp.n_pairs_, 0.0);
        lints::ERI4Kernel kern(sp, sp);
        int na = lints::numSphericals(sp.la_), nb = lints::numSphericals(sp.lb_);
#pragma omp parallel for schedule(dynamic)
        for (size_t i = 0; i < sp.n_pairs_; i++)
        {
            lible::vec4d b = kern(i, i, sp, sp);
            double m = 0;
            for (int x = 0; x < na; x++)
                for (int y = 0; y < nb; y++)
                    m = std::max(m, std::fabs(b(x, y, x, y)));
            q[i] = std::sqrt(m);
        }
        return q;
    }
}

extern "C" {

const char *ref_last_error() { return g_err.c_str(); }

void ref_set_threads(int n)
{
    if (n > 0)
        omp_set_num_threads(n);
}

int ref_max_threads() { return omp_get_max_threads(); }

// Structure from named basis sets read from `main_dir` / `aux_dir` (reference text format and
// directory layout).  Coordinates in Angstrom, as the reference's Structure expects.
void *ref_structure_named(const char *main_dir, const char *aux_dir, const char *basis,
                          const char *aux_basis, int n_atoms, const int *Z, const double *xyz_ang)
{
    RefStructure *r = nullptr;
    int rc = guarded([&]
    {
        lints::BasisPaths::setMainBasisSetsPath(main_dir);
        if (aux_dir)
            lints::BasisPaths::setAuxBasisSetsPath(aux_dir);
        std::vector<int> z(Z, Z + n_atoms);
        std::vector<std::array<double, 3>> c(n_atoms);
        for (int a = 0; a < n_atoms; a++)
            c[a] = {xyz_ang[3 * a], xyz_ang[3 * a + 1], xyz_ang[3 * a + 2]};
        r = new RefStructure;
        if (aux_basis && aux_basis[0])
            r->s = std::make_unique<lints::Structure>(std::string(basis), std::string(aux_basis), z, c);
        else
            r->s = std::make_unique<lints::Structure>(std::string(basis), z, c);
    });
    if (rc)
    {
        delete r;
        return nullptr;
    }
    return r;
}

// Structure from explicit per-atom shells (the reference's basis_atoms_t path).
void *ref_structure_custom(int n_atoms, const int *Z, const double *xyz_ang,
                           const int *nsh, const int *sh_l, const int *sh_np, const double *exps,
                           const double *coeffs, const int *aux_nsh, const int *aux_l,
                           const int *aux_np, const double *aux_exps, const double *aux_coeffs)
{
    RefStructure *r = nullptr;
    int rc = guarded([&]
    {
        std::vector<int> z(Z, Z + n_atoms);
        std::vector<std::array<double, 3>> c(n_atoms);
        for (int a = 0; a < n_atoms; a++)
            c[a] = {xyz_ang[3 * a], xyz_ang[3 * a + 1], xyz_ang[3 * a + 2]};
        lints::basis_atoms_t main = makeBasisAtoms(n_atoms, Z, nsh, sh_l, sh_np, exps, coeffs);
        r = new RefStructure;
        if (aux_nsh)
        {
            lints::basis_atoms_t aux = makeBasisAtoms(n_atoms, Z, aux_nsh, aux_l, aux_np, aux_exps,
                                                      aux_coeffs);
            r->s = std::make_unique<lints::Structure>(main, aux, z, c);
        }
        else
            r->s = std::make_unique<lints::Structure>(main, z, c);
    });
    if (rc)
    {
        delete r;
        return nullptr;
    }
    return r;
}

void ref_structure_free(void *h) { delete static_cast<RefStructure *>(h); }

long ref_dim_ao(void *h) { return (long)static_cast<RefStructure *>(h)->s->getDimAO(); }
long ref_dim_ao_aux(void *h) { return (long)static_cast<RefStructure *>(h)->s->getDimAOAux(); }
long ref_n_atoms(void *h) { return (long)static_cast<RefStructure *>(h)->s->getNAtoms(); }

int ref_eri4(void *h, double *out)
{
    return guarded([&]
    {
        lible::vec4d v = lints::eri4(*static_cast<RefStructure *>(h)->s);
        std::memcpy(out, v.memptr(), v.size() * sizeof(double));
    });
}

int ref_eri4_diagonal(void *h, double *out)
{
    return guarded([&]
    {
        lible::vec2d v = lints::eri4Diagonal(*static_cast<RefStructure *>(h)->s);
        std::memcpy(out, v.memptr(), v.size() * sizeof(double));
    });
}

int ref_eri3(void *h, double *out)
{
    return guarded([&]
    {
        lible::vec3d v = lints::eri3(*static_cast<RefStructure *>(h)->s);
        std::memcpy(out, v.memptr(), v.size() * sizeof(double));
    });
}

int ref_eri2(void *h, double *out)
{
    return guarded([&]
    {
        lible::vec2d v = lints::eri2(*static_cast<RefStructure *>(h)->s);
        std::memcpy(out, v.memptr(), v.size() * sizeof(double));
    });
}

// All ERI4SOCKernel / ERI3SOCKernel batches of one class pair, [n_ab][n_cd][3][block]
// (src/lible/ints/twoel/eri_kernels.hpp:187-223).
int ref_eri4soc_class(void *h, int use_symm, int iab, int icd, double *out)
{
    return guarded([&]
    {
        auto sp = lints::shellPairData(use_symm != 0, *static_cast<RefStructure *>(h)->s);
        const auto &ab = sp.at(iab);
        const auto &cd = sp.at(icd);
        lints::ERI4SOCKernel k(ab, cd);
        size_t blk = lints::numSphericals(ab.la_) * lints::numSphericals(ab.lb_) *
                     lints::numSphericals(cd.la_) * lints::numSphericals(cd.lb_);
#pragma omp parallel for schedule(dynamic)
        for (size_t i = 0; i < ab.n_pairs_; i++)
            for (size_t j = 0; j < cd.n_pairs_; j++)
            {
                auto b = k(i, j, ab, cd);
                for (int x = 0; x < 3; x++)
                    std::memcpy(out + ((i * cd.n_pairs_ + j) * 3 + x) * blk, b[x].memptr(), blk * sizeof(double));
            }
    });
}

int ref_eri3soc_class(void *h, int use_symm, int iab, int ic, double *out)
{
    return guarded([&]
    {
        auto &S = *static_cast<RefStructure *>(h)->s;
        auto sp = lints::shellPairData(use_symm != 0, S);
        auto sh = lints::shellDataAux(S);
        const auto &ab = sp.at(iab);
        const auto &c = sh.at(ic);
        lints::ERI3SOCKernel k(ab, c);
        size_t blk = lints::numSphericals(ab.la_) * lints::numSphericals(ab.lb_) * lints::numSphericals(c.l_);
#pragma omp parallel for schedule(dynamic)
        for (size_t i = 0; i < ab.n_pairs_; i++)
            for (size_t j = 0; j < c.n_shells_; j++)
            {
                auto b = k(i, j, ab, c);
                for (int x = 0; x < 3; x++)
                    std::memcpy(out + ((i * c.n_shells_ + j) * 3 + x) * blk, b[x].memptr(), blk * sizeof(double));
            }
    });
}

// All ERI2D2Kernel batches of one auxiliary class pair, [n_a][n_b][6][6][Sa Sb]
// (eri_kernels.hpp:171-185).
int ref_eri2d2_class(void *h, int ia, int ib, double *out)
{
    return guarded([&]
    {
        auto sh = lints::shellDataAux(*static_cast<RefStructure *>(h)->s);
        const auto &a = sh.at(ia);
        const auto &b = sh.at(ib);
        lints::ERI2D2Kernel k(a, b);
        size_t blk = lints::numSphericals(a.l_) * lints::numSphericals(b.l_);
#pragma omp parallel for schedule(dynamic)
        for (size_t i = 0; i < a.n_shells_; i++)
            for (size_t j = 0; j < b.n_shells_; j++)
            {
                auto r = k(i, j, a, b);
                for (int x = 0; x < 6; x++)
                    for (int y = 0; y < 6; y++)
                        std::memcpy(out + (((i * b.n_shells_ + j) * 6 + x) * 6 + y) * blk, r[x][y].memptr(),
                                    blk * sizeof(double));
            }
    });
}

// The reference's per-pair one-electron kernels for every pair of one class, [n_pairs][blocks][Sa Sb]:
// op 0 overlapKernel, 1 kineticEnergyKernel, 2 externalChargesKernel, 3 overlapD1Kernel,
// 4 kineticEnergyD1Kernel, 5 externalChargesD1Kernel (oneelints.cpp:57-789).
int ref_one_electron_class(void *h, int use_symm, int iab, int op, const double *charges, int n_charges, double *out)
{
    return guarded([&]
    {
        auto sp = lints::shellPairData(use_symm != 0, *static_cast<RefStructure *>(h)->s);
        const auto &ab = sp.at(iab);
        std::vector<std::array<double, 4>> q(n_charges);
        for (int i = 0; i < n_charges; i++)
            q[i] = {charges[4 * i], charges[4 * i + 1], charges[4 * i + 2], charges[4 * i + 3]};
        const int lab = ab.la_ + ab.lb_;
        lints::BoysGrid grid(op == 5 ? lab + 1 : lab);
        size_t blk = lints::numSphericals(ab.la_) * lints::numSphericals(ab.lb_);
        const int nb = op >= 3 ? 6 : 1;
        for (size_t i = 0; i < ab.n_pairs_; i++)
        {
            double *o = out + i * nb * blk;
            if (op < 3)
            {
                lible::vec2d v = op == 0 ? lints::overlapKernel(i, ab)
                                 : op == 1 ? lints::kineticEnergyKernel(i, ab)
                                           : lints::externalChargesKernel(i, q, grid, ab);
                std::memcpy(o, v.memptr(), blk * sizeof(double));
            }
            else
            {
                std::array<lible::vec2d, 6> v = op == 3 ? lints::overlapD1Kernel(i, ab)
                                                : op == 4 ? lints::kineticEnergyD1Kernel(i, ab)
                                                          : lints::externalChargesD1Kernel(i, q, grid, ab);
                for (int d = 0; d < 6; d++)
                    std::memcpy(o + d * blk, v[d].memptr(), blk * sizeof(double));
            }
        }
    });
}

// One-electron integrals of the reference (src/lible/ints/oneelints.cpp): 0 overlap, 1 kinetic
// energy, 2 nuclear attraction, 3 external point charges (charges [n][4] x, y, z (bohr), q).
int ref_one_electron(void *h, int which, const double *charges, int n_charges, double *out)
{
    return guarded([&]
    {
        const lints::Structure &st = *static_cast<RefStructure *>(h)->s;
        lible::vec2d v;
        if (which == 0)
            v = lints::overlap(st);
        else if (which == 1)
            v = lints::kineticEnergy(st);
        else if (which == 2)
            v = lints::nuclearAttraction(st);
        else
        {
            std::vector<std::array<double, 4>> q(n_charges);
            for (int i = 0; i < n_charges; i++)
                q[i] = {charges[4 * i], charges[4 * i + 1], charges[4 * i + 2], charges[4 * i + 3]};
            v = lints::externalCharges(q, st);
        }
        std::memcpy(out, v.memptr(), v.size() * sizeof(double));
    });
}

// The reference's remaining per-pair one-electron kernels for every pair of one class:
// op 6 dipoleMomentKernel, 7 momentumKernel, 8 angularMomentumKernel ([n_pairs][3][Sa Sb]; origin
// for 6 and 8), 9 externalChargesErfKernel ([n_pairs][Sa Sb]; one omega per charge),
// 10 externalChargesErfD1Kernel ([n_pairs][6][Sa Sb]), 11 externalChargesOperatorD1Kernel and
// 12 externalChargesOperatorErfD1Kernel ([n_pairs][n_charges][3][Sa Sb]), 13
// potentialAtExternalChargesKernel and 14 potentialAtExternalChargesErfKernel
// ([n_pairs][n_charges][Sa Sb]), 15 spinOrbitCoupling1ElKernel ([n_pairs][3][Sa Sb]), 16 pVpKernel
// ([n_pairs][9][Sa Sb]) (oneelints.cpp:
// 379-473, 587-680, 791-1086, 1209-1316, 1513-1577, 1617-1701, 1844-2060).
int ref_one_electron_class_ex(void *h, int use_symm, int iab, int op, const double *charges, const double *omegas,
                              int n_charges, const double *origin, double *out)
{
    return guarded([&]
    {
        auto sp = lints::shellPairData(use_symm != 0, *static_cast<RefStructure *>(h)->s);
        const auto &ab = sp.at(iab);
        std::vector<std::array<double, 4>> q(n_charges);
        for (int i = 0; i < n_charges; i++)
            q[i] = {charges[4 * i], charges[4 * i + 1], charges[4 * i + 2], charges[4 * i + 3]};
        std::vector<double> w(omegas ? omegas : charges, omegas ? omegas + n_charges : charges);
        const std::array<double, 3> o = origin ? std::array<double, 3>{origin[0], origin[1], origin[2]}
                                               : std::array<double, 3>{0, 0, 0};
        const bool d1 = op == 10 || op == 11 || op == 12 || op == 15;
        lints::BoysGrid grid(ab.la_ + ab.lb_ + (op == 16 ? 2 : d1 ? 1 : 0));
        const size_t blk = lints::numSphericals(ab.la_) * lints::numSphericals(ab.lb_);
        const size_t nq = (size_t)n_charges;
        const size_t nb = op == 9    ? 1
                          : op == 10 ? 6
                          : op == 16 ? 9
                          : (op == 11 || op == 12) ? 3 * nq
                          : (op == 13 || op == 14) ? nq
                                                   : 3;
        for (size_t i = 0; i < ab.n_pairs_; i++)
        {
            double *dst = out + i * nb * blk;
            if (op == 9)
            {
                lible::vec2d v = lints::externalChargesErfKernel(i, q, w, grid, ab);
                std::memcpy(dst, v.memptr(), blk * sizeof(double));
                continue;
            }
            if (op == 10)
            {
                std::array<lible::vec2d, 6> v = lints::externalChargesErfD1Kernel(i, q, w, grid, ab);
                for (int d = 0; d < 6; d++)
                    std::memcpy(dst + d * blk, v[d].memptr(), blk * sizeof(double));
                continue;
            }
            if (op == 11 || op == 12)
            {
                std::vector<std::array<lible::vec2d, 3>> v =
                    op == 11 ? lints::externalChargesOperatorD1Kernel(i, q, grid, ab)
                             : lints::externalChargesOperatorErfD1Kernel(i, q, w, grid, ab);
                for (size_t c = 0; c < nq; c++)
                    for (int d = 0; d < 3; d++)
                        std::memcpy(dst + (3 * c + d) * blk, v[c][d].memptr(), blk * sizeof(double));
                continue;
            }
            if (op == 16)
            {
                lible::arr2d<lible::vec2d, 3, 3> v = lints::pVpKernel(i, q, grid, ab);
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++)
                        std::memcpy(dst + (3 * a + b) * blk, v[a][b].memptr(), blk * sizeof(double));
                continue;
            }
            if (op == 15)
            {
                std::array<lible::vec2d, 3> v = lints::spinOrbitCoupling1ElKernel(i, q, grid, ab);
                for (int d = 0; d < 3; d++)
                    std::memcpy(dst + d * blk, v[d].memptr(), blk * sizeof(double));
                continue;
            }
            if (op >= 13)
            {
                std::vector<lible::vec2d> v = op == 13 ? lints::potentialAtExternalChargesKernel(i, q, grid, ab)
                                                       : lints::potentialAtExternalChargesErfKernel(i, q, w, grid, ab);
                for (size_t c = 0; c < nq; c++)
                    std::memcpy(dst + c * blk, v[c].memptr(), blk * sizeof(double));
                continue;
            }
            std::array<lible::vec2d, 3> v = op == 6 ? lints::dipoleMomentKernel(i, o, ab)
                                            : op == 7 ? lints::momentumKernel(i, ab)
                                                      : lints::angularMomentumKernel(i, o, ab);
            for (int d = 0; d < 3; d++)
                std::memcpy(dst + d * blk, v[d].memptr(), blk * sizeof(double));
        }
    });
}

// The reference's whole-matrix drivers: 4 dipoleMoment, 5 momentum, 6 angularMomentum, 9
// spinOrbitCoupling1El ([3][nao][nao]; origin for 4 and 6), 7 nuclearAttractionErf (one omega per
// atom), 8 externalChargesErf (one omega per charge) (oneelints.cpp:475-505, 1122-1162, 1164-1207,
// 1477-1511, 1579-1615, 1746-1791).
int ref_one_electron_ex(void *h, int which, const double *charges, const double *omegas, int n_charges,
                        const double *origin, double *out)
{
    return guarded([&]
    {
        const lints::Structure &st = *static_cast<RefStructure *>(h)->s;
        const std::array<double, 3> o = origin ? std::array<double, 3>{origin[0], origin[1], origin[2]}
                                               : std::array<double, 3>{0, 0, 0};
        if ((which >= 4 && which <= 6) || which == 9)
        {
            std::array<lible::vec2d, 3> v = which == 4   ? lints::dipoleMoment(o, st)
                                            : which == 5 ? lints::momentum(st)
                                            : which == 6 ? lints::angularMomentum(o, st)
                                                         : lints::spinOrbitCoupling1El(st);
            const size_t n = v[0].size();
            for (int d = 0; d < 3; d++)
                std::memcpy(out + d * n, v[d].memptr(), n * sizeof(double));
            return;
        }
        lible::vec2d v;
        if (which == 7)
            v = lints::nuclearAttractionErf(st, std::vector<double>(omegas, omegas + st.getNAtoms()));
        else
        {
            std::vector<std::array<double, 4>> q(n_charges);
            for (int i = 0; i < n_charges; i++)
                q[i] = {charges[4 * i], charges[4 * i + 1], charges[4 * i + 2], charges[4 * i + 3]};
            v = lints::externalChargesErf(q, std::vector<double>(omegas, omegas + n_charges), st);
        }
        std::memcpy(out, v.memptr(), v.size() * sizeof(double));
    });
}

int ref_eri2_diagonal(void *h, double *out)
{
    return guarded([&]
    {
        std::vector<double> v = lints::eri2Diagonal(*static_cast<RefStructure *>(h)->s);
        std::memcpy(out, v.data(), v.size() * sizeof(double));
    });
}

// Number of shell-pair classes and their sizes for shellPairData(use_symm).
int ref_pair_classes(void *h, int use_symm, int *n_classes, int *ls, long *n_pairs, long *n_ppairs)
{
    return guarded([&]
    {
        auto sp = lints::shellPairData(use_symm != 0, *static_cast<RefStructure *>(h)->s);
        *n_classes = (int)sp.size();
        if (ls)
            for (size_t i = 0; i < sp.size(); i++)
            {
                ls[2 * i] = sp[i].la_;
                ls[2 * i + 1] = sp[i].lb_;
                n_pairs[i] = (long)sp[i].n_pairs_;
                n_ppairs[i] = (long)sp[i].n_ppairs_;
            }
    });
}

// Pair data of one class: exps/coeffs [2*n_ppairs], coords [6*n_pairs], nrs_ppairs [n_pairs],
// offsets_sph [2*n_pairs], shell_idxs [2*n_pairs], atomic_idxs [2*n_pairs], norms.
int ref_pair_data(void *h, int use_symm, int iclass, double *exps, double *coeffs, double *coords,
                  long *nrs_ppairs, long *offsets_sph, long *shell_idxs, long *atomic_idxs)
{
    return guarded([&]
    {
        auto sp = lints::shellPairData(use_symm != 0, *static_cast<RefStructure *>(h)->s);
        const auto &d = sp.at(iclass);
        std::copy(d.exps_.begin(), d.exps_.end(), exps);
        std::copy(d.coeffs_.begin(), d.coeffs_.end(), coeffs);
        std::copy(d.coords_.begin(), d.coords_.end(), coords);
        for (size_t i = 0; i < d.n_pairs_; i++)
        {
            nrs_ppairs[i] = (long)d.nrs_ppairs_[i];
            for (int k = 0; k < 2; k++)
            {
                offsets_sph[2 * i + k] = (long)d.offsets_sph_[2 * i + k];
                shell_idxs[2 * i + k] = (long)d.shell_idxs_[2 * i + k];
                atomic_idxs[2 * i + k] = (long)d.atomic_idxs_[2 * i + k];
            }
        }
    });
}

// All ERI4Kernel batches of one class pair, [n_ab][n_cd][Sa Sb Sc Sd] row-major.
int ref_eri4_class(void *h, int use_symm, int iab, int icd, double *out)
{
    return guarded([&]
    {
        auto sp = lints::shellPairData(use_symm != 0, *static_cast<RefStructure *>(h)->s);
        const auto &ab = sp.at(iab);
        const auto &cd = sp.at(icd);
        lints::ERI4Kernel k(ab, cd);
        size_t blk = lints::numSphericals(ab.la_) * lints::numSphericals(ab.lb_) *
                     lints::numSphericals(cd.la_) * lints::numSphericals(cd.lb_);
#pragma omp parallel for schedule(dynamic)
        for (size_t i = 0; i < ab.n_pairs_; i++)
            for (size_t j = 0; j < cd.n_pairs_; j++)
            {
                lible::vec4d b = k(i, j, ab, cd);
                std::memcpy(out + (i * cd.n_pairs_ + j) * blk, b.memptr(), blk * sizeof(double));
            }
    });
}

// All ERI4D1Kernel batches of one class pair, [n_ab][n_cd][12][Sa Sb Sc Sd].
int ref_eri4d1_class(void *h, int use_symm, int iab, int icd, double *out)
{
    return guarded([&]
    {
        auto sp = lints::shellPairData(use_symm != 0, *static_cast<RefStructure *>(h)->s);
        const auto &ab = sp.at(iab);
        const auto &cd = sp.at(icd);
        lints::ERI4D1Kernel k(ab, cd);
        size_t blk = lints::numSphericals(ab.la_) * lints::numSphericals(ab.lb_) *
                     lints::numSphericals(cd.la_) * lints::numSphericals(cd.lb_);
#pragma omp parallel for schedule(dynamic)
        for (size_t i = 0; i < ab.n_pairs_; i++)
            for (size_t j = 0; j < cd.n_pairs_; j++)
            {
                auto b = k(i, j, ab, cd);
                for (int x = 0; x < 12; x++)
                    std::memcpy(out + ((i * cd.n_pairs_ + j) * 12 + x) * blk, b[x].memptr(),
                                blk * sizeof(double));
            }
    });
}

// All ERI3Kernel batches for main pair class iab and aux shell class ic, [n_ab][n_c][Sa Sb Sc].
int ref_eri3_class(void *h, int use_symm, int iab, int ic, double *out)
{
    return guarded([&]
    {
        auto &S = *static_cast<RefStructure *>(h)->s;
        auto sp = lints::shellPairData(use_symm != 0, S);
        auto sh = lints::shellDataAux(S);
        const auto &ab = sp.at(iab);
        const auto &c = sh.at(ic);
        lints::ERI3Kernel k(ab, c);
        size_t blk = lints::numSphericals(ab.la_) * lints::numSphericals(ab.lb_) *
                     lints::numSphericals(c.l_);
#pragma omp parallel for schedule(dynamic)
        for (size_t i = 0; i < ab.n_pairs_; i++)
            for (size_t j = 0; j < c.n_shells_; j++)
            {
                lible::vec3d b = k(i, j, ab, c);
                std::memcpy(out + (i * c.n_shells_ + j) * blk, b.memptr(), blk * sizeof(double));
            }
    });
}

// All ERI3D1Kernel batches, [n_ab][n_c][9][Sa Sb Sc].
int ref_eri3d1_class(void *h, int use_symm, int iab, int ic, double *out)
{
    return guarded([&]
    {
        auto &S = *static_cast<RefStructure *>(h)->s;
        auto sp = lints::shellPairData(use_symm != 0, S);
        auto sh = lints::shellDataAux(S);
        const auto &ab = sp.at(iab);
        const auto &c = sh.at(ic);
        lints::ERI3D1Kernel k(ab, c);
        size_t blk = lints::numSphericals(ab.la_) * lints::numSphericals(ab.lb_) *
                     lints::numSphericals(c.l_);
#pragma omp parallel for schedule(dynamic)
        for (size_t i = 0; i < ab.n_pairs_; i++)
            for (size_t j = 0; j < c.n_shells_; j++)
            {
                auto b = k(i, j, ab, c);
                for (int x = 0; x < 9; x++)
                    std::memcpy(out + ((i * c.n_shells_ + j) * 9 + x) * blk, b[x].memptr(),
                                blk * sizeof(double));
            }
    });
}

// All ERI2D1Kernel batches between aux classes ia and ib, [n_a][n_b][6][Sa Sb].
int ref_eri2d1_class(void *h, int ia, int ib, double *out)
{
    return guarded([&]
    {
        auto sh = lints::shellDataAux(*static_cast<RefStructure *>(h)->s);
        const auto &a = sh.at(ia);
        const auto &b = sh.at(ib);
        lints::ERI2D1Kernel k(a, b);
        size_t blk = lints::numSphericals(a.l_) * lints::numSphericals(b.l_);
        for (size_t i = 0; i < a.n_shells_; i++)
            for (size_t j = 0; j < b.n_shells_; j++)
            {
                auto r = k(i, j, a, b);
                for (int x = 0; x < 6; x++)
                    std::memcpy(out + ((i * b.n_shells_ + j) * 6 + x) * blk, r[x].memptr(),
                                blk * sizeof(double));
            }
    });
}

int ref_aux_classes(void *h, int *n_classes, int *ls, long *n_shells)
{
    return guarded([&]
    {
        auto sh = lints::shellDataAux(*static_cast<RefStructure *>(h)->s);
        *n_classes = (int)sh.size();
        if (ls)
            for (size_t i = 0; i < sh.size(); i++)
            {
                ls[i] = sh[i].l_;
                n_shells[i] = (long)sh[i].n_shells_;
            }
    });
}

// The reference's kernel-API golden-sum loops (test/tests_ints.cpp:873-1053):
// which = 0 deployERI4Kernel, 1 deployERI3Kernel, 2 deployERI2Kernel, 3 deployERI4D1Kernel,
// 4 deployERI3D1Kernel, 5 deployERI2D1Kernel.
double ref_deploy_sum(void *h, int which)
{
    double total = 0;
    int rc = guarded([&]
    {
        auto &S = *static_cast<RefStructure *>(h)->s;
        if (which == 0 || which == 3)
        {
            auto sp = lints::shellPairData(which == 3, S);
            for (const auto &ab : sp)
                for (const auto &cd : sp)
                {
                    if (which == 0)
                    {
                        lints::ERI4Kernel k(ab, cd);
                        for (size_t i = 0; i < ab.n_pairs_; i++)
                            for (size_t j = 0; j < cd.n_pairs_; j++)
                                for (double v : k(i, j, ab, cd))
                                    total += std::fabs(v);
                    }
                    else
                    {
                        lints::ERI4D1Kernel k(ab, cd);
                        for (size_t i = 0; i < ab.n_pairs_; i++)
                            for (size_t j = 0; j < cd.n_pairs_; j++)
                                for (auto &blk : k(i, j, ab, cd))
                                    for (double v : blk)
                                        total += std::fabs(v);
                    }
                }
        }
        else if (which == 1 || which == 4)
        {
            auto sp = lints::shellPairData(false, S);
            auto sh = lints::shellDataAux(S);
            for (const auto &ab : sp)
                for (const auto &c : sh)
                {
                    if (which == 1)
                    {
                        lints::ERI3Kernel k(ab, c);
                        for (size_t i = 0; i < ab.n_pairs_; i++)
                            for (size_t j = 0; j < c.n_shells_; j++)
                                for (double v : k(i, j, ab, c))
                                    total += std::fabs(v);
                    }
                    else
                    {
                        lints::ERI3D1Kernel k(ab, c);
                        for (size_t i = 0; i < ab.n_pairs_; i++)
                            for (size_t j = 0; j < c.n_shells_; j++)
                                for (auto &blk : k(i, j, ab, c))
                                    for (double v : blk)
                                        total += std::fabs(v);
                    }
                }
        }
        else
        {
            auto sh = lints::shellDataAux(S);
            for (const auto &a : sh)
                for (const auto &b : sh)
                {
                    if (which == 2)
                    {
                        lints::ERI2Kernel k(a, b);
                        for (size_t i = 0; i < a.n_shells_; i++)
                            for (size_t j = 0; j < b.n_shells_; j++)
                                for (double v : k(i, j, a, b))
                                    total += std::fabs(v);
                    }
                    else
                    {
                        lints::ERI2D1Kernel k(a, b);
                        for (size_t i = 0; i < a.n_shells_; i++)
                            for (size_t j = 0; j < b.n_shells_; j++)
                                for (auto &blk : k(i, j, a, b))
                                    for (double v : blk)
                                        total += std::fabs(v);
                    }
                }
        }
    });
    return rc ? std::nan("") : total;
}

// Direct J/K from the reference's ERI4Kernel batches.  Unique quartets follow the eri4 driver's
// enumeration (class pairs cd <= ab, and ipair_cd <= ipair_ab inside one class); a quartet is kept
// iff Q_ab * Q_cd >= schwarz.  Every `bra_stride`-th bra pair is processed (1 = all), which lets the
// benchmark time a bounded, class-balanced sample.  J = A + A^T and K = B + B^T with the weighted
// 8-fold updates described in the product's digestion kernel.  Returns quartets processed.
int ref_jk(void *h, const double *D, double *J, double *K, double schwarz, int bra_stride,
           long long *n_quartets, double *seconds)
{
    return guarded([&]
    {
        auto &S = *static_cast<RefStructure *>(h)->s;
        auto t0 = std::chrono::steady_clock::now();
        auto sp = lints::shellPairData(true, S);
        const size_t n = S.getDimAO();
        std::vector<std::vector<double>> Q(sp.size());
        for (size_t c = 0; c < sp.size(); c++)
            Q[c] = schwarzFactors(sp[c]);
        int nt = omp_get_max_threads();
        std::vector<std::vector<double>> Jt(nt, std::vector<double>(n * n, 0.0));
        std::vector<std::vector<double>> Kt(nt, std::vector<double>(n * n, 0.0));
        long long nq = 0;
        int stride = bra_stride > 0 ? bra_stride : 1;
        for (size_t cab = 0; cab < sp.size(); cab++)
            for (size_t ccd = 0; ccd <= cab; ccd++)
            {
                const auto &ab = sp[cab];
                const auto &cd = sp[ccd];
                lints::ERI4Kernel kern(ab, cd);
                const int na = lints::numSphericals(ab.la_), nb = lints::numSphericals(ab.lb_);
                const int nc = lints::numSphericals(cd.la_), nd = lints::numSphericals(cd.lb_);
                const bool same = cab == ccd;
#pragma omp parallel for schedule(dynamic) reduction(+ : nq)
                for (size_t i = 0; i < ab.n_pairs_; i += stride)
                {
                    double *Ja = Jt[omp_get_thread_num()].data();
                    double *Ka = Kt[omp_get_thread_num()].data();
                    size_t bound = same ? i + 1 : cd.n_pairs_;
                    for (size_t j = 0; j < bound; j++)
                    {
                        if (Q[cab][i] * Q[ccd][j] < schwarz)
                            continue;
                        nq++;
                        lible::vec4d b = kern(i, j, ab, cd);
                        double f = quartetWeight(ab, i, cd, j, same);
                        size_t oa = ab.offsets_sph_[2 * i], ob = ab.offsets_sph_[2 * i + 1];
                        size_t oc = cd.offsets_sph_[2 * j], od = cd.offsets_sph_[2 * j + 1];
                        const double *v = b.memptr();
                        for (int x = 0; x < na; x++)
                            for (int y = 0; y < nb; y++)
                                for (int z = 0; z < nc; z++)
                                    for (int w = 0; w < nd; w++)
                                    {
                                        double g = f * v[((x * nb + y) * nc + z) * nd + w];
                                        size_t m = oa + x, nu = ob + y, k = oc + z, t = od + w;
                                        Ja[m * n + nu] += 2 * g * D[k * n + t];
                                        Ja[k * n + t] += 2 * g * D[m * n + nu];
                                        Ka[m * n + k] += g * D[nu * n + t];
                                        Ka[m * n + t] += g * D[nu * n + k];
                                        Ka[nu * n + k] += g * D[m * n + t];
                                        Ka[nu * n + t] += g * D[m * n + k];
                                    }
                    }
                }
            }
        for (size_t x = 0; x < n * n; x++)
        {
            double sj = 0, sk = 0;
            for (int t = 0; t < nt; t++)
            {
                sj += Jt[t][x];
                sk += Kt[t][x];
            }
            J[x] = sj;
            K[x] = sk;
        }
        for (size_t r = 0; r < n; r++)
            for (size_t c = 0; c <= r; c++)
            {
                double j = J[r * n + c] + J[c * n + r];
                double k = K[r * n + c] + K[c * n + r];
                J[r * n + c] = J[c * n + r] = j;
                K[r * n + c] = K[c * n + r] = k;
            }
        *n_quartets = nq;
        *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    });
}

// Gradient of E = 1/2 Tr(DJ) - 1/4 Tr(DK) with respect to the nuclear coordinates, from the
// reference's ERI4D1Kernel batches over the unique quartets (no Schwarz screening, which keeps the
// result exact for finite-difference checks).  grad is [n_atoms][3].
// `schwarz` > 0 keeps a quartet iff Q_ab Q_cd >= schwarz (the screened backward pass of the
// product keeps the same ones); `bra_stride` > 1 processes every bra_stride-th bra pair only, a
// bounded sample for timing.  Returns the quartets processed and the wall time.
static void jkGradImpl(void *h, const double *D, double *grad, double schwarz, int bra_stride, long long *n_quartets,
                       double *seconds)
{
    auto &S = *static_cast<RefStructure *>(h)->s;
    auto t0 = std::chrono::steady_clock::now();
    auto sp = lints::shellPairData(true, S);
    const size_t n = S.getDimAO();
    const size_t na_t = S.getNAtoms();
    std::vector<std::vector<double>> Q(sp.size());
    if (schwarz > 0)
        for (size_t c = 0; c < sp.size(); c++)
            Q[c] = schwarzFactors(sp[c]);
    const int stride = bra_stride > 0 ? bra_stride : 1;
    int nt = omp_get_max_threads();
    std::vector<std::vector<double>> Gt(nt, std::vector<double>(3 * na_t, 0.0));
    long long nq = 0;
    for (size_t cab = 0; cab < sp.size(); cab++)
        for (size_t ccd = 0; ccd <= cab; ccd++)
        {
            const auto &ab = sp[cab];
            const auto &cd = sp[ccd];
            lints::ERI4D1Kernel kern(ab, cd);
            const int na = lints::numSphericals(ab.la_), nb = lints::numSphericals(ab.lb_);
            const int nc = lints::numSphericals(cd.la_), nd = lints::numSphericals(cd.lb_);
            const bool same = cab == ccd;
#pragma omp parallel for schedule(dynamic) reduction(+ : nq)
            for (size_t i = 0; i < ab.n_pairs_; i += stride)
            {
                double *G = Gt[omp_get_thread_num()].data();
                size_t bound = same ? i + 1 : cd.n_pairs_;
                for (size_t j = 0; j < bound; j++)
                {
                    if (schwarz > 0 && Q[cab][i] * Q[ccd][j] < schwarz)
                        continue;
                    nq++;
                    auto blocks = kern(i, j, ab, cd);
                    double f = quartetWeight(ab, i, cd, j, same);
                    size_t oa = ab.offsets_sph_[2 * i], ob = ab.offsets_sph_[2 * i + 1];
                    size_t oc = cd.offsets_sph_[2 * j], od = cd.offsets_sph_[2 * j + 1];
                    size_t atoms[4] = {ab.atomic_idxs_[2 * i], ab.atomic_idxs_[2 * i + 1],
                                       cd.atomic_idxs_[2 * j], cd.atomic_idxs_[2 * j + 1]};
                    double acc[12] = {};
                    for (int x = 0; x < na; x++)
                        for (int y = 0; y < nb; y++)
                            for (int z = 0; z < nc; z++)
                                for (int w = 0; w < nd; w++)
                                {
                                    size_t m = oa + x, nu = ob + y, k = oc + z, t = od + w;
                                    double gam = f * (4 * D[m * n + nu] * D[k * n + t] -
                                                      D[m * n + k] * D[nu * n + t] -
                                                      D[m * n + t] * D[nu * n + k]);
                                    size_t e = ((x * nb + y) * nc + z) * nd + w;
                                    for (int c = 0; c < 12; c++)
                                        acc[c] += gam * blocks[c].memptr()[e];
                                }
                    for (int c = 0; c < 12; c++)
                        G[3 * atoms[c / 3] + c % 3] += acc[c];
                }
            }
        }
    for (size_t x = 0; x < 3 * na_t; x++)
    {
        double s = 0;
        for (int t = 0; t < nt; t++)
            s += Gt[t][x];
        grad[x] = s;
    }
    if (n_quartets)
        *n_quartets = nq;
    if (seconds)
        *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

int ref_jk_grad(void *h, const double *D, double *grad)
{
    return guarded([&] { jkGradImpl(h, D, grad, 0.0, 1, nullptr, nullptr); });
}

int ref_jk_grad_sample(void *h, const double *D, double *grad, double schwarz, int bra_stride, long long *n_quartets,
                       double *seconds)
{
    return guarded([&] { jkGradImpl(h, D, grad, schwarz, bra_stride, n_quartets, seconds); });
}

// RI-J pieces from the reference kernels: gamma_P = sum_mn (mn|P) D_mn over all pairs (ERI3Kernel
// over the symmetric pair list with the off-diagonal factor 2), and J_mn = sum_P (mn|P) d_P.
int ref_rij_gamma(void *h, const double *D, double *gamma)
{
    return guarded([&]
    {
        auto &S = *static_cast<RefStructure *>(h)->s;
        auto sp = lints::shellPairData(true, S);
        auto sh = lints::shellDataAux(S);
        const size_t n = S.getDimAO(), naux = S.getDimAOAux();
        std::fill(gamma, gamma + naux, 0.0);
        for (const auto &ab : sp)
            for (const auto &c : sh)
            {
                lints::ERI3Kernel kern(ab, c);
                const int na = lints::numSphericals(ab.la_), nb = lints::numSphericals(ab.lb_);
                const int nc = lints::numSphericals(c.l_);
                for (size_t i = 0; i < ab.n_pairs_; i++)
                {
                    bool diag = ab.shell_idxs_[2 * i] == ab.shell_idxs_[2 * i + 1];
                    size_t oa = ab.offsets_sph_[2 * i], ob = ab.offsets_sph_[2 * i + 1];
                    for (size_t j = 0; j < c.n_shells_; j++)
                    {
                        lible::vec3d b = kern(i, j, ab, c);
                        size_t oc = c.offsets_sph_[j];
                        for (int x = 0; x < na; x++)
                            for (int y = 0; y < nb; y++)
                            {
                                double d = D[(oa + x) * n + ob + y] * (diag ? 1.0 : 2.0);
                                for (int z = 0; z < nc; z++)
                                    gamma[oc + z] += d * b(x, y, z);
                            }
                    }
                }
            }
    });
}

int ref_rij_j(void *h, const double *dcoef, double *J)
{
    return guarded([&]
    {
        auto &S = *static_cast<RefStructure *>(h)->s;
        auto sp = lints::shellPairData(true, S);
        auto sh = lints::shellDataAux(S);
        const size_t n = S.getDimAO();
        std::fill(J, J + n * n, 0.0);
        for (const auto &ab : sp)
            for (const auto &c : sh)
            {
                lints::ERI3Kernel kern(ab, c);
                const int na = lints::numSphericals(ab.la_), nb = lints::numSphericals(ab.lb_);
                const int nc = lints::numSphericals(c.l_);
                for (size_t i = 0; i < ab.n_pairs_; i++)
                {
                    // a diagonal shell pair's batch already holds both (m, n) and (n, m)
                    bool diag = ab.shell_idxs_[2 * i] == ab.shell_idxs_[2 * i + 1];
                    size_t oa = ab.offsets_sph_[2 * i], ob = ab.offsets_sph_[2 * i + 1];
                    for (size_t j = 0; j < c.n_shells_; j++)
                    {
                        lible::vec3d b = kern(i, j, ab, c);
                        size_t oc = c.offsets_sph_[j];
                        for (int x = 0; x < na; x++)
                            for (int y = 0; y < nb; y++)
                            {
                                double s = 0;
                                for (int z = 0; z < nc; z++)
                                    s += b(x, y, z) * dcoef[oc + z];
                                J[(oa + x) * n + ob + y] += s;
                                if (!diag)
                                    J[(ob + y) * n + oa + x] += s;
                            }
                    }
                }
            }
    });
}

} // extern "C"
