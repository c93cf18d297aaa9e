/*
 * lible_b200.hpp: C++20 drop-in for the `lible::ints` ERI calls of MihkuU/Lible, over the C ABI of
 * lible_b200.h.  Header-only; link with -llible_b200 and compile against the reference's headers
 * (the functions take and return the reference's own types), with the reference's own build
 * definitions (LIBLE_MAIN_BASIS_DIR, LIBLE_AUX_BASIS_DIR, which its ints.hpp requires).
 *
 *   lible::ints::Structure s("cc-pvdz", {8, 1, 1}, coords_angstrom);
 *   lible::vec4d V = lible::ints::gpu::eri4(s);            // as lible::ints::eri4(s)
 *   lible::ints::gpu::Context ctx(s);                      // keep the device copy for many calls
 *   auto sp = lible::ints::shellPairData(true, s);
 *   lible::ints::gpu::ERI4Kernel k(ctx, sp[1], sp[0]);
 *   lible::vec4d b = k(0, 0, sp[1], sp[0]);                // as ERI4Kernel::operator()
 *
 * Replaced reference interfaces (paths relative to the reference project):
 *   eri4, eri4Diagonal, eri3, eri2, eri2Diagonal            src/lible/ints/ints.hpp:165-179
 *   ERI4Kernel, ERI3Kernel, ERI2Kernel, ERI4D1Kernel,
 *   ERI3D1Kernel, ERI2D1Kernel (operator())                 src/lible/ints/twoel/eri_kernels.hpp:60-169
 *   overlap, kineticEnergy, nuclearAttraction, nuclearAttractionErf, externalCharges,
 *   externalChargesErf, dipoleMoment, momentum, angularMomentum,
 *   spinOrbitCoupling1El, pVpIntegrals                       src/lible/ints/ints.hpp:29-154
 * Failures throw std::runtime_error with the library's message, as the reference throws
 * std::runtime_error for its own error cases.  jk(), jkEnergy() and jkEnergyGradient() have no
 * reference counterpart.
 */
#pragma once

#include <lible/ints/ints.hpp>
#include <lible/ints/shell_pair_data.hpp>
#include <lible/ints/structure.hpp>
#include <lible/types.hpp>

#include "lible_b200.h"

#include <algorithm>
#include <array>
#include <cstddef>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace lible::ints::gpu
{
    /// One device copy of a structure (its shells, shell pairs, E coefficients and Schwarz factors
    /// are built on the GPU once and reused by every call on the context).
    class Context
    {
    public:
        explicit Context(const Structure &structure, int device = 0)
        {
            check(lible_gpu_create(device, &ctx_));
            upload(structure);
        }
        ~Context()
        {
            if (ctx_)
                lible_gpu_destroy(ctx_);
        }
        Context(const Context &) = delete;
        Context &operator=(const Context &) = delete;
        Context(Context &&o) noexcept : ctx_(std::exchange(o.ctx_, nullptr)), nao_(o.nao_), naux_(o.naux_),
                                        n_atoms_(o.n_atoms_) {}

        lible_gpu_ctx *get() const { return ctx_; }
        std::size_t dimAO() const { return (std::size_t)nao_; }
        std::size_t dimAOAux() const { return (std::size_t)naux_; }
        std::size_t nAtoms() const { return (std::size_t)n_atoms_; }

        void check(int rc) const
        {
            if (rc != LIBLE_GPU_OK)
                throw std::runtime_error(std::string("lible_b200: ") +
                                         (ctx_ ? lible_gpu_last_error(ctx_) : "context creation failed"));
        }

        /// Index of the shell-pair class (la, lb) in shellPairData(use_symm, structure) order.
        int pairClass(const ShellPairData &sp) const
        {
            int n = 0;
            check(lible_gpu_pair_classes(ctx_, sp.uses_symm_ ? 1 : 0, &n, nullptr, nullptr, nullptr));
            std::vector<int> ls(2 * (std::size_t)n);
            check(lible_gpu_pair_classes(ctx_, sp.uses_symm_ ? 1 : 0, &n, ls.data(), nullptr, nullptr));
            for (int i = 0; i < n; i++)
                if (ls[2 * i] == sp.la_ && ls[2 * i + 1] == sp.lb_)
                    return i;
            throw std::runtime_error("lible_b200: shell-pair class not found in this structure");
        }

        /// Index of the auxiliary shell class of angular momentum l in shellDataAux(structure) order.
        int auxClass(const ShellData &sh) const
        {
            int n = 0;
            check(lible_gpu_aux_classes(ctx_, &n, nullptr, nullptr));
            std::vector<int> ls((std::size_t)n);
            check(lible_gpu_aux_classes(ctx_, &n, ls.data(), nullptr));
            for (int i = 0; i < n; i++)
                if (ls[i] == sh.l_)
                    return i;
            throw std::runtime_error("lible_b200: auxiliary shell class not found in this structure");
        }

    private:
        // Shells in the caller's atom order, coordinates in bohr as the reference keeps them.
        static void flatten(const std::vector<Shell> &shells, std::size_t n_atoms, std::vector<int> &per_atom,
                            std::vector<int> &l, std::vector<int> &nprim, std::vector<double> &exps,
                            std::vector<double> &coeffs)
        {
            per_atom.assign(n_atoms, 0);
            for (const Shell &s : shells)
            {
                per_atom.at(s.idx_atom_)++;
                l.push_back(s.l_);
                nprim.push_back((int)s.exps_.size());
                exps.insert(exps.end(), s.exps_.begin(), s.exps_.end());
                coeffs.insert(coeffs.end(), s.coeffs_.begin(), s.coeffs_.end());
            }
        }

        void upload(const Structure &structure)
        {
            const std::size_t n_atoms = structure.getNAtoms();
            std::vector<int> Z(n_atoms);
            std::vector<double> xyz(3 * n_atoms);
            for (std::size_t i = 0; i < n_atoms; i++)
            {
                Z[i] = structure.getZ(i);
                const auto c = structure.getCoordsAtom(i);
                xyz[3 * i] = c[0];
                xyz[3 * i + 1] = c[1];
                xyz[3 * i + 2] = c[2];
            }
            std::vector<int> pa, l, np, apa, al, anp;
            std::vector<double> ex, co, aex, aco;
            flatten(structure.getShells(), n_atoms, pa, l, np, ex, co);
            const bool ri = structure.getUseRI();
            if (ri)
                flatten(structure.getShellsAux(), n_atoms, apa, al, anp, aex, aco);
            check(lible_gpu_set_structure(ctx_, (int)n_atoms, Z.data(), xyz.data(), 1, pa.data(), l.data(), np.data(),
                                          ex.data(), co.data(), ri ? apa.data() : nullptr,
                                          ri ? al.data() : nullptr, ri ? anp.data() : nullptr,
                                          ri ? aex.data() : nullptr, ri ? aco.data() : nullptr));
            int max_l = 0;
            check(lible_gpu_dims(ctx_, &nao_, &naux_, &n_atoms_, &max_l));
        }

        lible_gpu_ctx *ctx_ = nullptr;
        long long nao_ = 0, naux_ = 0;
        int n_atoms_ = 0;
    };

    // ---- free functions (ints.hpp:165-179) --------------------------------------------------------

    inline vec4d eri4(Context &c)
    {
        const std::size_t n = c.dimAO();
        vec4d out(n, n, n, n);
        c.check(lible_gpu_eri4(c.get(), out.memptr()));
        return out;
    }
    inline vec4d eri4(const Structure &structure, int device = 0)
    {
        Context c(structure, device);
        return eri4(c);
    }

    inline vec2d eri4Diagonal(Context &c)
    {
        const std::size_t n = c.dimAO();
        vec2d out(n, n);
        c.check(lible_gpu_eri4_diagonal(c.get(), out.memptr()));
        return out;
    }
    inline vec2d eri4Diagonal(const Structure &structure, int device = 0)
    {
        Context c(structure, device);
        return eri4Diagonal(c);
    }

    inline vec3d eri3(Context &c)
    {
        vec3d out(c.dimAO(), c.dimAO(), c.dimAOAux());
        c.check(lible_gpu_eri3(c.get(), out.memptr()));
        return out;
    }
    inline vec3d eri3(const Structure &structure, int device = 0)
    {
        Context c(structure, device);
        return eri3(c);
    }

    inline vec2d eri2(Context &c)
    {
        vec2d out(c.dimAOAux(), c.dimAOAux());
        c.check(lible_gpu_eri2(c.get(), out.memptr()));
        return out;
    }
    inline vec2d eri2(const Structure &structure, int device = 0)
    {
        Context c(structure, device);
        return eri2(c);
    }

    inline std::vector<double> eri2Diagonal(Context &c)
    {
        std::vector<double> out(c.dimAOAux());
        c.check(lible_gpu_eri2_diagonal(c.get(), out.data()));
        return out;
    }
    inline std::vector<double> eri2Diagonal(const Structure &structure, int device = 0)
    {
        Context c(structure, device);
        return eri2Diagonal(c);
    }

    // ---- one-electron drivers (ints.hpp:29-151) ---------------------------------------------------
    // Point charges are {x, y, z, q} with coordinates in bohr, as the reference's.

    namespace detail
    {
        inline std::vector<double> flatCharges(const std::vector<std::array<double, 4>> &q)
        {
            std::vector<double> f;
            f.reserve(4 * q.size());
            for (const auto &c : q)
                f.insert(f.end(), c.begin(), c.end());
            return f;
        }
        inline std::array<vec2d, 3> three(Context &c, const std::vector<double> &flat)
        {
            const std::size_t n = c.dimAO();
            std::array<vec2d, 3> out{vec2d(n, n), vec2d(n, n), vec2d(n, n)};
            for (int d = 0; d < 3; d++)
                std::copy(flat.begin() + (std::ptrdiff_t)(d * n * n), flat.begin() + (std::ptrdiff_t)((d + 1) * n * n),
                          out[d].memptr());
            return out;
        }
    }

    inline vec2d overlap(Context &c)
    {
        vec2d out(c.dimAO(), c.dimAO());
        c.check(lible_gpu_overlap(c.get(), out.memptr()));
        return out;
    }
    inline vec2d overlap(const Structure &structure, int device = 0)
    {
        Context c(structure, device);
        return overlap(c);
    }
    inline vec2d kineticEnergy(Context &c)
    {
        vec2d out(c.dimAO(), c.dimAO());
        c.check(lible_gpu_kinetic_energy(c.get(), out.memptr()));
        return out;
    }
    inline vec2d kineticEnergy(const Structure &structure, int device = 0)
    {
        Context c(structure, device);
        return kineticEnergy(c);
    }
    inline vec2d nuclearAttraction(Context &c)
    {
        vec2d out(c.dimAO(), c.dimAO());
        c.check(lible_gpu_nuclear_attraction(c.get(), out.memptr()));
        return out;
    }
    inline vec2d nuclearAttraction(const Structure &structure, int device = 0)
    {
        Context c(structure, device);
        return nuclearAttraction(c);
    }
    inline vec2d nuclearAttractionErf(Context &c, const std::vector<double> &omegas)
    {
        if (omegas.size() != (std::size_t)c.nAtoms())
            throw std::runtime_error("nuclearAttractionErf(): number of omega values must match number of atoms");
        vec2d out(c.dimAO(), c.dimAO());
        c.check(lible_gpu_nuclear_attraction_erf(c.get(), omegas.data(), out.memptr()));
        return out;
    }
    inline vec2d nuclearAttractionErf(const Structure &structure, const std::vector<double> &omegas, int device = 0)
    {
        Context c(structure, device);
        return nuclearAttractionErf(c, omegas);
    }
    inline vec2d externalCharges(const std::vector<std::array<double, 4>> &point_charges, Context &c)
    {
        const std::vector<double> q = detail::flatCharges(point_charges);
        vec2d out(c.dimAO(), c.dimAO());
        c.check(lible_gpu_external_charges(c.get(), q.data(), (int)point_charges.size(), out.memptr()));
        return out;
    }
    inline vec2d externalCharges(const std::vector<std::array<double, 4>> &point_charges, const Structure &structure,
                                 int device = 0)
    {
        Context c(structure, device);
        return externalCharges(point_charges, c);
    }
    inline vec2d externalChargesErf(const std::vector<std::array<double, 4>> &point_charges,
                                    const std::vector<double> &omegas, Context &c)
    {
        if (omegas.size() != point_charges.size())
            throw std::runtime_error("externalChargesErf(): number of omega values must match number of charges");
        const std::vector<double> q = detail::flatCharges(point_charges);
        vec2d out(c.dimAO(), c.dimAO());
        c.check(lible_gpu_external_charges_erf(c.get(), q.data(), omegas.data(), (int)point_charges.size(),
                                               out.memptr()));
        return out;
    }
    inline vec2d externalChargesErf(const std::vector<std::array<double, 4>> &point_charges,
                                    const std::vector<double> &omegas, const Structure &structure, int device = 0)
    {
        Context c(structure, device);
        return externalChargesErf(point_charges, omegas, c);
    }
    inline std::array<vec2d, 3> dipoleMoment(const std::array<double, 3> &origin, Context &c)
    {
        std::vector<double> flat(3 * c.dimAO() * c.dimAO());
        c.check(lible_gpu_dipole_moment(c.get(), origin.data(), flat.data()));
        return detail::three(c, flat);
    }
    inline std::array<vec2d, 3> dipoleMoment(const std::array<double, 3> &origin, const Structure &structure,
                                             int device = 0)
    {
        Context c(structure, device);
        return dipoleMoment(origin, c);
    }
    // The full antisymmetric matrices of -<m| d/dr |n> (the reference's driver writes only one
    // orientation of each pair of different shells, negated).
    inline std::array<vec2d, 3> momentum(Context &c)
    {
        std::vector<double> flat(3 * c.dimAO() * c.dimAO());
        c.check(lible_gpu_momentum(c.get(), flat.data()));
        return detail::three(c, flat);
    }
    inline std::array<vec2d, 3> momentum(const Structure &structure, int device = 0)
    {
        Context c(structure, device);
        return momentum(c);
    }
    inline std::array<vec2d, 3> angularMomentum(const std::array<double, 3> &origin, Context &c)
    {
        std::vector<double> flat(3 * c.dimAO() * c.dimAO());
        c.check(lible_gpu_angular_momentum(c.get(), origin.data(), flat.data()));
        return detail::three(c, flat);
    }
    inline std::array<vec2d, 3> angularMomentum(const std::array<double, 3> &origin, const Structure &structure,
                                                int device = 0)
    {
        Context c(structure, device);
        return angularMomentum(origin, c);
    }
    inline std::array<vec2d, 3> spinOrbitCoupling1El(Context &c)
    {
        std::vector<double> flat(3 * c.dimAO() * c.dimAO());
        c.check(lible_gpu_spin_orbit_coupling_1el(c.get(), flat.data()));
        return detail::three(c, flat);
    }
    inline std::array<vec2d, 3> spinOrbitCoupling1El(const Structure &structure, int device = 0)
    {
        Context c(structure, device);
        return spinOrbitCoupling1El(c);
    }
    // <d_i m| V |d_j n> for the nuclei, [i][j]; the integrals themselves, where the reference's
    // pVpIntegrals differs (lible_b200.h, lible_gpu_pvp_integrals).
    inline arr2d<vec2d, 3, 3> pVpIntegrals(Context &c)
    {
        const std::size_t n = c.dimAO();
        std::vector<double> flat(9 * n * n);
        c.check(lible_gpu_pvp_integrals(c.get(), nullptr, 0, flat.data()));
        arr2d<vec2d, 3, 3> out;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
            {
                out[i][j] = vec2d(n, n);
                std::copy(flat.begin() + (std::ptrdiff_t)((3 * i + j) * n * n),
                          flat.begin() + (std::ptrdiff_t)((3 * i + j + 1) * n * n), out[i][j].memptr());
            }
        return out;
    }
    inline arr2d<vec2d, 3, 3> pVpIntegrals(const Structure &structure, int device = 0)
    {
        Context c(structure, device);
        return pVpIntegrals(c);
    }

    // ---- kernel functors (eri_kernels.hpp:60-169) -------------------------------------------------
    // Each functor evaluates one shell-pair (or shell) combination per operator() call, as the
    // reference's do; batch() evaluates many in one launch, which is the fast form on a GPU.

    namespace detail
    {
        inline std::size_t nsph(int l) { return 2 * (std::size_t)l + 1; }
    }

    class ERI4Kernel
    {
    public:
        ERI4Kernel(Context &c, const ShellPairData &sp_ab, const ShellPairData &sp_cd)
            : c_(&c), symm_(sp_ab.uses_symm_), cab_(c.pairClass(sp_ab)), ccd_(c.pairClass(sp_cd)),
              dims_{detail::nsph(sp_ab.la_), detail::nsph(sp_ab.lb_), detail::nsph(sp_cd.la_), detail::nsph(sp_cd.lb_)}
        {
        }
        /// out[i] = the [Sa][Sb][Sc][Sd] batch of pairs[i] = (ipair_ab, ipair_cd).
        void batch(const std::vector<std::array<unsigned, 2>> &pairs, double *out) const
        {
            c_->check(call(c_->get(), symm_ ? 1 : 0, cab_, ccd_, (long long)pairs.size(),
                           pairs.empty() ? nullptr : &pairs[0][0], out));
        }
        vec4d operator()(std::size_t ipair_ab, std::size_t ipair_cd, const ShellPairData &,
                         const ShellPairData &) const
        {
            vec4d out(dims_[0], dims_[1], dims_[2], dims_[3]);
            batch({{(unsigned)ipair_ab, (unsigned)ipair_cd}}, out.memptr());
            return out;
        }

    protected:
        using Fn = int (*)(lible_gpu_ctx *, int, int, int, long long, const unsigned *, double *);
        Fn call = &lible_gpu_eri4_batch;
        Context *c_;
        bool symm_;
        int cab_, ccd_;
        std::array<std::size_t, 4> dims_;
    };

    class ERI4D1Kernel : public ERI4Kernel
    {
    public:
        ERI4D1Kernel(Context &c, const ShellPairData &sp_ab, const ShellPairData &sp_cd) : ERI4Kernel(c, sp_ab, sp_cd)
        {
            call = &lible_gpu_eri4d1_batch;
        }
        /// The 12 derivative blocks [A, B, C, D] x [x, y, z] (eri_kernels.hpp:114-132).
        std::array<vec4d, 12> operator()(std::size_t ipair_ab, std::size_t ipair_cd, const ShellPairData &,
                                         const ShellPairData &) const
        {
            const std::size_t blk = dims_[0] * dims_[1] * dims_[2] * dims_[3];
            std::vector<double> tmp(12 * blk);
            batch({{(unsigned)ipair_ab, (unsigned)ipair_cd}}, tmp.data());
            std::array<vec4d, 12> out;
            for (int k = 0; k < 12; k++)
            {
                out[k] = vec4d(dims_[0], dims_[1], dims_[2], dims_[3]);
                std::copy(tmp.begin() + k * blk, tmp.begin() + (k + 1) * blk, out[k].memptr());
            }
            return out;
        }
    };

    class ERI3Kernel
    {
    public:
        ERI3Kernel(Context &c, const ShellPairData &sp_ab, const ShellData &sh_c)
            : c_(&c), symm_(sp_ab.uses_symm_), cab_(c.pairClass(sp_ab)), cx_(c.auxClass(sh_c)),
              dims_{detail::nsph(sp_ab.la_), detail::nsph(sp_ab.lb_), detail::nsph(sh_c.l_)}
        {
        }
        /// out[i] = the [Sa][Sb][Sc] batch of idx[i] = (ipair_ab, ishell_c).
        void batch(const std::vector<std::array<unsigned, 2>> &idx, double *out) const
        {
            c_->check(call(c_->get(), symm_ ? 1 : 0, cab_, cx_, (long long)idx.size(), idx.empty() ? nullptr : &idx[0][0],
                           out));
        }
        vec3d operator()(std::size_t ipair_ab, std::size_t ishell_c, const ShellPairData &, const ShellData &) const
        {
            vec3d out(dims_[0], dims_[1], dims_[2]);
            batch({{(unsigned)ipair_ab, (unsigned)ishell_c}}, out.memptr());
            return out;
        }

    protected:
        using Fn = int (*)(lible_gpu_ctx *, int, int, int, long long, const unsigned *, double *);
        Fn call = &lible_gpu_eri3_batch;
        Context *c_;
        bool symm_;
        int cab_, cx_;
        std::array<std::size_t, 3> dims_;
    };

    class ERI3D1Kernel : public ERI3Kernel
    {
    public:
        ERI3D1Kernel(Context &c, const ShellPairData &sp_ab, const ShellData &sh_c) : ERI3Kernel(c, sp_ab, sh_c)
        {
            call = &lible_gpu_eri3d1_batch;
        }
        /// The 9 derivative blocks [A, B, C] x [x, y, z] (eri_kernels.hpp:134-151).
        std::array<vec3d, 9> operator()(std::size_t ipair_ab, std::size_t ishell_c, const ShellPairData &,
                                        const ShellData &) const
        {
            const std::size_t blk = dims_[0] * dims_[1] * dims_[2];
            std::vector<double> tmp(9 * blk);
            batch({{(unsigned)ipair_ab, (unsigned)ishell_c}}, tmp.data());
            std::array<vec3d, 9> out;
            for (int k = 0; k < 9; k++)
            {
                out[k] = vec3d(dims_[0], dims_[1], dims_[2]);
                std::copy(tmp.begin() + k * blk, tmp.begin() + (k + 1) * blk, out[k].memptr());
            }
            return out;
        }
    };

    class ERI2Kernel
    {
    public:
        ERI2Kernel(Context &c, const ShellData &sh_a, const ShellData &sh_b)
            : c_(&c), ca_(c.auxClass(sh_a)), cb_(c.auxClass(sh_b)), dims_{detail::nsph(sh_a.l_), detail::nsph(sh_b.l_)}
        {
        }
        void batch(const std::vector<std::array<unsigned, 2>> &idx, double *out) const
        {
            c_->check(call(c_->get(), ca_, cb_, (long long)idx.size(), idx.empty() ? nullptr : &idx[0][0], out));
        }
        vec2d operator()(std::size_t ishell_a, std::size_t ishell_b, const ShellData &, const ShellData &) const
        {
            vec2d out(dims_[0], dims_[1]);
            batch({{(unsigned)ishell_a, (unsigned)ishell_b}}, out.memptr());
            return out;
        }

    protected:
        using Fn = int (*)(lible_gpu_ctx *, int, int, long long, const unsigned *, double *);
        Fn call = &lible_gpu_eri2_batch;
        Context *c_;
        int ca_, cb_;
        std::array<std::size_t, 2> dims_;
    };

    class ERI2D1Kernel : public ERI2Kernel
    {
    public:
        ERI2D1Kernel(Context &c, const ShellData &sh_a, const ShellData &sh_b) : ERI2Kernel(c, sh_a, sh_b)
        {
            call = &lible_gpu_eri2d1_batch;
        }
        /// The 6 derivative blocks [A, B] x [x, y, z] (eri_kernels.hpp:153-169).
        std::array<vec2d, 6> operator()(std::size_t ishell_a, std::size_t ishell_b, const ShellData &,
                                        const ShellData &) const
        {
            const std::size_t blk = dims_[0] * dims_[1];
            std::vector<double> tmp(6 * blk);
            batch({{(unsigned)ishell_a, (unsigned)ishell_b}}, tmp.data());
            std::array<vec2d, 6> out;
            for (int k = 0; k < 6; k++)
            {
                out[k] = vec2d(dims_[0], dims_[1]);
                std::copy(tmp.begin() + k * blk, tmp.begin() + (k + 1) * blk, out[k].memptr());
            }
            return out;
        }
    };

    // ---- direct J/K and its energy gradient (no reference counterpart) -----------------------------

    /// J_mn = sum (mn|ls) D_ls and K_mn = sum (ml|ns) D_ls for a symmetric density, over the
    /// quartets with Q_ab Q_cd >= schwarz; mixed = FP32 for quartets with Q_ab Q_cd < fp32_threshold.
    inline void jk(Context &c, const vec2d &D, vec2d &J, vec2d &K, double schwarz = 1e-12, bool mixed = false,
                   double fp32_threshold = 1e-4)
    {
        const std::size_t n = c.dimAO();
        J = vec2d(n, n);
        K = vec2d(n, n);
        lible_gpu_jk_opts o{schwarz, fp32_threshold, mixed ? 1 : 0, 0};
        c.check(lible_gpu_jk(c.get(), D.memptr(), J.memptr(), K.memptr(), &o, nullptr));
    }

    /// E = 1/2 Tr(DJ) - 1/4 Tr(DK) (the forward pass).
    inline double jkEnergy(Context &c, const vec2d &D, double schwarz = 1e-12)
    {
        lible_gpu_jk_opts o{schwarz, 1e-4, 0, 0};
        double e = 0;
        c.check(lible_gpu_jk_energy_forward(c.get(), D.memptr(), &o, &e, nullptr, nullptr));
        return e;
    }

    /// dE/dR per atom (the backward pass): first-derivative integrals contracted with the
    /// two-particle density of E on the device.
    inline std::vector<std::array<double, 3>> jkEnergyGradient(Context &c, const vec2d &D, double schwarz = 1e-12)
    {
        std::vector<std::array<double, 3>> g(c.nAtoms());
        lible_gpu_jk_opts o{schwarz, 1e-4, 0, 0};
        c.check(lible_gpu_jk_energy_backward(c.get(), D.memptr(), &o, g.empty() ? nullptr : &g[0][0]));
        return g;
    }
}
