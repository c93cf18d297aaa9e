// Host-side data model of the B200 ERI engine: basis sets, shells, shell-pair classes and the
// device-resident copies the kernels read.  Mirrors the reference's Structure / Shell /
// ShellData / ShellPairData (src/lible/ints/structure.hpp, shell.hpp, shell_pair_data.hpp) with
// identical ordering, normalization and primitive screening, because those decide per-integral
// parity.
#pragma once

#include "lible_math.hpp"

#include <vector_types.h>

#include <array>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

namespace lible_b200
{
    struct SphTerm
    {
        int row;    // spherical index (m order 0, +1, -1, ...)
        int cart;   // Cartesian index
        double val;
    };

    std::vector<SphTerm> sphericalTrafo(int l);
    std::vector<double> boysGrid();
    std::vector<float> boysGridF();
    void boysHost(int n, double x, const std::vector<double> &grid, double *F);

    struct BasisShell
    {
        int l = 0;
        std::vector<double> exps, coeffs;
    };

    struct BasisAtom
    {
        int z = 0;
        std::vector<BasisShell> shells;
    };

    // Reads element `z` from a basis file in the reference's text format
    // (src/lible/ints/basis_sets.cpp:214-277).  Throws std::runtime_error when absent.
    BasisAtom readBasisAtom(const std::string &path, int z);
    // Locates `<root>/<family>/<name>.txt` (case-insensitive name), like
    // src/lible/ints/basis_sets.cpp:318-360.
    std::string findBasisFile(const std::string &root, const std::string &name);

    struct Shell
    {
        int l = 0, z = 0;
        int mol = 0;                 // molecule of a batch (0 for a single structure)
        size_t idx = 0, atom = 0, ofs_sph = 0;
        double xyz[3] = {0, 0, 0};
        std::vector<double> exps, coeffs, prim_norms, norms;  // norms: one per spherical AO
    };

    double purePrimitiveNorm(int l, double a);
    // Contracted spherical AO norms from the self-overlap (src/lible/ints/shell.cpp:11-46).
    std::vector<double> shellNorms(int l, const std::vector<double> &exps,
                                   const std::vector<double> &coeffs,
                                   const std::vector<double> &prim_norms);
    std::vector<Shell> constructShells(const std::vector<BasisAtom> &atoms,
                                       const std::vector<std::array<double, 3>> &xyz_bohr);

    // One shell-pair class (la, lb) in the reference's ShellPairData layout.  `single` marks a
    // class built from single shells (auxiliary basis): each "pair" is (shell, unit s function of
    // exponent 0 on the same centre), which turns 3- and 2-centre integrals into 4-centre ones.
    struct PairClass
    {
        int la = 0, lb = 0;
        bool single = false;
        size_t n_pairs = 0, n_ppairs = 0;
        std::vector<double> exps, coeffs;       // [2 n_ppairs]: (a, b), (d_a, d_b) incl. primitive norms
        std::vector<double> coords;             // [6 n_pairs]
        std::vector<uint32_t> pofs;             // [n_pairs + 1] first primitive pair of each pair
        std::vector<int32_t> ao_a, ao_b;        // first spherical AO of each shell
        std::vector<int32_t> atom_a, atom_b;
        std::vector<int32_t> shell_a, shell_b;  // shell indices (for degeneracy factors)
        std::vector<double> norms_a, norms_b;   // [n_pairs * S_a], [n_pairs * S_b]
        // batches: per pair, the first element of its molecule's packed N_m x N_m matrices and N_m
        // (empty for a single structure: base 0, stride N)
        std::vector<int32_t> mat_base, mat_n;
    };

    // Appends the pairs of `src` to `dst` (same la, lb), tagging them with a packed-matrix block.
    void appendPairClass(PairClass &dst, const PairClass &src, int32_t mat_base, int32_t mat_n);

    PairClass buildPairClass(bool use_symm, int la, int lb, const std::vector<Shell> &sa,
                             const std::vector<Shell> &sb, double thr = kPrimitiveThreshold);
    PairClass buildSingleClass(int l, const std::vector<Shell> &s);

    // Device buffers of one pair class.
    struct DevPairClass
    {
        int la = 0, lb = 0;
        bool single = false;
        size_t n_pairs = 0, n_ppairs = 0;
        double *pP = nullptr;       // [n_ppairs][8]: p, Px, Py, Pz, 1/p, a, b, 0
        double *ab = nullptr;       // [n_ppairs][2]: a, b
        uint32_t *pofs = nullptr;   // [n_pairs + 1]
        int32_t *info = nullptr;    // [n_pairs][8]: ao_a, ao_b, atom_a, atom_b, shell_a, shell_b, 0, 0
        double *coords = nullptr;   // [n_pairs][6]
        double *E = nullptr;        // [n_ppairs][S_ab][H_ab]
        double *Et = nullptr;       // [n_ppairs][H_ab][S_ab]
        float *Ef = nullptr;        // fp32 copies (mixed precision)
        float *Etf = nullptr;
        double *E1 = nullptr;       // [n_ppairs][3][S_ab][H_ab]  d/d(A-B)
        double *E1t = nullptr;      // [n_ppairs][3][H_ab][S_ab]
        double *Q = nullptr;        // [n_pairs] Schwarz factors
        std::vector<double> Qh;     // host copy
        // Bra-side copies in Schwarz order, structure of arrays per (molecule, K) group g of n_g
        // pairs: element (prim k, field f) of the pair at group offset i sits at
        // base_g + (k * F + f) * n_g + i, so lanes holding consecutive Schwarz positions read
        // consecutive words.  soa[position] = (pP base + i, E base + i, n_g, FP32 record base + i).
        double *pPs = nullptr;      // F = 5: p, Px, Py, Pz, 1/p
        double *Es = nullptr;       // F = S_ab H_ab
        float *Efs = nullptr;
        float *pPfs = nullptr;      // F = 8: the FP32 record below, at soa.w
        uint4 *soa = nullptr;
        float *pPf = nullptr;       // [n_ppairs][8] FP32 record: p, 1/p, P (float hi), P - hi (float lo)
        int4 *soa2 = nullptr;       // per Schwarz position: ao_a, ao_b, packed-block base,
                                    // N_m | K << 16 | (same shell) << 31
        double *Dab = nullptr;      // per J/K call: D_ab of every pair, [mn][position]
        double *EtP = nullptr;      // Et zero-padded to the DMMA tile layout [ppair][rows][pitch]
    };
}
