// Basis sets, shells and shell-pair classes on the host.
#include "engine.hpp"

#include <algorithm>
#include <cctype>
#include <filesystem>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace fs = std::filesystem;

namespace lible_b200
{
    BasisAtom readBasisAtom(const std::string &path, int z)
    {
        std::ifstream in(path);
        if (!in)
            throw std::runtime_error("cannot open basis file " + path);
        const std::string begin = "element=" + std::to_string(z);
        const std::string end = "end=" + std::to_string(z);
        BasisAtom atom;
        atom.z = z;
        bool inside = false, found = false;
        std::string line;
        while (std::getline(in, line))
        {
            if (!line.empty() && line.back() == '\r')
                line.pop_back();
            if (!inside)
            {
                if (line == begin)
                    inside = found = true;
                continue;
            }
            if (line == end)
                break;
            auto pos = line.find("l=");
            if (pos != std::string::npos)
            {
                BasisShell sh;
                sh.l = line[pos + 2] - '0';
                atom.shells.push_back(sh);
                continue;
            }
            std::istringstream ss(line);
            double e, c;
            if (ss >> e >> c)
            {
                if (atom.shells.empty())
                    throw std::runtime_error("malformed basis file " + path);
                atom.shells.back().exps.push_back(e);
                atom.shells.back().coeffs.push_back(c);
            }
        }
        if (!found)
            throw std::runtime_error("basis set in " + path + " has no element Z=" + std::to_string(z));
        return atom;
    }

    std::string findBasisFile(const std::string &root, const std::string &name)
    {
        std::string want = name;
        std::transform(want.begin(), want.end(), want.begin(), [](unsigned char c) { return std::tolower(c); });
        if (fs::is_directory(root))
            for (const auto &fam : fs::directory_iterator(root))
            {
                if (!fam.is_directory())
                    continue;
                for (const auto &f : fs::directory_iterator(fam.path()))
                {
                    std::string stem = f.path().filename().string();
                    stem = stem.substr(0, stem.find('.'));
                    if (stem == want)
                        return f.path().string();
                }
            }
        throw std::runtime_error("basis set " + name + " not found under " + root);
    }

    static double doubleFactorial(int n)
    {
        double r = 1.0;
        for (int i = n; i >= 2; i -= 2)
            r *= i;
        return r;
    }

    // sqrt((2a/pi)^{3/2} (4a)^l / (2l-1)!!), src/lible/ints/utils.cpp:6-10.
    double purePrimitiveNorm(int l, double a)
    {
        return std::sqrt(std::pow(2 * a / M_PI, 1.5) * std::pow(4 * a, l) / doubleFactorial(2 * l - 1));
    }

    std::vector<double> shellNorms(int l, const std::vector<double> &exps,
                                   const std::vector<double> &coeffs,
                                   const std::vector<double> &prim_norms)
    {
        const int nc = ncart(l);
        std::vector<double> S(nc * nc, 0.0);
        std::vector<double> Ex((l + 1) * (l + 1) * (2 * l + 1));
        // Cartesian exponents in the reference order
        std::vector<std::array<int, 3>> ce;
        for (int x = l; x >= 0; x--)
            for (int y = l - x; y >= 0; y--)
                ce.push_back({x, y, l - x - y});
        for (size_t ia = 0; ia < exps.size(); ia++)
            for (size_t ib = 0; ib < exps.size(); ib++)
            {
                double a = exps[ia], b = exps[ib], p = a + b;
                double fac = coeffs[ia] * prim_norms[ia] * coeffs[ib] * prim_norms[ib] * std::pow(M_PI / p, 1.5);
                hermiteE(l, l, 0.5 / p, 0.0, 0.0, 1.0, Ex.data());
                auto e = [&](int i, int j) { return Ex[(i * (l + 1) + j) * (2 * l + 1)]; };
                for (int m = 0; m < nc; m++)
                    for (int n = 0; n < nc; n++)
                        S[m * nc + n] += fac * e(ce[m][0], ce[n][0]) * e(ce[m][1], ce[n][1]) *
                                         e(ce[m][2], ce[n][2]);
            }
        auto T = sphericalTrafo(l);
        std::vector<double> norms(nsph(l));
        for (int r = 0; r < nsph(l); r++)
        {
            double s = 0;
            for (const auto &t1 : T)
                if (t1.row == r)
                    for (const auto &t2 : T)
                        if (t2.row == r)
                            s += t1.val * t2.val * S[t1.cart * nc + t2.cart];
            norms[r] = 1.0 / std::sqrt(s);
        }
        return norms;
    }

    std::vector<Shell> constructShells(const std::vector<BasisAtom> &atoms,
                                       const std::vector<std::array<double, 3>> &xyz_bohr)
    {
        if (atoms.size() != xyz_bohr.size())
            throw std::runtime_error("constructShells(): number of atoms and coordinates differ");
        std::vector<Shell> shells;
        size_t ofs = 0;
        for (size_t a = 0; a < atoms.size(); a++)
            for (const auto &bs : atoms[a].shells)
            {
                if (bs.exps.size() != bs.coeffs.size() || bs.exps.empty())
                    throw std::runtime_error("constructShells(): exponents/coefficients mismatch");
                if (bs.l < 0 || bs.l > kMaxL)
                    throw std::runtime_error("constructShells(): angular momentum " + std::to_string(bs.l) +
                                             " exceeds the supported maximum");
                Shell s;
                s.l = bs.l;
                s.z = atoms[a].z;
                s.idx = shells.size();
                s.atom = a;
                s.ofs_sph = ofs;
                for (int k = 0; k < 3; k++)
                    s.xyz[k] = xyz_bohr[a][k];
                s.exps = bs.exps;
                s.coeffs = bs.coeffs;
                for (double e : bs.exps)
                    s.prim_norms.push_back(purePrimitiveNorm(bs.l, e));
                s.norms = shellNorms(bs.l, s.exps, s.coeffs, s.prim_norms);
                ofs += nsph(bs.l);
                shells.push_back(std::move(s));
            }
        return shells;
    }

    // src/lible/ints/shell_pair_data.cpp:73-202: pairs in (i, j) loop order, j <= i when the two
    // shell lists are the same class and symmetry is used; a primitive pair survives iff
    // |d_a d_b exp(-ab/(a+b) R_AB^2)| >= thr; pairs without survivors are dropped.
    PairClass buildPairClass(bool use_symm, int la, int lb, const std::vector<Shell> &sa,
                             const std::vector<Shell> &sb, double thr)
    {
        PairClass pc;
        pc.la = la;
        pc.lb = lb;
        pc.pofs.push_back(0);
        for (size_t i = 0; i < sa.size(); i++)
        {
            size_t bound = (use_symm && la == lb) ? i + 1 : sb.size();
            for (size_t j = 0; j < bound; j++)
            {
                const Shell &A = sa[i], &B = sb[j];
                if (A.l != la || B.l != lb)
                    throw std::runtime_error("buildPairClass(): shell angular momentum mismatch");
                double r2 = 0;
                for (int k = 0; k < 3; k++)
                    r2 += (A.xyz[k] - B.xyz[k]) * (A.xyz[k] - B.xyz[k]);
                size_t kept = 0;
                for (size_t ia = 0; ia < A.exps.size(); ia++)
                    for (size_t ib = 0; ib < B.exps.size(); ib++)
                    {
                        double a = A.exps[ia], b = B.exps[ib];
                        double da = A.prim_norms[ia] * A.coeffs[ia];
                        double db = B.prim_norms[ib] * B.coeffs[ib];
                        double mu = a * b / (a + b);
                        if (std::fabs(da * db * std::exp(-mu * r2)) >= thr)
                        {
                            pc.exps.push_back(a);
                            pc.exps.push_back(b);
                            pc.coeffs.push_back(da);
                            pc.coeffs.push_back(db);
                            kept++;
                        }
                    }
                if (kept == 0)
                    continue;
                for (int k = 0; k < 3; k++)
                    pc.coords.push_back(A.xyz[k]);
                for (int k = 0; k < 3; k++)
                    pc.coords.push_back(B.xyz[k]);
                pc.pofs.push_back(pc.pofs.back() + (uint32_t)kept);
                pc.ao_a.push_back((int32_t)A.ofs_sph);
                pc.ao_b.push_back((int32_t)B.ofs_sph);
                pc.atom_a.push_back((int32_t)A.atom);
                pc.atom_b.push_back((int32_t)B.atom);
                pc.shell_a.push_back((int32_t)A.idx);
                pc.shell_b.push_back((int32_t)B.idx);
                pc.norms_a.insert(pc.norms_a.end(), A.norms.begin(), A.norms.end());
                pc.norms_b.insert(pc.norms_b.end(), B.norms.begin(), B.norms.end());
            }
        }
        pc.n_pairs = pc.ao_a.size();
        pc.n_ppairs = pc.pofs.back();
        return pc;
    }

    void appendPairClass(PairClass &dst, const PairClass &src, int32_t mat_base, int32_t mat_n)
    {
        if (dst.pofs.empty())
        {
            dst.la = src.la;
            dst.lb = src.lb;
            dst.single = src.single;
            dst.pofs.push_back(0);
        }
        if (dst.la != src.la || dst.lb != src.lb)
            throw std::runtime_error("appendPairClass(): class mismatch");
        const uint32_t p0 = dst.pofs.back();
        dst.exps.insert(dst.exps.end(), src.exps.begin(), src.exps.end());
        dst.coeffs.insert(dst.coeffs.end(), src.coeffs.begin(), src.coeffs.end());
        dst.coords.insert(dst.coords.end(), src.coords.begin(), src.coords.end());
        for (size_t i = 1; i < src.pofs.size(); i++)
            dst.pofs.push_back(p0 + src.pofs[i]);
        dst.ao_a.insert(dst.ao_a.end(), src.ao_a.begin(), src.ao_a.end());
        dst.ao_b.insert(dst.ao_b.end(), src.ao_b.begin(), src.ao_b.end());
        dst.atom_a.insert(dst.atom_a.end(), src.atom_a.begin(), src.atom_a.end());
        dst.atom_b.insert(dst.atom_b.end(), src.atom_b.begin(), src.atom_b.end());
        dst.shell_a.insert(dst.shell_a.end(), src.shell_a.begin(), src.shell_a.end());
        dst.shell_b.insert(dst.shell_b.end(), src.shell_b.begin(), src.shell_b.end());
        dst.norms_a.insert(dst.norms_a.end(), src.norms_a.begin(), src.norms_a.end());
        dst.norms_b.insert(dst.norms_b.end(), src.norms_b.begin(), src.norms_b.end());
        dst.mat_base.insert(dst.mat_base.end(), src.n_pairs, mat_base);
        dst.mat_n.insert(dst.mat_n.end(), src.n_pairs, mat_n);
        dst.n_pairs = dst.ao_a.size();
        dst.n_ppairs = dst.pofs.back();
    }

    PairClass buildSingleClass(int l, const std::vector<Shell> &s)
    {
        PairClass pc;
        pc.la = l;
        pc.lb = 0;
        pc.single = true;
        pc.pofs.push_back(0);
        for (const Shell &A : s)
        {
            if (A.l != l)
                throw std::runtime_error("buildSingleClass(): shell angular momentum mismatch");
            for (size_t ia = 0; ia < A.exps.size(); ia++)
            {
                pc.exps.push_back(A.exps[ia]);
                pc.exps.push_back(0.0);
                pc.coeffs.push_back(A.prim_norms[ia] * A.coeffs[ia]);
                pc.coeffs.push_back(1.0);
            }
            for (int r = 0; r < 2; r++)
                for (int k = 0; k < 3; k++)
                    pc.coords.push_back(A.xyz[k]);
            pc.pofs.push_back(pc.pofs.back() + (uint32_t)A.exps.size());
            pc.ao_a.push_back((int32_t)A.ofs_sph);
            pc.ao_b.push_back(-1);
            pc.atom_a.push_back((int32_t)A.atom);
            pc.atom_b.push_back((int32_t)A.atom);
            pc.shell_a.push_back((int32_t)A.idx);
            pc.shell_b.push_back(-1);
            pc.norms_a.insert(pc.norms_a.end(), A.norms.begin(), A.norms.end());
            pc.norms_b.push_back(1.0);
        }
        pc.n_pairs = pc.ao_a.size();
        pc.n_ppairs = pc.pofs.back();
        return pc;
    }
}
