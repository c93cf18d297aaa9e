// C++20 check of include/lible_b200.hpp against the reference itself: builds lible::ints::Structure
// objects of the reference (linked from oracle/_ref/liblible_ref.so, the reference's own sources)
// and compares every drop-in call with the reference call of the same name on the same object.
//
//   test_dropin <lible_b200/basis directory>     exit 0 = every difference <= 1e-12 (per integral)
//
// Molecules: O3 / def2-SVP with def2-universal-jkfit (the reference's eri4/eri3/eri2 golden
// molecule, test/tests_ints.cpp) and water / cc-pVDZ.  Test infrastructure only.
#include <lible_b200.hpp>

#include <lible/ints/ints.hpp>
#include <lible/ints/twoel/eri_kernels.hpp>

#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace lints = lible::ints;

// The per-element shells of a basis file in the reference's text format (element=Z, "l=L n=K"
// blocks of K "exponent coefficient" lines, end=Z).
static lints::basis_atoms_t readBasis(const std::string &path, const std::vector<int> &Z)
{
    std::ifstream in(path);
    if (!in)
        throw std::runtime_error("cannot open " + path);
    std::map<int, lints::basis_shells_t> elems;
    std::string line;
    int z = -1;
    while (std::getline(in, line))
    {
        if (line.rfind("element=", 0) == 0)
            z = std::stoi(line.substr(8));
        else if (line.rfind("l=", 0) == 0)
        {
            int l = 0, n = 0;
            std::sscanf(line.c_str(), "l=%d n=%d", &l, &n);
            lints::BasisShell sh;
            sh.l_ = l;
            for (int i = 0; i < n; i++)
            {
                std::getline(in, line);
                std::istringstream ss(line);
                double e, c;
                ss >> e >> c;
                sh.exps_.push_back(e);
                sh.coeffs_.push_back(c);
            }
            elems[z].push_back(sh);
        }
    }
    lints::basis_atoms_t atoms;
    for (int zz : Z)
        atoms.push_back({zz, elems.at(zz)});
    return atoms;
}

static int failures = 0;

static void report(const char *what, double err, double tol = 1e-12)
{
    std::printf("%-40s max |diff| = %.3e %s\n", what, err, err <= tol ? "ok" : "FAIL");
    if (!(err <= tol))
        failures++;
}

template <class V>
static double maxDiff(const V &a, const V &b)
{
    if (a.size() != b.size())
        return INFINITY;
    double m = 0;
    for (std::size_t i = 0; i < a.size(); i++)
        m = std::max(m, std::fabs(a.memptr()[i] - b.memptr()[i]));
    return m;
}

int main(int argc, char **argv)
{
    if (argc != 2)
    {
        std::fprintf(stderr, "usage: test_dropin <lible_b200/basis directory>\n");
        return 2;
    }
    const std::string root = argv[1];
    try
    {
        // O3 / def2-SVP + def2-universal-jkfit, Angstrom (the reference's golden molecule)
        const std::vector<int> Z3 = {8, 8, 8};
        const std::vector<std::array<double, 3>> X3 = {{0, 0, 0}, {0, 1, 1}, {0, 0, 2}};
        lints::Structure s3(readBasis(root + "/main/ahlrichs/def2-svp.txt", Z3),
                            readBasis(root + "/aux/ahlrichs/def2-universal-jkfit.txt", Z3), Z3, X3);
        lints::gpu::Context c3(s3);

        report("eri4(Structure)", maxDiff(lints::gpu::eri4(s3), lints::eri4(s3)));
        report("eri4Diagonal(Structure)", maxDiff(lints::gpu::eri4Diagonal(c3), lints::eri4Diagonal(s3)));
        report("eri3(Structure)", maxDiff(lints::gpu::eri3(c3), lints::eri3(s3)));
        report("eri2(Structure)", maxDiff(lints::gpu::eri2(c3), lints::eri2(s3)));
        {
            auto a = lints::gpu::eri2Diagonal(c3), b = lints::eri2Diagonal(s3);
            double m = a.size() == b.size() ? 0 : INFINITY;
            for (std::size_t i = 0; i < std::min(a.size(), b.size()); i++)
                m = std::max(m, std::fabs(a[i] - b[i]));
            report("eri2Diagonal(Structure)", m);
        }

        // kernel functors over every pair combination of a few class pairs
        auto sp = lints::shellPairData(true, s3);
        auto sh = lints::shellDataAux(s3);
        double e4 = 0, e4d = 0, e3 = 0, e3d = 0, e2 = 0, e2d = 0;
        for (auto [i, j] : std::vector<std::pair<int, int>>{{0, 0}, {2, 1}, {5, 3}, {4, 5}})
        {
            lints::gpu::ERI4Kernel g(c3, sp[i], sp[j]);
            lints::ERI4Kernel r(sp[i], sp[j]);
            lints::gpu::ERI4D1Kernel gd(c3, sp[i], sp[j]);
            lints::ERI4D1Kernel rd(sp[i], sp[j]);
            for (std::size_t p = 0; p < sp[i].n_pairs_; p++)
                for (std::size_t q = 0; q < sp[j].n_pairs_; q++)
                {
                    e4 = std::max(e4, maxDiff(g(p, q, sp[i], sp[j]), r(p, q, sp[i], sp[j])));
                    auto bg = gd(p, q, sp[i], sp[j]);
                    auto br = rd(p, q, sp[i], sp[j]);
                    for (int k = 0; k < 12; k++)
                        e4d = std::max(e4d, maxDiff(bg[k], br[k]));
                }
        }
        for (std::size_t i = 0; i < sp.size(); i += 2)
            for (std::size_t x = 0; x < sh.size(); x += 2)
            {
                lints::gpu::ERI3Kernel g(c3, sp[i], sh[x]);
                lints::ERI3Kernel r(sp[i], sh[x]);
                lints::gpu::ERI3D1Kernel gd(c3, sp[i], sh[x]);
                lints::ERI3D1Kernel rd(sp[i], sh[x]);
                for (std::size_t p = 0; p < sp[i].n_pairs_; p++)
                    for (std::size_t q = 0; q < sh[x].n_shells_; q += 3)
                    {
                        e3 = std::max(e3, maxDiff(g(p, q, sp[i], sh[x]), r(p, q, sp[i], sh[x])));
                        auto bg = gd(p, q, sp[i], sh[x]);
                        auto br = rd(p, q, sp[i], sh[x]);
                        for (int k = 0; k < 9; k++)
                            e3d = std::max(e3d, maxDiff(bg[k], br[k]));
                    }
            }
        for (std::size_t a = 0; a < sh.size(); a += 2)
            for (std::size_t b = 0; b < sh.size(); b += 3)
            {
                lints::gpu::ERI2Kernel g(c3, sh[a], sh[b]);
                lints::ERI2Kernel r(sh[a], sh[b]);
                lints::gpu::ERI2D1Kernel gd(c3, sh[a], sh[b]);
                lints::ERI2D1Kernel rd(sh[a], sh[b]);
                for (std::size_t p = 0; p < sh[a].n_shells_; p += 2)
                    for (std::size_t q = 0; q < sh[b].n_shells_; q += 2)
                    {
                        e2 = std::max(e2, maxDiff(g(p, q, sh[a], sh[b]), r(p, q, sh[a], sh[b])));
                        auto bg = gd(p, q, sh[a], sh[b]);
                        auto br = rd(p, q, sh[a], sh[b]);
                        for (int k = 0; k < 6; k++)
                            e2d = std::max(e2d, maxDiff(bg[k], br[k]));
                    }
            }
        report("ERI4Kernel::operator()", e4);
        report("ERI4D1Kernel::operator()", e4d, 1e-11);
        report("ERI3Kernel::operator()", e3);
        report("ERI3D1Kernel::operator()", e3d, 1e-11);
        report("ERI2Kernel::operator()", e2);
        report("ERI2D1Kernel::operator()", e2d, 1e-11);

        // water / cc-pVDZ through the one-call form (context made and dropped inside)
        const std::vector<int> Zw = {8, 1, 1};
        const std::vector<std::array<double, 3>> Xw = {{0, 0, 0}, {0.757, 0.586, 0}, {-0.757, 0.586, 0}};
        lints::Structure sw(readBasis(root + "/main/dunning/cc-pvdz.txt", Zw), Zw, Xw);
        report("eri4(Structure), water cc-pVDZ", maxDiff(lints::gpu::eri4(sw), lints::eri4(sw)));

        // one-electron drivers: CO2 / 6-31+G (the reference's erf-attenuated test molecule) and
        // ethane / cc-pVDZ (its dipole test molecule), Angstrom
        const std::vector<int> Zc = {6, 8, 8};
        const std::vector<std::array<double, 3>> Xc = {{0, 0, 0.32942}, {0, 1.15362, -0.12353},
                                                       {0, -1.15362, -0.12353}};
        lints::Structure sc(readBasis(root + "/main/pople/6-31+g.txt", Zc), Zc, Xc);
        lints::gpu::Context cc(sc);
        report("overlap(Structure)", maxDiff(lints::gpu::overlap(cc), lints::overlap(sc)));
        report("kineticEnergy(Structure)", maxDiff(lints::gpu::kineticEnergy(cc), lints::kineticEnergy(sc)));
        report("nuclearAttraction(Structure)", maxDiff(lints::gpu::nuclearAttraction(cc), lints::nuclearAttraction(sc)));
        const std::vector<double> om = {0.0035, -0.5, 0.6};
        report("nuclearAttractionErf(Structure)",
               maxDiff(lints::gpu::nuclearAttractionErf(cc, om), lints::nuclearAttractionErf(sc, om)));
        const std::vector<std::array<double, 4>> q = {{1.0, -2.0, 0.5, 0.7}, {-3.0, 1.0, -6.0, -1.2}};
        const std::vector<double> oq = {1.2, -10.5};
        report("externalCharges(Structure)", maxDiff(lints::gpu::externalCharges(q, cc), lints::externalCharges(q, sc)));
        report("externalChargesErf(Structure)",
               maxDiff(lints::gpu::externalChargesErf(q, oq, cc), lints::externalChargesErf(q, oq, sc)));
        const std::vector<int> Ze = {1, 6, 1, 1, 6, 1, 1, 1};
        const std::vector<std::array<double, 3>> Xe = {{1.1851, -0.0039, 0.9875}, {0.7516, -0.0225, -0.0209},
                                                       {1.1669, 0.8330, -0.5693}, {1.1155, -0.9329, -0.5145},
                                                       {-0.7516, 0.0225, 0.0209}, {-1.1669, -0.8334, 0.5687},
                                                       {-1.1157, 0.9326, 0.5151}, {-1.1850, 0.0044, -0.9875}};
        lints::Structure se(readBasis(root + "/main/dunning/cc-pvdz.txt", Ze), Ze, Xe);
        lints::gpu::Context ce(se);
        const std::array<double, 3> o = {0.3, -0.2, 0.5};
        const auto dg = lints::gpu::dipoleMoment(o, ce), dr = lints::dipoleMoment(o, se);
        const auto ag = lints::gpu::angularMomentum(o, ce), ar = lints::angularMomentum(o, se);
        double dd = 0, da = 0;
        for (int k = 0; k < 3; k++)
        {
            dd = std::max(dd, maxDiff(dg[k], dr[k]));
            da = std::max(da, maxDiff(ag[k], ar[k]));
        }
        report("dipoleMoment(origin, Structure)", dd);
        report("angularMomentum(origin, Structure)", da);
        const auto sg = lints::gpu::spinOrbitCoupling1El(ce), sr = lints::spinOrbitCoupling1El(se);
        double ds = 0;
        for (int k = 0; k < 3; k++)
            ds = std::max(ds, maxDiff(sg[k], sr[k]));
        report("spinOrbitCoupling1El(Structure)", ds);
    }
    catch (const std::exception &e)
    {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    std::printf("%s\n", failures ? "FAILED" : "all ok");
    return failures ? 1 : 0;
}
