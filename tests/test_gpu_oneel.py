"""One-electron integrals through the C ABI against the reference's own overlap / kineticEnergy /
nuclearAttraction / externalCharges (oracle/_ref) and its golden sums
(test/tests_ints.cpp:167-358: C2H4 cc-pVDZ overlap and kinetic energy, CO2 6-31+G nuclear
attraction and external charges).  Tolerances: 1e-12 absolute per element (the reference's test
tolerance, test/tests_ints.cpp:15); golden sums to 1e-13 relative."""
import numpy as np
import pytest

from lible_b200 import ints as L
from lible_b200.workloads import water_cluster
from oracle import ref as R

pytestmark = pytest.mark.gpu

C2H4_Z = [6, 6, 1, 1, 1, 1]
C2H4_ANG = [[3.402, 0.773, -9.252], [4.697, 0.791, -8.909], [2.933, -0.150, -9.521],
            [2.837, 1.682, -9.258], [5.262, -0.118, -8.904], [5.167, 1.714, -8.641]]
CO2_Z = [6, 8, 8]
CO2_ANG = [[0.0, 0.0, 0.32942], [0.0, 1.15362, -0.12353], [0.0, -1.15362, -0.12353]]


def seqsum(x):
    return float(np.cumsum(np.abs(np.asarray(x)).ravel())[-1])


def golden(value, expected):
    return abs(value - expected) <= 1e-13 * abs(expected)


def test_overlap_and_kinetic_golden_c2h4():
    s = L.Structure("cc-pvdz", C2H4_Z, C2H4_ANG)
    r = R.RefStructure("cc-pvdz", C2H4_Z, C2H4_ANG, units="angstrom")
    S, T = L.overlap(s), L.kineticEnergy(s)
    assert golden(seqsum(S), 226.099184393591)
    assert golden(seqsum(T), 252.755644635021)
    assert np.abs(S - r.one_electron(0)).max() <= 1e-12
    assert np.abs(T - r.one_electron(1)).max() <= 1e-12


def test_nuclear_attraction_and_external_charges_golden_co2():
    s = L.Structure("6-31+g", CO2_Z, CO2_ANG)
    r = R.RefStructure("6-31+g", CO2_Z, CO2_ANG, units="angstrom")
    V = L.nuclearAttraction(s)
    assert golden(seqsum(V), 2141.927982294058)
    assert np.abs(V - r.one_electron(2)).max() <= 1e-12
    # the nuclei as explicit charges (structure.getZs() in the reference test)
    q = np.array([[x / 0.5291772083 for x in c] + [z] for c, z in zip(CO2_ANG, CO2_Z)])
    Vq = L.externalCharges(q, s)
    assert golden(seqsum(Vq), 2141.927982294058)
    assert np.abs(Vq - V).max() <= 1e-12


def test_one_electron_f_shells_and_random_charges_vs_reference():
    # cc-pVTZ water dimer: f shells on O (the l <= 3 limit), 200 random point charges
    Z, xyz, rng = water_cluster(2, 5)
    s = L.Structure("cc-pvtz", Z, xyz, units="bohr")
    r = R.RefStructure("cc-pvtz", Z, xyz)
    q = np.concatenate([rng.uniform(-8, 8, (200, 3)), rng.uniform(-1, 1, (200, 1))], axis=1)
    S, T, V = L.one_electron(s)
    assert np.abs(S - r.one_electron(0)).max() <= 1e-12
    assert np.abs(T - r.one_electron(1)).max() <= 1e-12
    assert np.abs(V - r.one_electron(2)).max() <= 1e-11 * max(1.0, np.abs(V).max())
    Vq = L.externalCharges(q, s)
    assert np.abs(Vq - r.one_electron(3, q)).max() <= 1e-12 * max(1.0, np.abs(Vq).max())
    assert np.abs(L.externalCharges(np.zeros((0, 4)), s)).max() == 0.0
    # symmetric (diagonal shell blocks are written from both orientations, as in the reference, so
    # to the last bit only), and the same matrices as the single-operator calls
    assert np.abs(S - S.T).max() <= 1e-15 and np.abs(L.overlap(s) - S).max() == 0.0


def _kernel_blocks(structure, use_symm, fn, *args):
    parts = []
    for sp in L.shellPairData(use_symm, structure):
        if sp.n_pairs_:
            parts.append(np.asarray(fn(list(range(sp.n_pairs_)), *args, sp)).ravel())
    return np.concatenate(parts)


def test_per_pair_kernels_golden():
    # the reference's kernel-API golden sums (test/tests_ints.cpp:185-300, 381-480): blocks summed
    # in class / pair / [derivative] / element order, as the reference's loops do
    c2h4 = L.Structure("cc-pvdz", C2H4_Z, C2H4_ANG)
    assert golden(seqsum(_kernel_blocks(c2h4, True, L.overlapKernel)), 137.049592196795)
    assert golden(seqsum(_kernel_blocks(c2h4, False, L.overlapD1Kernel)), 712.697494155785)
    assert golden(seqsum(_kernel_blocks(c2h4, False, L.kineticEnergyKernel)), 252.755644635020)
    assert golden(seqsum(_kernel_blocks(c2h4, False, L.kineticEnergyD1Kernel)), 1153.592041307799)
    co2 = L.Structure("6-31+g", CO2_Z, CO2_ANG)
    q = np.array([[x / 0.5291772083 for x in c] + [z] for c, z in zip(CO2_ANG, CO2_Z)])
    assert golden(seqsum(_kernel_blocks(co2, True, L.externalChargesKernel, q)), 1338.606063918550)
    assert golden(seqsum(_kernel_blocks(co2, True, L.externalChargesD1Kernel, q)), 3274.419345348923)
    # a single pair returns the block, or the list of six derivative blocks
    sp = L.shellPairData(True, c2h4)[0]
    assert np.abs(L.overlapKernel(0, sp) - L.overlapKernel([0], sp)[0]).max() == 0.0
    assert len(L.overlapD1Kernel(0, sp)) == 6


def test_one_electron_gradient_vs_finite_differences():
    """d/dR (sum D (T + V) - sum W S) against central differences (step 1e-4 bohr) of the forward
    integrals, cc-pVDZ and cc-pVTZ (f shells); translational invariance of the total."""
    for basis, nw, seed in (("cc-pvdz", 2, 3), ("cc-pvtz", 1, 8)):
        Z, xyz, rng = water_cluster(nw, seed)
        s = L.Structure(basis, Z, xyz, units="bohr")
        n = s.nao
        C = np.linalg.qr(rng.standard_normal((n, 5 * nw)))[0]
        D = C @ C.T
        X = rng.standard_normal((n, n)) * 0.1
        W = X + X.T
        g = L.one_electron_grad(s, D, W)
        assert np.abs(g.sum(axis=0)).max() <= 1e-9 * max(1.0, np.abs(g).max())

        def energy(c):
            S, T, V = L.one_electron(L.Structure(basis, Z, c, units="bohr"))
            return float(np.sum(D * (T + V)) - np.sum(W * S))

        h = 1e-4
        for atom, x in ((0, 0), (1, 1), (len(Z) - 1, 2)):
            cp, cm = xyz.copy(), xyz.copy()
            cp[atom, x] += h
            cm[atom, x] -= h
            fd = (energy(cp) - energy(cm)) / (2 * h)
            assert abs(fd - g[atom, x]) <= 1e-6 * max(1.0, abs(fd)), (basis, atom, x, fd, g[atom, x])
        # the D and W terms separately add up to the whole
        assert np.abs(L.one_electron_grad(s, D, None) + L.one_electron_grad(s, None, W) - g).max() <= 1e-10


def test_per_pair_kernels_vs_reference_elementwise():
    # every class of shellPairData with and without symmetry (la < lb classes included), all six
    # operators, against the reference's own per-pair kernels
    s = L.Structure("cc-pvdz", C2H4_Z, C2H4_ANG)
    r = R.RefStructure("cc-pvdz", C2H4_Z, C2H4_ANG, units="angstrom")
    q = np.array([[1.0, -2.0, 0.5, 0.7], [-3.0, 1.0, -16.0, -1.2], [6.0, 2.0, -17.0, 2.0]])
    fns = [L.overlapKernel, L.kineticEnergyKernel, L.externalChargesKernel, L.overlapD1Kernel,
           L.kineticEnergyD1Kernel, L.externalChargesD1Kernel]
    for use_symm in (True, False):
        for i, sp in enumerate(L.shellPairData(use_symm, s)):
            idx = list(range(sp.n_pairs_))
            for op, fn in enumerate(fns):
                got = fn(idx, q, sp) if op in (2, 5) else fn(idx, sp)
                want = r.one_electron_class(use_symm, i, op, q if op in (2, 5) else None)
                assert np.abs(got - want.reshape(got.shape)).max() <= 1e-12 * max(1.0, np.abs(want).max()), \
                    (use_symm, i, op)


C2H6_Z = [1, 6, 1, 1, 6, 1, 1, 1]
C2H6_ANG = [[1.1851, -0.0039, 0.9875], [0.7516, -0.0225, -0.0209], [1.1669, 0.8330, -0.5693],
            [1.1155, -0.9329, -0.5145], [-0.7516, 0.0225, 0.0209], [-1.1669, -0.8334, 0.5687],
            [-1.1157, 0.9326, 0.5151], [-1.1850, 0.0044, -0.9875]]


def test_dipole_moment_golden_c2h6_and_vs_reference():
    """dipoleMoment about the origin: the reference's golden sum (test/tests_ints.cpp:597-614, ethane
    cc-pVDZ) and element-wise against the reference's driver; about another origin too."""
    s = L.Structure("cc-pvdz", C2H6_Z, C2H6_ANG)
    r = R.RefStructure("cc-pvdz", C2H6_Z, C2H6_ANG, units="angstrom")
    M = L.dipoleMoment([0.0, 0.0, 0.0], s)
    assert golden(seqsum(M), 1205.074870756679)
    assert np.abs(M - r.one_electron_ex(4, origin=[0.0, 0.0, 0.0])).max() <= 1e-12
    o = [0.3, -1.2, 0.7]
    Mo = L.dipoleMoment(o, s)
    assert np.abs(Mo - r.one_electron_ex(4, origin=o)).max() <= 1e-12 * max(1.0, np.abs(Mo).max())
    assert np.abs(Mo - Mo.transpose(0, 2, 1)).max() <= 1e-15 * max(1.0, np.abs(Mo).max())


def test_erf_attenuated_attraction_golden_co2_and_vs_reference():
    """nuclearAttractionErf and externalChargesErf with the reference test's range parameters
    (negative ones included; test/tests_ints.cpp:321-338, 360-379): golden sums and element-wise
    against the reference's drivers."""
    s = L.Structure("6-31+g", CO2_Z, CO2_ANG)
    r = R.RefStructure("6-31+g", CO2_Z, CO2_ANG, units="angstrom")
    w = [0.0035, -0.5, 0.6]
    V = L.nuclearAttractionErf(s, w)
    assert golden(seqsum(V), 257.523987741588)
    assert np.abs(V - r.one_electron_ex(7, omegas=w)).max() <= 1e-12
    q = np.array([[x / 0.5291772083 for x in c] + [z] for c, z in zip(CO2_ANG, CO2_Z)])
    wq = [1.2, -10.5, 0.031]
    Vq = L.externalChargesErf(q, wq, s)
    assert golden(seqsum(Vq), 419.197077258843)
    assert np.abs(Vq - r.one_electron_ex(8, charges=q, omegas=wq)).max() <= 1e-12
    with pytest.raises(ValueError):
        L.nuclearAttractionErf(s, [0.5])


def test_momentum_and_angular_momentum_vs_reference():
    """Water dimer cc-pVTZ (f shells).  angularMomentum: element-wise against the reference's driver
    (antisymmetric).  momentum: the reference's driver (oneelints.cpp:1477-1511) writes only the
    (a, b) blocks of its unique pairs, negated; every element it writes off the diagonal equals the
    transposed element of the full antisymmetric matrix returned here, and its diagonal the diagonal."""
    Z, xyz, rng = water_cluster(2, 5)
    s = L.Structure("cc-pvtz", Z, xyz, units="bohr")
    r = R.RefStructure("cc-pvtz", Z, xyz)
    o = [0.4, 0.1, -0.8]
    A = L.angularMomentum(o, s)
    Ar = r.one_electron_ex(6, origin=o)
    scale = max(1.0, np.abs(Ar).max())
    assert np.abs(A - Ar).max() <= 1e-12 * scale
    assert np.abs(A + A.transpose(0, 2, 1)).max() <= 1e-15 * scale
    P = L.momentum(s)
    Pr = r.one_electron_ex(5)
    assert np.abs(P + P.transpose(0, 2, 1)).max() == 0.0
    n = s.nao
    written = Pr != 0.0
    off = written & ~np.eye(n, dtype=bool)[None]
    assert off.sum() > n * n  # the upper blocks of the unique pairs
    assert np.abs((Pr - P.transpose(0, 2, 1))[off]).max() <= 1e-12 * max(1.0, np.abs(P).max())
    assert np.abs(np.diagonal(P, axis1=1, axis2=2)).max() == 0.0


def test_spin_orbit_coupling_1el_vs_reference():
    """spinOrbitCoupling1El of the nuclei against the reference's driver, which evaluates every
    ordered shell pair (ethane cc-pVDZ, cc-pVTZ water dimer); the matrices are antisymmetric."""
    Z2, xyz2, _ = water_cluster(2, 7)
    for s, r in ((L.Structure("cc-pvdz", C2H6_Z, C2H6_ANG), R.RefStructure("cc-pvdz", C2H6_Z, C2H6_ANG, units="angstrom")),
                 (L.Structure("cc-pvtz", Z2, xyz2, units="bohr"), R.RefStructure("cc-pvtz", Z2, xyz2))):
        M, Mr = L.spinOrbitCoupling1El(s), r.one_electron_ex(9)
        scale = max(1.0, np.abs(Mr).max())
        assert np.abs(M - Mr).max() <= 1e-12 * scale
        assert np.abs(M + M.transpose(0, 2, 1)).max() == 0.0


def test_new_per_pair_kernels_vs_reference_elementwise():
    """dipoleMomentKernel, momentumKernel, angularMomentumKernel and externalChargesErfKernel for every
    class with and without symmetry (la < lb classes, stored swapped, included) against the
    reference's kernels; ethane cc-pVDZ and a cc-pVTZ water dimer."""
    q = np.array([[1.0, -2.0, 0.5, 0.7], [-3.0, 1.0, -6.0, -1.2], [6.0, 2.0, -7.0, 2.0]])
    w = np.array([0.4, -2.5, 11.0])
    o = [0.2, -0.4, 0.9]
    Z2, xyz2, _ = water_cluster(2, 7)
    cases = [(L.Structure("cc-pvdz", C2H6_Z, C2H6_ANG), R.RefStructure("cc-pvdz", C2H6_Z, C2H6_ANG, units="angstrom")),
             (L.Structure("cc-pvtz", Z2, xyz2, units="bohr"), R.RefStructure("cc-pvtz", Z2, xyz2))]
    for s, r in cases:
        for use_symm in (True, False):
            for i, sp in enumerate(L.shellPairData(use_symm, s)):
                if not sp.n_pairs_:
                    continue
                idx = list(range(sp.n_pairs_))
                for op, got in ((6, L.dipoleMomentKernel(idx, o, sp)), (7, L.momentumKernel(idx, sp)),
                                (8, L.angularMomentumKernel(idx, o, sp)),
                                (9, L.externalChargesErfKernel(idx, q, w, sp)),
                                (15, L.spinOrbitCoupling1ElKernel(idx, q, sp))):
                    want = r.one_electron_class_ex(use_symm, i, op, charges=q, omegas=w, origin=o)
                    assert np.abs(got - want.reshape(got.shape)).max() <= 1e-12 * max(1.0, np.abs(want).max()), \
                        (use_symm, i, op)
    # a single pair returns the three blocks
    sp = L.shellPairData(True, cases[0][0])[0]
    assert len(L.momentumKernel(0, sp)) == 3


def test_charge_kernels_golden_co2():
    """The reference's kernel-API golden sums for the attenuated and per-charge Coulomb kernels
    (test/tests_ints.cpp:414-596; CO2 6-31+G), summed in class / pair / charge / component / element
    order as the reference's loops do."""
    co2 = L.Structure("6-31+g", CO2_Z, CO2_ANG)
    q = np.array([[x / 0.5291772083 for x in c] + [z] for c, z in zip(CO2_ANG, CO2_Z)])
    assert golden(seqsum(_kernel_blocks(co2, False, L.externalChargesErfKernel, q, [1.2, -10.5, 0.031])),
                  419.197077258844)
    assert golden(seqsum(_kernel_blocks(co2, True, L.externalChargesOperatorD1Kernel, q)), 1067.752096834267)
    assert golden(seqsum(_kernel_blocks(co2, True, L.potentialAtExternalChargesKernel, q)), 1357.142718060126)
    q4 = np.array([[0.0, -0.025, 0.05, 1.0], [1.0, -0.025, 0.05, -1.0], [-1.0, 0.5, 0.6, 0.25],
                   [0.0, -0.5, 0.24, -0.3]])
    assert golden(seqsum(_kernel_blocks(co2, True, L.potentialAtExternalChargesErfKernel, q4,
                                        [0.1, -0.5, 0.61, 0.000015])), 66.950210612294)


def test_charge_kernels_vs_reference_elementwise():
    """externalChargesErfD1Kernel, externalChargesOperator(Erf)D1Kernel and
    potentialAtExternalCharges(Erf)Kernel for every class with and without symmetry against the
    reference's kernels (cc-pVTZ water dimer, f shells; three charges with range parameters)."""
    q = np.array([[1.0, -2.0, 0.5, 0.7], [-3.0, 1.0, -6.0, -1.2], [6.0, 2.0, -7.0, 2.0]])
    w = np.array([0.4, -2.5, 11.0])
    Z, xyz, _ = water_cluster(2, 7)
    s, r = L.Structure("cc-pvtz", Z, xyz, units="bohr"), R.RefStructure("cc-pvtz", Z, xyz)
    for use_symm in (True, False):
        for i, sp in enumerate(L.shellPairData(use_symm, s)):
            if not sp.n_pairs_:
                continue
            idx = list(range(sp.n_pairs_))
            for op, got in ((10, L.externalChargesErfD1Kernel(idx, q, w, sp)),
                            (11, L.externalChargesOperatorD1Kernel(idx, q, sp)),
                            (12, L.externalChargesOperatorErfD1Kernel(idx, q, w, sp)),
                            (13, L.potentialAtExternalChargesKernel(idx, q, sp)),
                            (14, L.potentialAtExternalChargesErfKernel(idx, q, w, sp))):
                want = r.one_electron_class_ex(use_symm, i, op, charges=q, omegas=w)
                got = np.asarray(got)
                assert np.abs(got.reshape(want.shape) - want).max() <= 1e-12 * max(1.0, np.abs(want).max()), \
                    (use_symm, i, op)


def test_pvp_against_finite_differences_of_charge_integrals():
    """pVp_ij(m, n) = <d_i m| V |d_j n> = d^2 V_mn / dA_i dB_j for m on atom A and n on atom B != A,
    with the point charges held fixed: central finite differences (step 1e-3 bohr, four displaced
    geometries per (i, j)) of externalCharges on an O-H pair in cc-pVDZ (s, p and d functions),
    to 2e-6 of the largest element.  The whole-matrix form satisfies pVp[i][j] = pVp[j][i]^T and
    matches the per-pair kernel blocks."""
    Z = [8, 1]
    X0 = np.array([[0.1, -0.2, 0.05], [0.3, 1.1, 1.4]])
    q = np.array([[1.5, 0.4, -0.7, 0.8], [-1.2, 2.0, 1.1, -0.5], [0.4, -1.6, 2.3, 1.3]])
    s = L.Structure("cc-pvdz", Z, X0, units="bohr")
    M = L.pVpIntegrals(s, q)
    assert np.abs(M - M.transpose(1, 0, 3, 2)).max() == 0.0
    n0 = 14  # cc-pVDZ O: 3s 2p 1d = 14 functions, then H
    h = 1e-3

    def V(dA, dB):
        X = X0.copy()
        X[0] += dA
        X[1] += dB
        return L.externalCharges(q, L.Structure("cc-pvdz", Z, X, units="bohr"))

    scale = np.abs(M[:, :, :n0, n0:]).max()
    for i in range(3):
        for j in range(3):
            ei, ej = np.eye(3)[i] * h, np.eye(3)[j] * h
            fd = (V(ei, ej) - V(ei, -ej) - V(-ei, ej) + V(-ei, -ej)) / (4 * h * h)
            assert np.abs(fd[:n0, n0:] - M[i, j, :n0, n0:]).max() <= 2e-6 * scale, (i, j)
    # the per-pair kernel gives the same blocks (first class, every pair)
    sp = L.shellPairData(True, s)[0]
    k = L.pVpKernel(list(range(sp.n_pairs_)), q, sp)
    assert k.shape[1:3] == (3, 3)


def test_pvp_reference_kernel_differs_as_documented():
    """The reference's pVpKernel (oneelints.cpp:1318-1475) does not give the integrals: it leaves out
    the E factor of its first term and the R factor of its last.  Shown here on s-only functions
    (6-31+G hydrogens), where it differs from the finite-difference-checked values of this library,
    while both agree that the integrals are defined per pair and component."""
    Z = [1, 1]
    X = [[0.0, 0.0, 0.0], [0.4, -0.3, 1.3]]
    s, r = L.Structure("6-31+g", Z, X, units="bohr"), R.RefStructure("6-31+g", Z, X)
    q = np.array([[0.7, 0.2, -0.5, 1.0]])
    sp = L.shellPairData(True, s)[0]
    mine = L.pVpKernel(list(range(sp.n_pairs_)), q, sp)
    ref = r.one_electron_class_ex(True, 0, 16, charges=q).reshape(mine.shape)
    assert np.abs(mine - ref).max() > 1e-3 * np.abs(mine).max()
