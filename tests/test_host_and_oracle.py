"""CPU tests: the oracle against the reference's golden vectors and the reference itself, the
engine's host-side set-up against the reference, and the C ABI's exported symbol set.

Golden sums are the reference's own test constants (test/tests_ints.cpp), compared at 1e-13
relative (see tests/test_gpu_eri.py for why); element-wise comparisons are absolute."""
import ctypes
import os
import re

import numpy as np
import pytest

from lible_b200 import _lib
from lible_b200.workloads import WATER_BOHR, WATER_Z, random_density, water_cluster
from oracle import port, ref

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
O3_BOHR = np.array([[0, 0, 0], [0, 1, 1], [0, 0, 2]], float) / 0.5291772083
needs_ref = pytest.mark.skipif(not ref.available(), reason="reference library not built")


def seqsum(x):
    return float(np.cumsum(np.abs(np.asarray(x)).ravel())[-1])


def test_capi_exports_every_declared_symbol():
    header = open(os.path.join(ROOT, "include", "lible_b200.h")).read()
    declared = set(re.findall(r"\b(lible_(?:gpu|host)_\w+)\s*\(", header))
    assert len(declared) >= 30
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python mirror declares a signature for each of them
    assert declared - {"lible_gpu_last_error"} <= set(_lib.SIGNATURES)


def test_port_boys_golden():
    # calcBoysF(n=5, x=2.5), sum of values: test/tests_ints.cpp:1296-1313
    assert abs(seqsum(port.boys(5, 2.5)) - 0.728561124180) < 1e-12


def test_host_boys_matches_port_and_golden():
    lib = _lib.load()
    for n, x in [(5, 2.5), (0, 0.0), (8, 1e-3), (12, 17.3), (13, 29.999), (4, 31.0), (10, 250.0)]:
        F = np.empty(n + 1)
        assert lib.lible_host_boys(n, x, F.ctypes.data) == 0
        assert np.allclose(F, port.boys(n, x), rtol=1e-14, atol=1e-300)
    F = np.empty(6)
    lib.lible_host_boys(5, 2.5, F.ctypes.data)
    assert abs(seqsum(F) - 0.728561124180) < 1e-12


def test_host_spherical_trafo_golden():
    # sphericalTrafo(8): sum |val| + i + j = 7005.923248093791 (test/tests_ints.cpp:856-871)
    lib = _lib.load()
    n = ctypes.c_int(1000)
    rows, carts, vals = np.zeros(1000, np.int32), np.zeros(1000, np.int32), np.zeros(1000)
    assert lib.lible_host_spherical_trafo(8, ctypes.byref(n), rows.ctypes.data, carts.ctypes.data,
                                          vals.ctypes.data) == 0
    k = n.value
    assert abs(np.sum(np.abs(vals[:k]) + rows[:k] + carts[:k]) - 7005.923248093791) < 1e-9


def test_host_shell_norms_normalise_overlap():
    # A normalised contracted s shell: cc-pVDZ O 1s coefficients (norm close to 1 by construction)
    lib = _lib.load()
    atoms = port.read_basis("cc-pvdz", [8])[0]
    for l, e, c in atoms:
        norms = np.empty(2 * l + 1)
        assert lib.lible_host_shell_norms(l, len(e), np.asarray(e).ctypes.data, np.asarray(c).ctypes.data,
                                          norms.ctypes.data) == 0
        assert np.all(norms > 0.5) and np.all(norms < 3.0)


@needs_ref
@pytest.mark.parametrize("basis,Z,xyz", [("def2-svp", [8, 8, 8], O3_BOHR), ("cc-pvtz", WATER_Z, WATER_BOHR)])
def test_host_pair_classes_match_reference(basis, Z, xyz):
    lib = _lib.load()
    r = ref.RefStructure(basis, Z, xyz)
    for use_symm in (0, 1):
        n = ctypes.c_int()
        ls = np.zeros(64, np.int32)
        npr, npp = np.zeros(32, np.int64), np.zeros(32, np.int64)
        Zs = np.asarray(Z, np.int32)
        x = np.ascontiguousarray(xyz, float)
        assert lib.lible_host_pair_classes(os.path.join(ROOT, "lible_b200", "basis", "main").encode(), basis.encode(),
                                           len(Z), Zs.ctypes.data, x.ctypes.data, 1, use_symm, ctypes.byref(n),
                                           ls.ctypes.data, npr.ctypes.data, npp.ctypes.data) == 0
        mine = [(int(ls[2 * i]), int(ls[2 * i + 1]), int(npr[i]), int(npp[i])) for i in range(n.value)]
        assert mine == r.pair_classes(bool(use_symm))


@needs_ref
def test_reference_golden_sums():
    r = ref.RefStructure("def2-svp", [8, 8, 8], O3_BOHR)
    assert abs(seqsum(r.eri4()) - 8246.711763196334) < 1e-12
    assert abs(r.deploy_sum(0) - 8246.711763197583) < 1e-12


def test_port_golden_eri4_o3():
    V = port.PortMolecule("def2-svp", [8, 8, 8], O3_BOHR).eri4()
    assert abs(seqsum(V) - 8246.711763196334) <= 1e-13 * 8246.711763196334


@needs_ref
def test_port_matches_reference_elementwise():
    V = port.PortMolecule("cc-pvdz", WATER_Z, WATER_BOHR).eri4()
    Vr = ref.RefStructure("cc-pvdz", WATER_Z, WATER_BOHR).eri4()
    assert np.abs(V - Vr).max() <= 1e-12


@needs_ref
def test_port_jk_and_gradient_match_reference():
    Z, xyz, rng = water_cluster(2, seed=5)
    D = random_density(48, 10, rng)
    m = port.PortMolecule("cc-pvdz", Z, xyz)
    r = ref.RefStructure("cc-pvdz", Z, xyz)
    J, K, nq = m.jk(D, 1e-12)
    Jr, Kr, nqr, _ = r.jk(D, 1e-12)
    assert nq == nqr
    assert np.abs(J - Jr).max() <= 1e-11 and np.abs(K - Kr).max() <= 1e-11
    assert np.abs(m.jk_grad(D) - r.jk_grad(D)).max() <= 1e-11


def test_port_gradient_matches_finite_differences():
    Z, xyz, rng = water_cluster(1, seed=9)
    D = random_density(24, 5, rng)
    g = port.PortMolecule("cc-pvdz", Z, xyz).jk_grad(D)
    h = 1e-4

    def energy(c):
        J, K, _ = port.PortMolecule("cc-pvdz", Z, c).jk(D, 0.0)
        return float(np.sum(D * (0.5 * J - 0.25 * K)))

    for atom, x in [(0, 1), (2, 0)]:
        cp, cm = xyz.copy(), xyz.copy()
        cp[atom, x] += h
        cm[atom, x] -= h
        assert abs((energy(cp) - energy(cm)) / (2 * h) - g[atom, x]) <= 1e-6


def test_water_cluster_generator_is_seeded():
    Z1, x1, _ = water_cluster(32, 2024)
    Z2, x2, _ = water_cluster(32, 2024)
    assert Z1 == Z2 and np.array_equal(x1, x2)
    assert len(Z1) == 96
    # rigid waters: O-H distances preserved
    d = np.linalg.norm(x1[1::3] - x1[0::3], axis=1)
    assert np.allclose(d, np.linalg.norm([1.4305, 1.1093, 0.0]))


@needs_ref
def test_reference_one_electron_golden():
    # the compiled reference reproduces its own one-electron golden sums
    # (test/tests_ints.cpp:167-182, 236-251, 303-318); these pin the one-electron oracle
    c2h4 = [[3.402, 0.773, -9.252], [4.697, 0.791, -8.909], [2.933, -0.150, -9.521],
            [2.837, 1.682, -9.258], [5.262, -0.118, -8.904], [5.167, 1.714, -8.641]]
    r = ref.RefStructure("cc-pvdz", [6, 6, 1, 1, 1, 1], c2h4, units="angstrom")
    assert abs(seqsum(r.one_electron(0)) - 226.099184393591) <= 1e-13 * 226.1
    assert abs(seqsum(r.one_electron(1)) - 252.755644635021) <= 1e-13 * 252.8
    co2 = [[0.0, 0.0, 0.32942], [0.0, 1.15362, -0.12353], [0.0, -1.15362, -0.12353]]
    r2 = ref.RefStructure("6-31+g", [6, 8, 8], co2, units="angstrom")
    V = r2.one_electron(2)
    assert abs(seqsum(V) - 2141.927982294058) <= 1e-13 * 2141.9
    q = np.array([[x / 0.5291772083 for x in c] + [z] for c, z in zip(co2, [6, 8, 8])])
    assert np.abs(r2.one_electron(3, q) - V).max() <= 1e-13


@needs_ref
def test_reference_multipole_and_erf_golden():
    # the compiled reference reproduces its dipole-moment and erf-attenuated golden sums
    # (test/tests_ints.cpp:321-338, 360-379, 597-614); these pin the oracle of those operators
    co2 = [[0.0, 0.0, 0.32942], [0.0, 1.15362, -0.12353], [0.0, -1.15362, -0.12353]]
    r = ref.RefStructure("6-31+g", [6, 8, 8], co2, units="angstrom")
    assert abs(seqsum(r.one_electron_ex(7, omegas=[0.0035, -0.5, 0.6])) - 257.523987741588) <= 1e-13 * 257.5
    q = np.array([[x / 0.5291772083 for x in c] + [z] for c, z in zip(co2, [6, 8, 8])])
    Vq = r.one_electron_ex(8, charges=q, omegas=[1.2, -10.5, 0.031])
    assert abs(seqsum(Vq) - 419.197077258843) <= 1e-13 * 419.2
    c2h6 = [[1.1851, -0.0039, 0.9875], [0.7516, -0.0225, -0.0209], [1.1669, 0.8330, -0.5693],
            [1.1155, -0.9329, -0.5145], [-0.7516, 0.0225, 0.0209], [-1.1669, -0.8334, 0.5687],
            [-1.1157, 0.9326, 0.5151], [-1.1850, 0.0044, -0.9875]]
    r2 = ref.RefStructure("cc-pvdz", [1, 6, 1, 1, 6, 1, 1, 1], c2h6, units="angstrom")
    assert abs(seqsum(r2.one_electron_ex(4, origin=[0.0, 0.0, 0.0])) - 1205.074870756679) <= 1e-13 * 1205.1
    # angular momentum is antisymmetric; the momentum driver writes one orientation of each unique
    # pair of different shells only, so its matrices are not
    A = r2.one_electron_ex(6, origin=[0.1, 0.2, 0.3])
    assert np.abs(A + A.transpose(0, 2, 1)).max() <= 1e-14 * np.abs(A).max()
    P = r2.one_electron_ex(5)
    assert np.abs(P + P.transpose(0, 2, 1)).max() > 0.1 * np.abs(P).max()


@needs_ref
def test_reference_soc_and_d2_golden():
    # the compiled reference reproduces its ERI4SOC / ERI3SOC / ERI2D2 kernel golden sums
    # (test/tests_ints.cpp:1055-1150) through the oracle's per-class wrappers
    o3 = [[0, 0, 0], [0, 1, 1], [0, 0, 2]]
    r = ref.RefStructure("def2-svp", [8, 8, 8], o3, aux="def2-universal-jkfit", units="angstrom")
    nc, na = len(r.pair_classes(False)), len(r.aux_classes())

    def total(blocks):
        return seqsum(np.concatenate([np.ravel(b) for b in blocks]))

    assert abs(total(r.eri4soc_class(False, i, j) for i in range(nc) for j in range(nc)) -
               12940.953099658431) <= 1e-13 * 12940.95
    assert abs(total(r.eri3soc_class(False, i, j) for i in range(nc) for j in range(na)) -
               18124.713152990007) <= 1e-13 * 18124.71
    assert abs(total(r.eri2d2_class(i, j) for i in range(na) for j in range(na)) -
               175567.635699242965) <= 1e-13 * 175567.6
