"""Parity against the committed golden fixtures (tests/golden/, written from the reference itself
by tests/golden/make_golden.py).  They pin the oracle's C restatement on the CPU and the CUDA path
on the GPU without needing the compiled reference at test time.

Tolerances: 1e-12 absolute per integral (the reference's own test tolerance, test/tests_ints.cpp:15);
1e-11 for J/K and gradients, which are sums over ~1e5 integrals in a different order."""
import os

import numpy as np
import pytest

from lible_b200.workloads import WATER_BOHR, WATER_Z
from oracle import port, ri
from oracle import ref as R

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
H2O_ANG = [[0.0, 0.0, 0.0], [0.757, 0.586, 0.0], [-0.757, 0.586, 0.0]]


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def unique_of(V, idx):
    return V[idx[:, 0], idx[:, 1], idx[:, 2], idx[:, 3]]


# ---- oracle (CPU) ---------------------------------------------------------------------------

def test_port_eri4_matches_golden():
    g = load("h2o_ccpvdz_eri4.npz")
    V = port.PortMolecule("cc-pvdz", WATER_Z, WATER_BOHR).eri4()
    assert np.abs(unique_of(V, g["idx"]) - g["val"]).max() <= 1e-12
    # the permutational symmetry the unique list relies on
    assert np.abs(V - V.transpose(1, 0, 2, 3)).max() <= 1e-14
    assert np.abs(V - V.transpose(2, 3, 0, 1)).max() <= 1e-14


def test_port_jk_and_gradient_match_golden():
    g = load("dimer_ccpvdz_jk.npz")
    m = port.PortMolecule("cc-pvdz", list(g["Z"]), g["xyz"])
    J, K, nq = m.jk(g["D"], 0.0)
    assert nq == int(g["n_quartets"])
    assert np.abs(J - g["J"]).max() <= 1e-11 and np.abs(K - g["K"]).max() <= 1e-11
    assert np.abs(m.jk_grad(g["D"]) - g["grad"]).max() <= 1e-11


@pytest.mark.skipif(not R.available(), reason="reference library not built")
def test_ri_restatement_matches_golden():
    """oracle/ri.py on the reference's eri3 / eri2 reproduces the committed RI-K / RI-J fixture, and
    its RI-J agrees with the reference's own (mn|P) D_mn digestion."""
    g = load("dimer_rik.npz")
    r = R.RefStructure("cc-pvdz", list(g["Z"]), g["xyz"], aux="def2-universal-jkfit")
    B3, M = r.eri3(), r.eri2()
    D = g["C"] @ g["C"].T
    assert np.abs(ri.ri_exchange(B3, M, D) - g["K"]).max() <= 1e-12
    assert np.abs(ri.ri_exchange(B3, M, g["D2"]) - g["K2"]).max() <= 1e-12
    J = ri.ri_coulomb(B3, M, D)
    assert np.abs(J - g["J"]).max() <= 1e-12
    F, method = ri.metric_factor(M)
    assert method == 0
    assert np.abs(J - r.rij_j(F.T @ (F @ r.rij_gamma(D)))).max() <= 1e-11


# ---- CUDA path (GPU) --------------------------------------------------------------------------

@pytest.mark.gpu
def test_gpu_eri4_and_diagonal_match_golden():
    from lible_b200 import ints as L

    g = load("h2o_ccpvdz_eri4.npz")
    s = L.Structure("cc-pvdz", WATER_Z, WATER_BOHR, units="bohr")
    V = L.eri4(s)
    assert np.abs(unique_of(V, g["idx"]) - g["val"]).max() <= 1e-12
    assert np.abs(L.eri4Diagonal(s) - g["diag"]).max() <= 1e-12


@pytest.mark.gpu
def test_gpu_jk_and_gradient_match_golden():
    from lible_b200 import ints as L

    g = load("dimer_ccpvdz_jk.npz")
    s = L.Structure("cc-pvdz", list(g["Z"]), g["xyz"], units="bohr")
    J, K, st = L.jk(s, g["D"], schwarz=0.0)
    assert st["n_quartets"] == int(g["n_quartets"])
    assert np.abs(J - g["J"]).max() <= 1e-11 and np.abs(K - g["K"]).max() <= 1e-11
    Jg, Kg, _ = L.jk(s, g["D"], schwarz=0.0, use_graph=True)
    assert np.abs(Jg - g["J"]).max() <= 1e-11 and np.abs(Kg - g["K"]).max() <= 1e-11
    assert np.abs(L.jk_energy_backward(s, g["D"], schwarz=0.0) - g["grad"]).max() <= 1e-11


@pytest.mark.gpu
def test_gpu_d1_and_ri_batches_match_golden():
    from lible_b200 import ints as L

    g = load("h2o_def2svp_d1.npz")
    s = L.Structure("def2-svp", [8, 1, 1], H2O_ANG)
    sp = L.shellPairData(True, s)
    a, c = sp[int(g["class_ab"])], sp[int(g["class_cd"])]
    idx = [(i, j) for i in range(a.n_pairs_) for j in range(c.n_pairs_)]
    got = L.ERI4D1Kernel(a, c).batch(idx).reshape(g["d1"].shape)
    assert np.abs(got - g["d1"]).max() <= 1e-11

    r = load("h2o_ri.npz")
    s = L.Structure("def2-svp", [8, 1, 1], H2O_ANG, "def2-universal-jkfit")
    sp = L.shellPairData(True, s)
    aux = L.shellDataAux(s)
    a, x = sp[int(r["class_ab"])], aux[int(r["aux_s"])]
    idx = [(i, j) for i in range(a.n_pairs_) for j in range(x.n_shells_)]
    got = L.ERI3Kernel(a, x).batch(idx).reshape(r["eri3"].shape)
    assert np.abs(got - r["eri3"]).max() <= 1e-12
    assert np.abs(L.eri2(s) - r["eri2"]).max() <= 1e-12


@pytest.mark.gpu
def test_gpu_rik_matches_golden():
    """RI-K through the C ABI from the density factor and from D itself (an indefinite D exercises
    the C+ / C- split).  Tolerance 1e-10: the metric's condition number is ~4e7."""
    from lible_b200 import ints as L

    g = load("dimer_rik.npz")
    s = L.Structure("cc-pvdz", list(g["Z"]), g["xyz"], "def2-universal-jkfit", units="bohr")
    K, info = L.rik(s, C=g["C"], schwarz=0.0, info=True)
    assert np.abs(K - g["K"]).max() <= 1e-10
    assert np.abs(K - K.T).max() == 0.0
    assert info["n_pos"] == 10 and info["n_neg"] == 0 and info["n_blocks"] >= 1
    Kd = L.rik(s, D=g["C"] @ g["C"].T, schwarz=0.0)
    assert np.abs(Kd - g["K"]).max() <= 1e-10
    K2, info2 = L.rik(s, D=g["D2"], schwarz=0.0, info=True)
    assert info2["n_pos"] == 6 and info2["n_neg"] == 3
    assert np.abs(K2 - g["K2"]).max() <= 1e-10
    J, gam, dco = L.rij(s, g["C"] @ g["C"].T, schwarz=0.0)
    assert np.abs(J - g["J"]).max() <= 1e-10
    assert L.rij_last_solve(s)["method"] == "cholesky"
    # that call contracted the cached three-centre tensor; evaluating the integrals on every call
    # gives the same J, gamma and fitting coefficients (summation order differs only; d = M^-1 gamma
    # carries the metric's condition number, ~4e7, so its bound is 1e-8 relative)
    L.rij_set_cached(s, 0)
    Jn, gn, dn = L.rij(s, g["C"] @ g["C"].T, schwarz=0.0)
    assert np.abs(Jn - g["J"]).max() <= 1e-10
    assert np.abs(Jn - J).max() <= 1e-12
    assert np.abs(gn - gam).max() <= 1e-12 * max(1.0, np.abs(gn).max())
    assert np.abs(dn - dco).max() <= 1e-8 * max(1.0, np.abs(dn).max())
    L.rij_set_cached(s, 1)
    Jc, gc, dc = L.rij(s, g["C"] @ g["C"].T, schwarz=0.0)
    assert np.abs(Jc - J).max() <= 1e-12 and np.abs(gc - gam).max() <= 1e-12 * max(1.0, np.abs(gc).max())
    # the first call built the fitted three-centre tensor; the streaming path gives the same K
    assert info["fitted"] == 1 and info2["fitted"] == 1
    L.rik_set_fitted(s, 0)
    Ks, infos = L.rik(s, C=g["C"], schwarz=0.0, info=True)
    assert infos["fitted"] == 0 and infos["n_blocks"] >= 1
    assert np.abs(Ks - g["K"]).max() <= 1e-10
    L.rik_set_fitted(s, 1)
