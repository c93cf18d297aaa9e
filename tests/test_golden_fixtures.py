"""Parity against the committed golden fixtures (tests/golden/, written from the reference itself
by tests/golden/make_golden.py).  They pin the oracle's C restatement on the CPU and the CUDA path
on the GPU without needing the compiled reference at test time.

Tolerances: 1e-12 absolute per integral (the reference's own test tolerance, test/tests_ints.cpp:15);
1e-11 for J/K and gradients, which are sums over ~1e5 integrals in a different order."""
import os

import numpy as np
import pytest

from lible_b200.workloads import WATER_BOHR, WATER_Z
from oracle import port

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
