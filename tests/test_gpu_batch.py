"""Batched J/K of several molecules (one work-queue launch per quartet class for the whole batch),
CUDA-graph replay and the launch autotuner.

The batch path has no reference counterpart; it must reproduce, molecule by molecule, the J and K
of the single-structure path (itself checked against the reference's ERI4Kernel digestion in
test_gpu_eri.py) and of the oracle's C restatement, to 1e-11 absolute (summation order differs)."""
import numpy as np
import pytest

from lible_b200 import ints as L
from lible_b200.workloads import random_density, water_cluster
from oracle import port

pytestmark = pytest.mark.gpu

SPECS = [(1, "cc-pvdz", 3), (2, "cc-pvtz", 5), (3, "cc-pvdz", 7), (1, "cc-pvtz", 11), (2, "cc-pvdz", 13)]


def _batch(specs):
    mols, Ds = [], []
    for n, basis, seed in specs:
        Z, xyz, rng = water_cluster(n, seed)
        mols.append((basis, Z, xyz))
    b = L.Batch(mols)
    for m, (n, basis, seed) in enumerate(specs):
        _, _, rng = water_cluster(n, seed)
        Ds.append(random_density(int(b.nao[m]), 5 * n, rng))
    return b, mols, Ds


def test_batch_jk_matches_single_structures_and_oracle():
    b, mols, Ds = _batch(SPECS)
    J, K, st = L.jk(b, b.pack(Ds), schwarz=1e-12)
    Js, Ks = b.unpack(J), b.unpack(K)
    total = 0
    for m, (basis, Z, xyz) in enumerate(mols):
        s = L.Structure(basis, Z, xyz, units="bohr")
        Jm, Km, stm = L.jk(s, Ds[m], schwarz=1e-12)
        total += stm["n_quartets"]
        assert np.abs(Js[m] - Jm).max() <= 1e-11, m
        assert np.abs(Ks[m] - Km).max() <= 1e-11, m
    assert st["n_quartets"] == total
    # molecules small enough for the C restatement, unscreened
    J0, K0, _ = L.jk(b, b.pack(Ds), schwarz=0.0)
    for m in (0, 2):
        basis, Z, xyz = mols[m]
        Jr, Kr = port.jk(basis, Z, xyz, Ds[m])
        assert np.abs(b.unpack(J0)[m] - Jr).max() <= 1e-11
        assert np.abs(b.unpack(K0)[m] - Kr).max() <= 1e-11


def test_batch_graph_replay_matches_direct_launches():
    import torch

    b, mols, Ds = _batch(SPECS)
    Dp = b.pack(Ds)
    J, K, _ = L.jk(b, Dp)
    Dd = torch.tensor(Dp, device="cuda")
    Jd, Kd = torch.empty_like(Dd), torch.empty_like(Dd)
    for _ in range(3):  # first call captures, the others replay
        L.jk(b, Dd, J=Jd, K=Kd, use_graph=True)
        assert np.abs(Jd.cpu().numpy() - J).max() <= 1e-12
        assert np.abs(Kd.cpu().numpy() - K).max() <= 1e-12
    # a new density in the same buffers is picked up by the replay
    Dd.mul_(0.5)
    L.jk(b, Dd, J=Jd, K=Kd, use_graph=True)
    assert np.abs(Jd.cpu().numpy() - 0.5 * J).max() <= 1e-12


def test_batch_rejects_single_structure_calls():
    import ctypes

    from lible_b200 import _lib

    b, _, _ = _batch(SPECS[:2])
    lib = _lib.load()
    out = np.zeros(1)
    assert lib.lible_gpu_eri4_diagonal(b.ctx, ctypes.c_void_p(out.ctypes.data)) == 5
    assert b"single structure" in lib.lible_gpu_last_error(b.ctx)


def test_single_structure_graph_mixed_matches_direct():
    Z, xyz, rng = water_cluster(4, 21)
    s = L.Structure("cc-pvdz", Z, xyz, units="bohr")
    D = random_density(s.nao, 20, rng)
    J, K, _ = L.jk(s, D, 1e-12, "mixed")
    Jg, Kg, _ = L.jk(s, D, 1e-12, "mixed", use_graph=True)
    assert np.abs(Jg - J).max() <= 1e-12 and np.abs(Kg - K).max() <= 1e-12


def test_autotune_keeps_results_and_cache_round_trips(tmp_path):
    b, mols, Ds = _batch(SPECS[:3])
    Dp = b.pack(Ds)
    J, K, _ = L.jk(b, Dp)
    cache = str(tmp_path / "tune.txt")
    summary = L.jk_autotune(b, Dp, cache=cache)
    lines = [x for x in summary.splitlines() if x.strip()]
    assert lines and all("grid_div=" in x and "chunk_mult=" in x for x in lines)
    Jt, Kt, _ = L.jk(b, Dp)
    assert np.abs(Jt - J).max() <= 1e-12 and np.abs(Kt - K).max() <= 1e-12
    entries = open(cache).read().splitlines()
    assert len(entries) == len(lines)
    for e in entries:
        gpu, cls, fp32, bucket, choice = e.split("|")
        gd, cm, shape = (int(x) for x in choice.split())
        assert gd in (1, 2) and cm in (2, 8, 32) and shape in (0, 1, 2) and fp32 == "0"
    # a fresh batch built with the cache reproduces the same results
    b2 = L.Batch(mols)
    L.set_tune_cache(b2, cache)
    J2, K2, _ = L.jk(b2, Dp)
    assert np.abs(J2 - J).max() <= 1e-12 and np.abs(K2 - K).max() <= 1e-12


@pytest.mark.parametrize("basis,precision,shape", [("cc-pvdz", "mixed", 1), ("cc-pvtz", "mixed", 1),
                                                  ("cc-pvtz", "fp64", 1), ("cc-pvtz", "fp64", 2),
                                                  ("cc-pvtz", "mixed", 2), ("cc-pvdz", "fp64", 2)])
def test_alternative_tile_shapes_give_the_same_jk(tmp_path, basis, precision, shape):
    # every class forced to its alternative shape (where it has one) through a tune cache; shape 1:
    # the register path with the next larger thread group, the group paths with twice the warps,
    # the occupancy-bounded classes with the default bound; shape 2: the class in the other
    # orientation (bra and ket exchanged) where that takes the register path; the J/K must not change
    Z, xyz, rng = water_cluster(3, 23)
    s = L.Structure(basis, Z, xyz, units="bohr")
    D = random_density(s.nao, 15, rng)
    J, K, _ = L.jk(s, D, 1e-12, precision)
    cache = str(tmp_path / "tune.txt")
    L.jk_autotune(s, D, 1e-12, precision, cache=cache)
    lines = open(cache).read().splitlines()
    forced = []
    for e in lines:
        head, choice = e.rsplit("|", 1)
        gd, cm, _ = choice.split()
        forced.append(f"{head}|{gd} {cm} {shape}")
    open(cache, "w").write("\n".join(forced) + "\n")
    s2 = L.Structure(basis, Z, xyz, units="bohr")
    L.set_tune_cache(s2, cache)
    J2, K2, _ = L.jk(s2, D, 1e-12, precision)
    prof = L.jk_profile(s2, D, 1e-12, precision)
    assert any(r["shape"] == shape for r in prof)
    tol = 1e-12 if precision == "fp64" else 1e-9
    assert np.abs(J2 - J).max() <= tol and np.abs(K2 - K).max() <= tol


def test_jk_profile_times_every_launch_and_returns_the_build():
    Z, xyz, rng = water_cluster(3, 17)
    s = L.Structure("cc-pvdz", Z, xyz, units="bohr")
    D = random_density(s.nao, 15, rng)
    J, K, _ = L.jk(s, D, 1e-12, "mixed")
    Jp, Kp = np.empty_like(J), np.empty_like(K)
    prof = L.jk_profile(s, D, 1e-12, "mixed", J=Jp, K=Kp)
    assert np.abs(Jp - J).max() <= 1e-12 and np.abs(Kp - K).max() <= 1e-12
    plan = L.jk_plan(s, 1e-12, "mixed")
    assert sum(r["tasks"] for r in prof) == plan["n_quartets"]
    assert any(r["fp32"] for r in prof) and all(r["ms"] > 0 for r in prof)
    assert abs(sum(r["flops"] for r in prof) - plan["flops_fp64"] - plan["flops_fp32"]) <= 1e-6 * plan["flops_fp64"]


def test_full_c3_batch_vs_single_structures_and_reference():
    """The whole heterogeneous batch of the batch benchmark (64 water clusters of 1..12 waters, half
    cc-pVDZ, half cc-pVTZ, Schwarz 1e-12), built as one batch: every molecule's FP64 J and K against
    its own single-structure build (1e-11), the mixed-precision batch within the 1e-8 Eh energy bound
    of FP64 per molecule, and the molecules of up to three waters against the reference's
    ERI4Kernel J/K digestion over the same screened quartets (1e-11)."""
    from lible_b200.workloads import batch_clusters
    from oracle import ref as R

    specs = batch_clusters()
    b = L.Batch([(bs, Z, xyz) for bs, Z, xyz, _ in specs])
    Ds = [mk(int(b.nao[m])) for m, (_, _, _, mk) in enumerate(specs)]
    Dp = b.pack(Ds)
    J, K, st = L.jk(b, Dp, schwarz=1e-12)
    Jm, Km, _ = L.jk(b, Dp, schwarz=1e-12, precision="mixed")
    Js, Ks, Jms, Kms = b.unpack(J), b.unpack(K), b.unpack(Jm), b.unpack(Km)
    total, n_ref = 0, 0
    for m, (basis, Z, xyz, _) in enumerate(specs):
        s = L.Structure(basis, Z, xyz, units="bohr")
        J1, K1, st1 = L.jk(s, Ds[m], schwarz=1e-12)
        total += st1["n_quartets"]
        assert np.abs(Js[m] - J1).max() <= 1e-11, m
        assert np.abs(Ks[m] - K1).max() <= 1e-11, m
        E = 0.5 * np.sum(Ds[m] * Js[m]) - 0.25 * np.sum(Ds[m] * Ks[m])
        Emix = 0.5 * np.sum(Ds[m] * Jms[m]) - 0.25 * np.sum(Ds[m] * Kms[m])
        assert abs(Emix - E) <= 1e-8, m
        if len(Z) <= 9:
            r = R.RefStructure(basis, Z, xyz)
            Jr, Kr, nq, _ = r.jk(Ds[m], 1e-12)
            assert nq == st1["n_quartets"], m
            assert np.abs(Js[m] - Jr).max() <= 1e-11, m
            assert np.abs(Ks[m] - Kr).max() <= 1e-11, m
            n_ref += 1
    assert st["n_quartets"] == total
    assert n_ref >= 10
