"""Parity of the CUDA path (through the C ABI) with the reference's own CPU integrals.

Tolerances: 1e-12 absolute per integral for FP64 integrals (the bar the reference's tests use,
test/tests_ints.cpp:15, applied element-wise against the reference's own output).  The reference's
golden sums (sum of |values| over whole tensors of up to 3.6e6 elements, test/tests_ints.cpp) are
checked to 1e-13 relative: last-bit differences of individual integrals, which any independent
implementation has, accumulate to ~1e-14 relative in such a sum."""
import numpy as np
import pytest

from lible_b200 import ints as L
from lible_b200.workloads import WATER_BOHR, WATER_Z, random_density, water_cluster
from oracle import ref as R

pytestmark = pytest.mark.gpu

O3_ANG = [[0, 0, 0], [0, 1, 1], [0, 0, 2]]
H2O_ANG = [[0.0, 0.0, 0.0], [0.757, 0.586, 0.0], [-0.757, 0.586, 0.0]]


def golden(value, expected):
    return abs(value - expected) <= 1e-13 * abs(expected)


def seqsum(x):
    """Sum of |x| in storage order, accumulated sequentially like the reference's tests."""
    return float(np.cumsum(np.abs(np.asarray(x)).ravel())[-1])


@pytest.fixture(scope="module")
def water_dz():
    return L.Structure("cc-pvdz", WATER_Z, WATER_BOHR, units="bohr")


def test_eri4_water_ccpvdz_elementwise(water_dz):
    V = L.eri4(water_dz)
    ref = R.RefStructure("cc-pvdz", WATER_Z, WATER_BOHR).eri4()
    assert V.shape == (24,) * 4
    assert np.abs(V - ref).max() <= 1e-12


def test_eri4_golden_o3_def2svp():
    s = L.Structure("def2-svp", [8, 8, 8], O3_ANG)
    V = L.eri4(s)
    assert golden(seqsum(V), 8246.711763196334)
    ref = R.RefStructure("def2-svp", [8, 8, 8], O3_ANG, units="angstrom").eri4()
    assert np.abs(V - ref).max() <= 1e-12


def test_eri4_diagonal_golden_o3_def2tzvp():
    s = L.Structure("def2-tzvp", [8, 8, 8], O3_ANG)
    d = L.eri4Diagonal(s)
    assert golden(seqsum(d), 306.806419250122)
    ref = R.RefStructure("def2-tzvp", [8, 8, 8], O3_ANG, units="angstrom").eri4_diagonal()
    assert np.abs(d - ref).max() <= 1e-12


def test_eri3_golden_o3():
    s = L.Structure("def2-tzvp", [8, 8, 8], O3_ANG, "def2-qzvp-rifit")
    v = L.eri3(s)
    assert golden(seqsum(v), 25854.105851585416531)
    ref = R.RefStructure("def2-tzvp", [8, 8, 8], O3_ANG, aux="def2-qzvp-rifit", units="angstrom").eri3()
    assert np.abs(v - ref).max() <= 1e-12


def test_eri2_golden_h2o():
    s = L.Structure("def2-svp", [8, 1, 1], H2O_ANG, "def2-qzvp-rifit")
    v = L.eri2(s)
    assert golden(seqsum(v), 8801.334703460838)
    ref = R.RefStructure("def2-svp", [8, 1, 1], H2O_ANG, aux="def2-qzvp-rifit", units="angstrom").eri2()
    assert np.abs(v - ref).max() <= 1e-12


def test_eri2_diagonal_golden_h2o():
    s = L.Structure("def2-svp", [8, 1, 1], H2O_ANG, "def2-universal-jkfit")
    d = L.eri2Diagonal(s)
    assert golden(seqsum(d), 830.788976485982)


def test_ri_required_errors():
    s = L.Structure("def2-svp", [8, 1, 1], H2O_ANG)
    with pytest.raises(L.LibleGpuError) as e:
        L.eri3(s)
    assert e.value.code == 4


def _deploy4(s, use_symm, d1=False):
    sp = L.shellPairData(use_symm, s)
    total = 0.0
    parts = []
    for a in sp:
        for c in sp:
            k = (L.ERI4D1Kernel if d1 else L.ERI4Kernel)(a, c)
            idx = [(i, j) for i in range(a.n_pairs_) for j in range(c.n_pairs_)]
            if idx:
                parts.append(k.batch(idx).ravel())
    return seqsum(np.concatenate(parts))


def test_deploy_eri4_kernel_golden():
    s = L.Structure("def2-svp", [8, 8, 8], O3_ANG)
    assert golden(_deploy4(s, False), 8246.711763197583)


def test_deploy_eri4d1_kernel_golden():
    s = L.Structure("def2-svp", [8, 8, 8], O3_ANG)
    assert golden(_deploy4(s, True, d1=True), 30546.780073140635)


def test_eri4_class_batches_elementwise():
    s = L.Structure("def2-svp", [8, 8, 8], O3_ANG)
    r = R.RefStructure("def2-svp", [8, 8, 8], O3_ANG, units="angstrom")
    for use_symm in (False, True):
        sp = L.shellPairData(use_symm, s)
        assert [(x.la_, x.lb_, x.n_pairs_, x.n_ppairs_) for x in sp] == r.pair_classes(use_symm)
        for a in sp:
            for c in sp:
                idx = [(i, j) for i in range(a.n_pairs_) for j in range(c.n_pairs_)]
                got = L.ERI4Kernel(a, c).batch(idx).reshape(a.n_pairs_, c.n_pairs_, -1)
                want = r.eri4_class(use_symm, a.index, c.index).reshape(a.n_pairs_, c.n_pairs_, -1)
                assert np.abs(got - want).max() <= 1e-12, (a.getLPair(), c.getLPair())


def test_eri4_class_batches_elementwise_f_shells():
    # def2-TZVP water has f functions on O: every class pair up to (ff|ff), among them the
    # one-thread-per-quartet classes with the largest register budget ((fd|ss)) and the classes
    # evaluated by whole warps on the tensor-core path ((fd|ps), (ff|dd), ...)
    s = L.Structure("def2-tzvp", [8, 1, 1], H2O_ANG)
    r = R.RefStructure("def2-tzvp", [8, 1, 1], H2O_ANG, units="angstrom")
    sp = L.shellPairData(True, s)
    assert [(x.la_, x.lb_, x.n_pairs_, x.n_ppairs_) for x in sp] == r.pair_classes(True)
    assert max(x.la_ for x in sp) == 3
    for a in sp:
        for c in sp:
            idx = [(i, j) for i in range(a.n_pairs_) for j in range(c.n_pairs_)]
            got = L.ERI4Kernel(a, c).batch(idx).reshape(a.n_pairs_, c.n_pairs_, -1)
            want = r.eri4_class(True, a.index, c.index).reshape(a.n_pairs_, c.n_pairs_, -1)
            assert np.abs(got - want).max() <= 1e-12, (a.getLPair(), c.getLPair())


def test_eri4d1_class_batches_elementwise():
    s = L.Structure("def2-svp", [8, 1, 1], H2O_ANG)
    r = R.RefStructure("def2-svp", [8, 1, 1], H2O_ANG, units="angstrom")
    sp = L.shellPairData(True, s)
    for a in sp:
        for c in sp:
            idx = [(i, j) for i in range(a.n_pairs_) for j in range(c.n_pairs_)]
            got = L.ERI4D1Kernel(a, c).batch(idx).reshape(a.n_pairs_, c.n_pairs_, 12, -1)
            want = r.eri4_class(True, a.index, c.index, d1=True).reshape(a.n_pairs_, c.n_pairs_, 12, -1)
            assert np.abs(got - want).max() <= 1e-11, (a.getLPair(), c.getLPair())


def test_eri4d1_class_batches_elementwise_f_shells():
    s = L.Structure("def2-tzvp", [8, 1, 1], H2O_ANG)
    r = R.RefStructure("def2-tzvp", [8, 1, 1], H2O_ANG, units="angstrom")
    sp = L.shellPairData(True, s)
    for a in sp:
        for c in sp:
            idx = [(i, j) for i in range(a.n_pairs_) for j in range(c.n_pairs_)]
            got = L.ERI4D1Kernel(a, c).batch(idx).reshape(a.n_pairs_, c.n_pairs_, 12, -1)
            want = r.eri4_class(True, a.index, c.index, d1=True).reshape(a.n_pairs_, c.n_pairs_, 12, -1)
            assert np.abs(got - want).max() <= 1e-11, (a.getLPair(), c.getLPair())


def test_kernel_batches_empty_and_out_of_range():
    # an empty batch returns an empty block; pair and shell indices are checked on the host before
    # anything reaches the device, and the context stays usable after the error
    s = L.Structure("def2-svp", [8, 1, 1], H2O_ANG, "def2-universal-jkfit")
    r = R.RefStructure("def2-svp", [8, 1, 1], H2O_ANG, units="angstrom")
    sp = L.shellPairData(True, s)
    aux = L.shellDataAux(s)
    a, c, x = sp[1], sp[-1], aux[0]
    assert L.ERI4Kernel(a, c).batch(np.zeros((0, 2))).shape == (0, 3, 1, 5, 5)
    assert L.ERI4D1Kernel(a, c).batch(np.zeros((0, 2))).shape == (0, 12, 3, 1, 5, 5)
    assert L.ERI3Kernel(a, x).batch(np.zeros((0, 2))).shape == (0, 3, 1, 1)
    bad = [(L.ERI4Kernel(a, c), [[a.n_pairs_, 0]]), (L.ERI4Kernel(a, c), [[0, c.n_pairs_]]),
           (L.ERI4D1Kernel(a, c), [[0, c.n_pairs_]]), (L.ERI3Kernel(a, x), [[0, x.n_shells_]]),
           (L.ERI3D1Kernel(a, x), [[a.n_pairs_, 0]]), (L.ERI2Kernel(x, x), [[x.n_shells_, 0]]),
           (L.ERI2D1Kernel(x, x), [[0, x.n_shells_]])]
    for k, idx in bad:
        with pytest.raises(L.LibleGpuError) as e:
            k.batch(idx)
        assert e.value.code == 1, type(k).__name__
    idx = [(i, j) for i in range(a.n_pairs_) for j in range(c.n_pairs_)]
    got = L.ERI4Kernel(a, c).batch(idx).reshape(a.n_pairs_, c.n_pairs_, -1)
    want = r.eri4_class(True, a.index, c.index).reshape(a.n_pairs_, c.n_pairs_, -1)
    assert np.abs(got - want).max() <= 1e-12


def test_concurrent_calls_on_one_context():
    # the reference's drivers call one kernel functor from many OpenMP threads; here four threads
    # share one context, one of them also making failing calls whose messages must stay its own
    import threading

    s = L.Structure("def2-svp", [8, 1, 1], H2O_ANG)
    sp = L.shellPairData(True, s)
    jobs = [(a, c) for a in sp for c in sp]

    def run(a, c):
        idx = [(i, j) for i in range(a.n_pairs_) for j in range(c.n_pairs_)]
        return L.ERI4Kernel(a, c).batch(idx)

    serial = {(a.index, c.index): run(a, c) for a, c in jobs}
    got, errors, messages = {}, [], []

    def work(part, failing):
        try:
            for _ in range(3):
                for a, c in part:
                    got[(a.index, c.index)] = run(a, c)
                    if failing:
                        with pytest.raises(L.LibleGpuError) as e:
                            L.ERI4Kernel(a, c).batch([[a.n_pairs_, 0]])
                        messages.append(str(e.value))
        except Exception as e:  # reported below
            errors.append(e)

    threads = [threading.Thread(target=work, args=(jobs[i::4], i == 0)) for i in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    assert messages and all("out of range" in m for m in messages)
    for k, v in serial.items():
        assert np.array_equal(got[k], v), k


def test_bounded_wait_gives_up_and_context_survives():
    # a wait that nothing completes runs out of polls: ETIMEOUT on the host, and the same context
    # still builds the same J/K afterwards
    Z, xyz, rng = water_cluster(2, seed=7)
    s = L.Structure("cc-pvdz", Z, xyz, units="bohr")
    D = random_density(s.nao, 10, rng)
    J0, K0, _ = L.jk(s, D, schwarz=0.0)
    for polls in (1, 4096):
        with pytest.raises(L.LibleGpuError) as e:
            L.check_bounded_wait(s, polls)
        assert e.value.code == 6
    with pytest.raises(L.LibleGpuError) as e:
        L.check_bounded_wait(s, 0)
    assert e.value.code == 1
    J1, K1, _ = L.jk(s, D, schwarz=0.0)
    assert np.abs(J1 - J0).max() <= 1e-12
    assert np.abs(K1 - K0).max() <= 1e-12


def _dd_dd_class(sp):
    return next(c for c in sp if (c.la_, c.lb_) == (2, 2))


def test_store_mode_wait_gives_up_and_context_survives():
    # the (dd|dd) class runs on the DMMA path, whose ket tiles arrive by bulk copy; with the copies
    # withheld its first wait runs out of polls, the store call reports ETIMEOUT (allocating and
    # allocation-free forms), and the next calls on the same context match the reference
    import ctypes

    import torch

    from lible_b200 import _lib

    s = L.Structure("def2-svp", [8, 8, 8], O3_ANG)
    sp = L.shellPairData(True, s)
    dd = _dd_dd_class(sp)
    idx = np.array([(i, j) for i in range(dd.n_pairs_) for j in range(dd.n_pairs_)], dtype=np.uint32)
    ref = R.RefStructure("def2-svp", [8, 8, 8], O3_ANG, units="angstrom").eri4_class(True, dd.index, dd.index)
    for polls in (1, 4096):
        L.inject_wait_timeout(s, polls)
        with pytest.raises(L.LibleGpuError) as e:
            L.ERI4Kernel(dd, dd).batch(idx)
        assert e.value.code == 6
        got = L.ERI4Kernel(dd, dd).batch(idx)
        assert np.abs(got.reshape(ref.shape) - ref).max() <= 1e-12
    lib = _lib.load()
    out = torch.zeros(ref.size, dtype=torch.float64, device="cuda")
    L.inject_wait_timeout(s, 64)
    rc = lib.lible_gpu_eri4_batch_noalloc(s.ctx, 1, dd.index, dd.index, len(idx), ctypes.c_void_p(idx.ctypes.data),
                                          ctypes.c_void_p(out.data_ptr()))
    assert rc == 6, lib.lible_gpu_last_error(s.ctx)
    rc = lib.lible_gpu_eri4_batch_noalloc(s.ctx, 1, dd.index, dd.index, len(idx), ctypes.c_void_p(idx.ctypes.data),
                                          ctypes.c_void_p(out.data_ptr()))
    assert rc == 0, lib.lible_gpu_last_error(s.ctx)
    assert np.abs(out.cpu().numpy().reshape(ref.shape) - ref).max() <= 1e-12
    with pytest.raises(L.LibleGpuError) as e:
        L.inject_wait_timeout(s, -1)
    assert e.value.code == 1


def test_deploy_eri3_eri2_golden():
    s = L.Structure("def2-svp", [8, 8, 8], O3_ANG, "def2-universal-jkfit")
    sp = L.shellPairData(False, s)
    aux = L.shellDataAux(s)
    parts3, parts3d, parts2, parts2d = [], [], [], []
    for a in sp:
        for c in aux:
            idx = [(i, j) for i in range(a.n_pairs_) for j in range(c.n_shells_)]
            parts3.append(L.ERI3Kernel(a, c).batch(idx).ravel())
            parts3d.append(L.ERI3D1Kernel(a, c).batch(idx).ravel())
    for a in aux:
        for b in aux:
            idx = [(i, j) for i in range(a.n_shells_) for j in range(b.n_shells_)]
            parts2.append(L.ERI2Kernel(a, b).batch(idx).ravel())
            parts2d.append(L.ERI2D1Kernel(a, b).batch(idx).ravel())
    assert golden(seqsum(np.concatenate(parts3)), 12350.130354189232)
    assert golden(seqsum(np.concatenate(parts2)), 21014.512841176023)
    assert golden(seqsum(np.concatenate(parts3d)), 78466.360848033844)
    assert golden(seqsum(np.concatenate(parts2d)), 39949.218421684251)


def test_jk_water_dimer_vs_reference_kernels():
    Z, xyz, rng = water_cluster(2, seed=7)
    s = L.Structure("cc-pvdz", Z, xyz, units="bohr")
    D = random_density(s.nao, 10, rng)
    r = R.RefStructure("cc-pvdz", Z, xyz)
    J, K, st = L.jk(s, D, schwarz=0.0)
    Jr, Kr, nq, _ = r.jk(D, schwarz=0.0)
    assert st["n_quartets"] == nq
    assert np.abs(J - Jr).max() <= 1e-11
    assert np.abs(K - Kr).max() <= 1e-11
    J2, K2, st2 = L.jk(s, D, schwarz=1e-12)
    assert np.abs(J2 - Jr).max() <= 1e-9
    assert np.abs(K2 - Kr).max() <= 1e-9


def test_jk_water_dimer_ccpvtz_vs_reference_kernels():
    # the J/K digestion epilogues of the f- and d-shell classes of cc-pVTZ (d on H, f on O)
    Z, xyz, rng = water_cluster(2, seed=11)
    s = L.Structure("cc-pvtz", Z, xyz, units="bohr")
    assert s.nao == 116
    D = random_density(s.nao, 10, rng)
    r = R.RefStructure("cc-pvtz", Z, xyz)
    J, K, st = L.jk(s, D, schwarz=0.0)
    Jr, Kr, nq, _ = r.jk(D, schwarz=0.0)
    assert st["n_quartets"] == nq
    assert np.abs(J - Jr).max() <= 1e-11
    assert np.abs(K - Kr).max() <= 1e-11
    J2, K2, _ = L.jk(s, D, schwarz=1e-12)
    assert np.abs(J2 - Jr).max() <= 1e-9
    assert np.abs(K2 - Kr).max() <= 1e-9


def test_jk_config_h2o16_ccpvdz_vs_reference():
    # the direct J/K configuration: (H2O)_16 cc-pVDZ (384 AOs), occupation 40, Schwarz 1e-12, FP64,
    # against the reference's ERI4Kernel batches digested on the host cores (unsampled)
    Z, xyz, rng = water_cluster(16, seed=2016)
    s = L.Structure("cc-pvdz", Z, xyz, units="bohr")
    assert s.nao == 384
    D = random_density(s.nao, 40, rng)
    J, K, st = L.jk(s, D, schwarz=1e-12)
    R.set_threads(R.max_threads())
    Jr, Kr, nq, _ = R.RefStructure("cc-pvdz", Z, xyz).jk(D, 1e-12, bra_stride=1)
    assert st["n_quartets"] == nq
    dJ, dK = np.abs(J - Jr).max(), np.abs(K - Kr).max()
    assert dJ <= 1e-11 and dK <= 1e-11, (dJ, dK, np.linalg.norm(J - Jr), np.linalg.norm(K - Kr))
    # the mixed-precision build of the same configuration stays within the energy bound
    Jm, Km, stm = L.jk(s, D, schwarz=1e-12, precision="mixed", fp32_threshold=1e-4)
    E = lambda J_, K_: float(np.sum(D * (0.5 * J_ - 0.25 * K_)))
    assert stm["n_fp32"] > 0
    assert abs(E(Jm, Km) - E(Jr, Kr)) <= 1e-8


def test_jk_gradient_h2o4_ccpvtz_vs_reference():
    # the gradient configuration's basis and density rule on (H2O)_4 cc-pVTZ (232 AOs, occupation
    # 20): the backward pass against the reference's ERI4D1Kernel batches contracted on the host
    Z, xyz, rng = water_cluster(4, seed=2008)
    s = L.Structure("cc-pvtz", Z, xyz, units="bohr")
    assert s.nao == 232
    D = random_density(s.nao, 20, rng)
    g = L.jk_energy_backward(s, D, schwarz=0.0)
    R.set_threads(R.max_threads())
    gr = R.RefStructure("cc-pvtz", Z, xyz).jk_grad(D)
    assert np.abs(g - gr).max() <= 1e-10, float(np.abs(g - gr).max())


def test_jk_gradient_vs_reference_and_fd():
    Z, xyz, rng = water_cluster(2, seed=3)
    s = L.Structure("cc-pvdz", Z, xyz, units="bohr")
    D = random_density(s.nao, 10, rng)
    g = L.jk_energy_backward(s, D, schwarz=0.0)
    gr = R.RefStructure("cc-pvdz", Z, xyz).jk_grad(D)
    assert np.abs(g - gr).max() <= 1e-10
    # central finite differences of the forward energy on two coordinates
    h = 1e-4
    for atom, x in [(0, 0), (4, 2)]:
        e = []
        for sgn in (1, -1):
            c = xyz.copy()
            c[atom, x] += sgn * h
            e.append(L.jk_energy_forward(L.Structure("cc-pvdz", Z, c, units="bohr"), D, schwarz=0.0))
        fd = (e[0] - e[1]) / (2 * h)
        assert abs(fd - g[atom, x]) <= 1e-6


def test_jk_gradient_ccpvtz_vs_reference():
    # f and d classes through the register form of the derivative contraction
    Z, xyz, rng = water_cluster(2, seed=5)
    s = L.Structure("cc-pvtz", Z, xyz, units="bohr")
    D = random_density(s.nao, 10, rng)
    g = L.jk_energy_backward(s, D, schwarz=0.0)
    gr = R.RefStructure("cc-pvtz", Z, xyz).jk_grad(D)
    assert np.abs(g - gr).max() <= 1e-10


def test_jk_gradient_screened_matches_screened_energy():
    # the backward pass keeps exactly the quartets of the forward pass at the same threshold
    Z, xyz, rng = water_cluster(3, seed=4)
    s = L.Structure("cc-pvdz", Z, xyz, units="bohr")
    D = random_density(s.nao, 15, rng)
    thr = 1e-10
    g = L.jk_energy_backward(s, D, schwarz=thr)
    h = 1e-4
    for atom, x in [(1, 1), (6, 0)]:
        e = []
        for sgn in (1, -1):
            c = xyz.copy()
            c[atom, x] += sgn * h
            e.append(L.jk_energy_forward(L.Structure("cc-pvdz", Z, c, units="bohr"), D, schwarz=thr))
        assert abs((e[0] - e[1]) / (2 * h) - g[atom, x]) <= 1e-6


def test_ri_contractions_vs_reference_kernels():
    Z, xyz, rng = water_cluster(2, seed=8)
    aux = "def2-universal-jkfit"
    s = L.Structure("cc-pvdz", Z, xyz, aux, units="bohr")
    r = R.RefStructure("cc-pvdz", Z, xyz, aux=aux)
    D = random_density(s.nao, 10, rng)
    g, _ = L.ri_contract(s, D=D, schwarz=0.0)
    gr = r.rij_gamma(D)
    assert np.abs(g - gr).max() <= 1e-11
    d = np.random.default_rng(1).standard_normal(s.naux)
    _, J = L.ri_contract(s, dcoef=d, schwarz=0.0)
    assert np.abs(J - r.rij_j(d)).max() <= 1e-11
    # full RI-J against a CPU solve of the reference's metric
    J, gamma, dc = L.rij(s, D, schwarz=0.0)
    M = r.eri2()
    dref = np.linalg.solve(M, gr)
    assert np.abs(dc - dref).max() <= 1e-7 * max(1.0, np.abs(dref).max())
    assert np.abs(J - r.rij_j(dref)).max() <= 1e-8


def test_mixed_precision_jk_error_small():
    Z, xyz, rng = water_cluster(4, seed=12)
    s = L.Structure("cc-pvdz", Z, xyz, units="bohr")
    D = random_density(s.nao, 20, rng)
    J, K, st = L.jk(s, D, 1e-12, "fp64")
    Jm, Km, stm = L.jk(s, D, 1e-12, "mixed", 1e-4)
    assert stm["n_fp32"] > 0
    E = np.sum(D * (0.5 * J - 0.25 * K))
    Em = np.sum(D * (0.5 * Jm - 0.25 * Km))
    assert abs(E - Em) <= 1e-8
    assert np.linalg.norm(Jm - J) <= 1e-6 and np.linalg.norm(Km - K) <= 1e-6


def test_mixed_precision_jk_ccpvtz():
    # FP32 quartets of the f- and d-shell classes of cc-pVTZ (register and shared-memory shapes)
    Z, xyz, rng = water_cluster(3, seed=13)
    s = L.Structure("cc-pvtz", Z, xyz, units="bohr")
    D = random_density(s.nao, 15, rng)
    J, K, st = L.jk(s, D, 1e-12, "fp64")
    Jm, Km, stm = L.jk(s, D, 1e-12, "mixed", 1e-4)
    assert stm["n_fp32"] > 0 and stm["n_quartets"] == st["n_quartets"]
    E = np.sum(D * (0.5 * J - 0.25 * K))
    Em = np.sum(D * (0.5 * Jm - 0.25 * Km))
    assert abs(E - Em) <= 1e-8
    assert np.linalg.norm(Jm - J) <= 1e-6 and np.linalg.norm(Km - K) <= 1e-6
    # every class pair takes part in both precisions at a loose threshold
    Jm2, Km2, stm2 = L.jk(s, D, 1e-12, "mixed", 1e-1)
    assert stm2["n_fp32"] > stm["n_fp32"]
    assert np.linalg.norm(Jm2 - J) <= 1e-4 and np.linalg.norm(Km2 - K) <= 1e-4


def test_rij_cached_packed_rows_odd_length():
    """The cached RI-J tensor keeps the packed lower triangle, nao (nao + 1) / 2 elements per
    auxiliary function.  H2 / cc-pVDZ has 10 AOs, so a row holds 55 elements and the passes take
    their scalar (unvectorised) form; the cached call matches the evaluating one and the
    reference's gamma, also for a density that is not symmetric."""
    xyz = np.array([[0.0, 0.0, 0.0], [0.0, 0.3, 1.4]])
    s = L.Structure("cc-pvdz", [1, 1], xyz, "def2-universal-jkfit", units="bohr")
    assert (s.nao * (s.nao + 1) // 2) % 2 == 1
    r = R.RefStructure("cc-pvdz", [1, 1], xyz, aux="def2-universal-jkfit")
    rng = np.random.default_rng(11)
    D = random_density(s.nao, 1, rng)
    J, g, d = L.rij(s, D, schwarz=0.0)  # the first call builds and uses the cached tensor
    gr = r.rij_gamma(D)
    assert np.abs(g - gr).max() <= 1e-12 * max(1.0, np.abs(gr).max())
    L.rij_set_cached(s, 0)
    Jn, gn, dn = L.rij(s, D, schwarz=0.0)
    L.rij_set_cached(s, 1)
    assert np.abs(J - Jn).max() <= 1e-12 and np.abs(J - J.T).max() == 0.0
    assert np.abs(g - gn).max() <= 1e-12 * max(1.0, np.abs(gn).max())
    # a non-symmetric density: the cached pass sums both triangles, (mn|P) (D_mn + D_nm)
    A = D + 0.1 * rng.standard_normal(D.shape)
    _, ga, _ = L.rij(s, A, schwarz=0.0)
    _, gs, _ = L.rij(s, 0.5 * (A + A.T), schwarz=0.0)
    assert np.abs(ga - gs).max() <= 1e-12 * max(1.0, np.abs(gs).max())


def test_rij_even_tempered_aux_vs_reference():
    # the s-f even-tempered auxiliary basis of the mixed-precision RI-J workload (0.1 * 2.5^k,
    # k = 0..11 per l), on one water
    from lible_b200.workloads import even_tempered_aux
    from oracle import port

    aux = even_tempered_aux(WATER_Z)
    s = L.Structure("cc-pvdz", WATER_Z, WATER_BOHR, aux, units="bohr")
    assert s.naux == 3 * 12 * (1 + 3 + 5 + 7)
    r = R.RefStructure(port.read_basis("cc-pvdz", WATER_Z), WATER_Z, WATER_BOHR, aux=aux)
    rng = np.random.default_rng(4)
    D = random_density(s.nao, 5, rng)
    J, gamma, dcoef = L.rij(s, D, schwarz=0.0)
    gr = r.rij_gamma(D)
    assert np.abs(gamma - gr).max() <= 1e-10 * max(1.0, np.abs(gr).max())
    # the same solve in numpy on the reference metric
    M = r.eri2()
    info = L.rij_last_solve(s)
    if info["method"] == "cholesky":
        dref = np.linalg.solve(M, gr)
    elif info["method"] == "cholesky+shift":
        dref = np.linalg.solve(M + info["shift"] * np.eye(len(M)), gr)
    else:
        w, V = np.linalg.eigh(M)
        keep = w > 1e-12 * w.max()
        dref = V[:, keep] @ ((V[:, keep].T @ gr) / w[keep])
    Jref = r.rij_j(dref)
    assert np.abs(J - Jref).max() <= 1e-6 * max(1.0, np.abs(Jref).max())


@pytest.mark.parametrize("occ", [15, 16])
def test_rik_multi_tile_vs_dense_contraction(occ):
    """RI-K of (H2O)_8 cc-pVDZ (192 AOs: two 128-row tiles per side, the second one partial) with
    def2-universal-jkfit, through the fitted tensor and through the streaming path, against the dense
    contraction K = sum (ml|P) (P|Q)^-1 (Q|ns) D_ls in numpy on the device's eri3 / eri2 (both checked
    against the reference elsewhere).  An odd occupation gives odd rows of the exchange operand, an
    even one even rows; tolerance 1e-9 relative."""
    Z, xyz, rng = water_cluster(8, 5)
    s = L.Structure("cc-pvdz", Z, xyz, "def2-universal-jkfit", units="bohr")
    C = np.linalg.qr(rng.standard_normal((s.nao, occ)))[0]
    B3, M = L.eri3(s), L.eri2(s)
    X = np.linalg.solve(M, B3.reshape(-1, s.naux).T).T.reshape(B3.shape)  # (ml|Q) M^-1_QP
    D = C @ C.T
    Kref = np.einsum("mlp,nsp,ls->mn", X, B3, D, optimize=True)
    scale = max(1.0, np.abs(Kref).max())
    K, info = L.rik(s, C=C, schwarz=0.0, info=True)
    assert info["fitted"] == 1
    assert np.abs(K - Kref).max() <= 1e-9 * scale
    assert np.abs(K - K.T).max() == 0.0
    L.rik_set_fitted(s, 0)
    Ks, infos = L.rik(s, C=C, schwarz=0.0, info=True)
    L.rik_set_fitted(s, 1)
    assert infos["fitted"] == 0
    assert np.abs(Ks - Kref).max() <= 1e-9 * scale


def test_rik_blocks_and_ill_conditioned_metric_vs_reference():
    """RI-K of a water trimer with the even-tempered s-f auxiliary basis, whose metric is not
    numerically positive definite (shifted Cholesky or eigendecomposition): against the numpy
    restatement on the reference's own eri3 / eri2 with the same metric policy, and with the Schwarz
    test on (its effect stays far below the tolerance)."""
    from oracle import ri

    from lible_b200.workloads import even_tempered_aux
    from oracle import port

    Z, xyz, rng = water_cluster(3, 11)
    aux = even_tempered_aux(Z)
    s = L.Structure("cc-pvdz", Z, xyz, aux, units="bohr")
    r = R.RefStructure(port.read_basis("cc-pvdz", Z), Z, xyz, aux=aux)
    B3, M = r.eri3(), r.eri2()
    C = np.linalg.qr(rng.standard_normal((s.nao, 15)))[0]
    K = L.rik(s, C=C, schwarz=0.0)
    F, method = ri.metric_factor(M)
    solve = L.rij_last_solve(s)
    assert {0: "cholesky", 1: "eigen", 2: "cholesky+shift"}[method] == solve["method"]
    Kref = ri.ri_exchange(B3, M, C @ C.T)
    assert np.abs(K - Kref).max() <= 1e-6 * max(1.0, np.abs(Kref).max())
    Ks = L.rik(s, C=C, schwarz=1e-12)
    assert np.abs(Ks - K).max() <= 1e-6 * max(1.0, np.abs(Kref).max())


def test_rij_gradient_vs_finite_differences():
    """Gradient of the RI-J energy 1/2 Tr(D J_RI) against central differences (step 1e-4 bohr) of the
    energy from lible_gpu_rij at displaced geometries; def2-universal-jkfit (aux up to g) on a water
    dimer, translational invariance, and the returned energy against 1/2 Tr(D J_RI)."""
    Z, xyz, rng = water_cluster(2, 21)
    aux = "def2-universal-jkfit"
    s = L.Structure("cc-pvdz", Z, xyz, aux, units="bohr")
    D = random_density(s.nao, 10, rng)
    g, E = L.rij_grad(s, D, schwarz=0.0)
    J, _, _ = L.rij(s, D, schwarz=0.0)
    assert abs(E - 0.5 * np.sum(D * J)) <= 1e-10 * abs(E)
    assert np.abs(g.sum(axis=0)).max() <= 1e-8 * max(1.0, np.abs(g).max())

    def energy(c):
        Jc, _, _ = L.rij(L.Structure("cc-pvdz", Z, c, aux, units="bohr"), D, schwarz=0.0)
        return 0.5 * float(np.sum(D * Jc))

    h = 1e-4
    for atom, x in ((0, 0), (2, 1), (4, 2)):
        cp, cm = xyz.copy(), xyz.copy()
        cp[atom, x] += h
        cm[atom, x] -= h
        fd = (energy(cp) - energy(cm)) / (2 * h)
        assert abs(fd - g[atom, x]) <= 1e-6 * max(1.0, abs(fd)), (atom, x, fd, g[atom, x])
    # the Schwarz-screened gradient stays within the screening error
    gs, _ = L.rij_grad(s, D, schwarz=1e-12)
    assert np.abs(gs - g).max() <= 1e-8


def test_soc_and_eri2d2_kernels_vs_reference():
    """ERI4SOCKernel, ERI3SOCKernel and ERI2D2Kernel batches of every class pair (shellPairData
    without symmetry, so classes with la < lb are included) element-wise against the reference's
    own kernels, and the reference's golden sums (test/tests_ints.cpp:1055-1150)."""
    s = L.Structure("def2-svp", [8, 8, 8], O3_ANG, "def2-universal-jkfit")
    r = R.RefStructure("def2-svp", [8, 8, 8], O3_ANG, aux="def2-universal-jkfit", units="angstrom")
    sp = L.shellPairData(False, s)
    aux = L.shellDataAux(s)
    parts4, parts3, parts2 = [], [], []
    for i, a in enumerate(sp):
        for j, c in enumerate(sp):
            idx = [(p, q) for p in range(a.n_pairs_) for q in range(c.n_pairs_)]
            got = L.ERI4SOCKernel(a, c).batch(idx)
            want = r.eri4soc_class(False, i, j).reshape(got.shape)
            assert np.abs(got - want).max() <= 1e-12, (i, j)
            parts4.append(got.ravel())
        for j, x in enumerate(aux):
            idx = [(p, q) for p in range(a.n_pairs_) for q in range(x.n_shells_)]
            got = L.ERI3SOCKernel(a, x).batch(idx)
            want = r.eri3soc_class(False, i, j).reshape(got.shape)
            assert np.abs(got - want).max() <= 1e-12, (i, j)
            parts3.append(got.ravel())
    for i, x in enumerate(aux):
        for j, y in enumerate(aux):
            idx = [(p, q) for p in range(x.n_shells_) for q in range(y.n_shells_)]
            got = L.ERI2D2Kernel(x, y).batch(idx)
            want = r.eri2d2_class(i, j).reshape(got.shape)
            assert np.abs(got - want).max() <= 1e-11 * max(1.0, np.abs(want).max()), (i, j)
            parts2.append(got.ravel())
    assert golden(seqsum(np.concatenate(parts4)), 12940.953099658431)
    assert golden(seqsum(np.concatenate(parts3)), 18124.713152990007)
    assert golden(seqsum(np.concatenate(parts2)), 175567.635699242965)
