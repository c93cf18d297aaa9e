"""Writes the golden fixtures of tests/golden/ from the reference itself.

Run from the repository root on a machine where the reference library has been built from the
reference sources (oracle/Makefile -> oracle/_ref/liblible_ref.so):

    python tests/golden/make_golden.py

Every array comes from the reference's own code (lible::ints::eri4, eri4Diagonal, the ERI4Kernel /
ERI4D1Kernel / ERI3Kernel / ERI2Kernel functors, and the CPU J/K / gradient digestion of those
kernels in oracle/ref_capi.cpp) on seeded inputs:

  h2o_ccpvdz_eri4.npz   water (O at 0, H at +-1.4305, 1.1093, 0 bohr), cc-pVDZ, 24 AOs: the unique
                        elements (ij|kl), i >= j, k >= l, ij >= kl, of the full eri4 tensor, and
                        eri4Diagonal
  dimer_ccpvdz_jk.npz   water dimer (cluster seed 7), density occ 10 (same seed): unscreened J, K and
                        the J/K energy gradient
  h2o_def2svp_d1.npz    ERI4D1Kernel blocks of class pair (p s | s s), symmetric pair lists
  h2o_ri.npz            ERI3Kernel batches of (s s | s-aux) and eri2 (P|Q) with def2-SVP /
                        def2-universal-jkfit
  dimer_rik.npz         water dimer (cluster seed 7), cc-pVDZ / def2-universal-jkfit: RI-K and RI-J
                        of D = C C^T (occ 10, same seed) and RI-K of an indefinite D = C1 C1^T - C2 C2^T,
                        from the reference's eri3 / eri2 through the numpy restatement in oracle/ri.py

Fixture names given on the command line regenerate only those (default: all).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from lible_b200.workloads import WATER_BOHR, WATER_Z, random_density, water_cluster  # noqa: E402
from oracle import ref as R  # noqa: E402
from oracle import ri  # noqa: E402

H2O_ANG = [[0.0, 0.0, 0.0], [0.757, 0.586, 0.0], [-0.757, 0.586, 0.0]]


def unique_indices(n):
    i, j, k, l = np.meshgrid(*([np.arange(n)] * 4), indexing="ij")
    ij = i * (i + 1) // 2 + j
    kl = k * (k + 1) // 2 + l
    mask = (i >= j) & (k >= l) & (ij >= kl)
    return np.stack([i[mask], j[mask], k[mask], l[mask]], axis=1).astype(np.int16)


def eri4_fixture():
    r = R.RefStructure("cc-pvdz", WATER_Z, WATER_BOHR)
    V = r.eri4()
    idx = unique_indices(V.shape[0])
    np.savez_compressed(os.path.join(HERE, "h2o_ccpvdz_eri4.npz"), idx=idx,
                        val=V[idx[:, 0], idx[:, 1], idx[:, 2], idx[:, 3]], diag=r.eri4_diagonal())


def jk_fixture():
    Z, xyz, rng = water_cluster(2, 7)
    D = random_density(48, 10, rng)
    rd = R.RefStructure("cc-pvdz", Z, xyz)
    J, K, nq, _ = rd.jk(D, 0.0)
    np.savez_compressed(os.path.join(HERE, "dimer_ccpvdz_jk.npz"), Z=np.asarray(Z), xyz=xyz, D=D, J=J, K=K,
                        n_quartets=nq, grad=rd.jk_grad(D))


def d1_fixture():
    rs = R.RefStructure("def2-svp", [8, 1, 1], H2O_ANG, units="angstrom")
    cls = rs.pair_classes(True)
    ps = [i for i, c in enumerate(cls) if c[:2] == (1, 0)][0]
    ss = [i for i, c in enumerate(cls) if c[:2] == (0, 0)][0]
    np.savez_compressed(os.path.join(HERE, "h2o_def2svp_d1.npz"), class_ab=ps, class_cd=ss,
                        d1=rs.eri4_class(True, ps, ss, d1=True))


def ri_fixture():
    rr = R.RefStructure("def2-svp", [8, 1, 1], H2O_ANG, aux="def2-universal-jkfit", units="angstrom")
    mcls = rr.pair_classes(True)
    acls = rr.aux_classes()
    ss = [i for i, c in enumerate(mcls) if c[:2] == (0, 0)][0]
    s_aux = [i for i, c in enumerate(acls) if c[0] == 0][0]
    np.savez_compressed(os.path.join(HERE, "h2o_ri.npz"), class_ab=ss, aux_s=s_aux,
                        eri3=rr.eri3_class(True, ss, s_aux), eri2=rr.eri2())


def rik_fixture():
    Z, xyz, rng = water_cluster(2, 7)
    n = 48
    C = np.linalg.qr(rng.standard_normal((n, 10)))[0]
    C1 = rng.standard_normal((n, 6)) * 0.3
    C2 = rng.standard_normal((n, 3)) * 0.2
    D2 = C1 @ C1.T - C2 @ C2.T
    r = R.RefStructure("cc-pvdz", Z, xyz, aux="def2-universal-jkfit")
    B3, M = r.eri3(), r.eri2()
    D = C @ C.T
    np.savez_compressed(os.path.join(HERE, "dimer_rik.npz"), Z=np.asarray(Z), xyz=xyz, C=C, D2=D2,
                        K=ri.ri_exchange(B3, M, D), J=ri.ri_coulomb(B3, M, D), K2=ri.ri_exchange(B3, M, D2))


FIXTURES = {"h2o_ccpvdz_eri4": eri4_fixture, "dimer_ccpvdz_jk": jk_fixture, "h2o_def2svp_d1": d1_fixture,
            "h2o_ri": ri_fixture, "dimer_rik": rik_fixture}


def main(names):
    if not R.available():
        raise SystemExit("oracle/_ref/liblible_ref.so is missing: run `make -C oracle ref` first")
    for name in names or list(FIXTURES):
        FIXTURES[name]()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main(sys.argv[1:])
