"""The allocation-free ERI4Kernel batch call (lible_gpu_eri4_batch_noalloc).

It exists for callers that must not allocate device memory during the call: programs that have
given all free device memory to their own pool allocator, or that overlap work on other streams and
cannot accept the device-wide synchronisation cudaFree implies.  It stages the pair list in a fixed
buffer inside the library instead of a per-call allocation.  This test calls it through the C ABI,
twice in a row for every class pair of a small molecule (so the second call runs on a buffer the
first one left behind), and compares with the regular allocating call at the 1e-12 per-integral
tolerance the other parity tests use, and one class pair directly with the reference's own
ERI4Kernel output.  It also checks that an oversized request and a batch context are refused.
"""
import ctypes

import numpy as np
import pytest

from lible_b200 import _lib
from lible_b200 import ints as L
from lible_b200.workloads import water_cluster
from oracle import ref as R

pytestmark = pytest.mark.gpu

O3_ANG = [[0, 0, 0], [0, 1, 1], [0, 0, 2]]
MAX_PAIRS = 1 << 20


def test_eri4_batch_noalloc_matches_allocating_call():
    import torch

    lib = _lib.load()
    s = L.Structure("def2-svp", [8, 8, 8], O3_ANG)
    for use_symm in (False, True):
        sp = L.shellPairData(use_symm, s)  # puts the pair classes on the device
        for a in sp:
            for c in sp:
                idx = np.array([(i, j) for i in range(a.n_pairs_) for j in range(c.n_pairs_)], dtype=np.uint32)
                want = L.ERI4Kernel(a, c).batch(idx)
                for _ in range(2):
                    out = torch.full(want.shape, float("nan"), dtype=torch.float64, device="cuda")
                    rc = lib.lible_gpu_eri4_batch_noalloc(s.ctx, int(use_symm), a.index, c.index, len(idx),
                                                          ctypes.c_void_p(idx.ctypes.data),
                                                          ctypes.c_void_p(out.data_ptr()))
                    assert rc == 0, lib.lible_gpu_last_error(s.ctx)
                    got = out.cpu().numpy()
                    assert np.abs(got - want).max() <= 1e-12, (a.getLPair(), c.getLPair())


def test_eri4_batch_noalloc_rejects_oversized_requests():
    import torch

    lib = _lib.load()
    s = L.Structure("def2-svp", [8, 1, 1], [[0.0, 0.0, 0.0], [0.757, 0.586, 0.0], [-0.757, 0.586, 0.0]])
    L.shellPairData(True, s)
    idx = np.zeros((4, 2), dtype=np.uint32)
    out = torch.zeros(16, dtype=torch.float64, device="cuda")
    rc = lib.lible_gpu_eri4_batch_noalloc(s.ctx, 1, 0, 0, MAX_PAIRS + 1, ctypes.c_void_p(idx.ctypes.data),
                                          ctypes.c_void_p(out.data_ptr()))
    assert rc == 1
    assert b"exceeds the maximum" in lib.lible_gpu_last_error(s.ctx)


def test_eri4_batch_noalloc_matches_reference_class():
    import torch

    lib = _lib.load()
    s = L.Structure("def2-svp", [8, 8, 8], O3_ANG)
    sp = L.shellPairData(True, s)
    r = R.RefStructure("def2-svp", [8, 8, 8], O3_ANG, units="angstrom")
    # (ss|ps) and (ds|dp): the bra has the smaller pair type, so the list is staged with its columns
    # swapped (the kernels take the larger pair type as the bra)
    for a, c in [(0, 1), (3, 4)]:
        A, C = sp[a], sp[c]
        want = r.eri4_class(True, A.index, C.index)
        idx = np.array([(i, j) for i in range(A.n_pairs_) for j in range(C.n_pairs_)], dtype=np.uint32)
        out = torch.zeros(want.size, dtype=torch.float64, device="cuda")
        for _ in range(2):
            rc = lib.lible_gpu_eri4_batch_noalloc(s.ctx, 1, A.index, C.index, len(idx), ctypes.c_void_p(idx.ctypes.data),
                                                  ctypes.c_void_p(out.data_ptr()))
            assert rc == 0, lib.lible_gpu_last_error(s.ctx)
            assert np.abs(out.cpu().numpy().reshape(want.shape) - want).max() <= 1e-12, (A.getLPair(), C.getLPair())


def test_eri4_batch_noalloc_refuses_a_batch_context():
    import torch

    lib = _lib.load()
    mols = []
    for seed in (1, 2):
        Z, xyz, _ = water_cluster(1, seed=seed)
        mols.append(("cc-pvdz", Z, xyz))
    b = L.Batch(mols)
    idx = np.zeros((1, 2), dtype=np.uint32)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = lib.lible_gpu_eri4_batch_noalloc(b.ctx, 1, 0, 0, 1, ctypes.c_void_p(idx.ctypes.data),
                                          ctypes.c_void_p(out.data_ptr()))
    assert rc == 5, lib.lible_gpu_last_error(b.ctx)
