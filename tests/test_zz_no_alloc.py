"""The allocation-free ERI4Kernel batch call (lible_gpu_eri4_batch_noalloc).

It exists for callers that must not allocate device memory during the call: programs that have
given all free device memory to their own pool allocator, or that overlap work on other streams and
cannot accept the device-wide synchronisation cudaFree implies.  It stages the pair list in a fixed
buffer inside the library instead of a per-call allocation.  This test calls it through the C ABI,
twice in a row for every class pair of a small molecule (so the second call runs on a buffer the
first one left behind), and compares with the regular allocating call at the 1e-12 per-integral
tolerance the other parity tests use.  It also checks that an oversized request is refused.
"""
import ctypes

import numpy as np
import pytest

from lible_b200 import _lib
from lible_b200 import ints as L

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
