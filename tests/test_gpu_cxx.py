"""The C++20 drop-in header (include/lible_b200.hpp) compiled against the reference's own headers:
oracle/_ref/test_dropin (built from tests/cxx/test_dropin.cpp by tests/cxx/Makefile) constructs the
reference's lible::ints::Structure objects and compares every replaced call -- eri4, eri4Diagonal,
eri3, eri2, eri2Diagonal and the ERI{4,3,2}Kernel / ERI{4,3,2}D1Kernel functors -- with the
reference's own call on the same object (1e-12 per integral, 1e-11 for the derivative blocks)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "test_dropin")

pytestmark = pytest.mark.gpu


def test_cxx20_dropin_header_matches_reference_calls():
    assert os.path.exists(BIN), "oracle/_ref/test_dropin is not built (make -C tests/cxx)"
    r = subprocess.run([BIN, os.path.join(ROOT, "lible_b200", "basis")], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "all ok" in r.stdout
