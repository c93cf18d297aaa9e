"""Direct tests of the device special functions the class kernels use (through the C ABI).

- e^{-x} (expNeg: Cody-Waite reduction plus a degree-13 Taylor polynomial, FP64 FMAs only) against
  numpy's exp over [0, 700], within 2 ulp of the result.
- FP64 Boys F_0..F_N (grid Taylor about the integers + downward recursion, asymptote above 30)
  against the oracle's restatement of the reference's calcBoysF (src/lible/ints/boys_function.cpp),
  itself pinned to the reference's golden value: 1e-14 relative for every order up to 14.
- The FP32 Boys form of FP32 quartets against the same oracle: 2e-6 relative (single precision).
"""
import numpy as np
import pytest

from lible_b200 import ints as L
from lible_b200.workloads import WATER_BOHR, WATER_Z
from oracle import port

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def s():
    return L.Structure("cc-pvdz", WATER_Z, WATER_BOHR, units="bohr")


def test_exp_neg_within_two_ulp(s):
    rng = np.random.default_rng(5)
    x = np.concatenate([np.linspace(0.0, 700.0, 200001), rng.uniform(0, 700, 100000), rng.uniform(0, 1, 100000),
                        np.arange(0, 701, dtype=float), np.arange(0, 700) * np.log(2.0)])
    y = L.eval_special(s, "exp", x)
    e = np.exp(-x)
    ulps = np.abs(y - e) / np.spacing(e)
    assert ulps.max() <= 2.0, (float(ulps.max()), float(x[np.argmax(ulps)]))


def _boys_sweep():
    return np.concatenate([[0.0, 1e-12, 1e-6, 0.49, 0.5, 0.51, 29.5, 29.999, 30.0, 30.001, 45.0, 117.0, 1e3],
                           np.linspace(0.0, 40.0, 4001)])


@pytest.mark.parametrize("order", [0, 1, 4, 8, 12, 14])
def test_boys_fp64_matches_oracle(s, order):
    x = _boys_sweep()
    F = L.eval_special(s, "boys", x, order)
    ref = np.array([port.boys(order, xi) for xi in x])
    rel = np.abs(F - ref) / np.abs(ref)
    assert rel.max() <= 1e-14, (float(rel.max()), float(x[np.unravel_index(np.argmax(rel), rel.shape)[0]]))


@pytest.mark.parametrize("order", [0, 2, 6, 8])
def test_boys_fp32_form_matches_oracle(s, order):
    x = _boys_sweep()
    F = L.eval_special(s, "boys32", x, order)
    ref = np.array([port.boys(order, xi) for xi in x])
    rel = np.abs(F - ref) / np.abs(ref)
    assert rel.max() <= 2e-6, (float(rel.max()), float(x[np.unravel_index(np.argmax(rel), rel.shape)[0]]))
