"""The library's Zolotarev coefficients (host code of the overlap operator)
against the reference's OverlapOperations::ZolotarevCoefficients compiled from
source, and the approximation property they must have."""
import numpy as np
import pytest

from _oracle import have_reference, ptr, reference
from overlap_b200 import zolotarev

INTERVALS = [(0.05, 30.0), (0.3, 12.0), (1e-3, 40.0), (0.9, 1.1)]


@pytest.mark.parametrize("lo,hi", INTERVALS)
def test_rational_approximates_inverse_sqrt(lo, hi):
    b, d, eps = zolotarev(lo, hi)
    x = np.exp(np.linspace(np.log(lo), np.log(hi), 2001))
    f = np.sqrt(x) * np.sum(b[None, :] / (x[:, None] + d[None, :]), axis=1)
    assert np.max(np.abs(f - 1.0)) < max(2 * eps, 1e-6)
    assert np.all(d > 0)


@pytest.mark.skipif(not have_reference("overlap"), reason="reference not built here")
@pytest.mark.parametrize("lo,hi", INTERVALS)
def test_matches_reference_coefficients(lo, hi):
    R = reference("overlap")
    rb = np.zeros(25)
    rd = np.zeros(25)
    reps = R.ovlref_zolotarev(lo, hi, ptr(rb), ptr(rd))
    b, d, eps = zolotarev(lo, hi)
    # the reference harness is built with FMA contraction; the library's host
    # code without it: the coefficients agree to rounding, the error estimate
    # (a max/min over single-precision sqrtf samples) to 1e-6 relative
    assert np.max(np.abs(b - rb) / np.abs(rb)) < 1e-12
    assert np.max(np.abs(d - rd) / np.abs(rd)) < 1e-12
    assert abs(eps - reps) <= 1e-6 * abs(reps)
