"""GPU parity of the gauge kernels (FP64): link update, staple force, improved
E.B (NCsDot) and the bulk observables, against the oracle and the reference's
golden vectors; Gauss-law preservation of the coupled gauge leapfrog."""
import ctypes as C

import numpy as np
import pytest

from _helpers import oracle_params, rel_err
from _oracle import have_reference, oracle, ptr, reference
from overlap_b200 import Context
from overlap_b200.inputs import random_efield, random_links, volume

pytestmark = pytest.mark.gpu

LATTICES = [(4, 4, 4), (6, 5, 4), (3, 7, 5)]


def ctx_with(N, U, E):
    ctx = Context(N=N, n_modes=32, precision="fp64", form="fused")
    ctx.set_links(U)
    ctx.set_efield(E)
    return ctx


@pytest.mark.parametrize("N", LATTICES)
def test_link_update_matches_oracle(N):
    U = random_links(N, 0.8, 1)
    E = random_efield(N, 0.5, 2)
    p = oracle_params(N)
    oU = U.copy()
    oracle().orc_update_links(C.byref(p), ptr(oU), ptr(E), 0.037)
    with ctx_with(N, U, E) as ctx:
        ctx.update_links(0.037)
        assert rel_err(ctx.get_links(), oU) < 1e-14


@pytest.mark.parametrize("N", LATTICES)
def test_staple_force_matches_oracle(N):
    U = random_links(N, 0.8, 3)
    E = random_efield(N, 0.5, 4)
    p = oracle_params(N)
    oE = E.copy()
    oracle().orc_update_efield(C.byref(p), ptr(U), ptr(oE), 0.05)
    with ctx_with(N, U, E) as ctx:
        ctx.update_efield(0.05)
        assert rel_err(ctx.get_efield(), oE) < 1e-13


@pytest.mark.parametrize("N", LATTICES)
def test_ncsdot_and_bulk_match_oracle(N):
    U = random_links(N, 0.9, 5)
    E = random_efield(N, 0.4, 6)
    p = oracle_params(N)
    ncs = oracle().orc_ncsdot(C.byref(p), ptr(U), ptr(E))
    b = np.zeros(10)
    oracle().orc_bulk(C.byref(p), ptr(U), ptr(E), ptr(b))
    with ctx_with(N, U, E) as ctx:
        assert abs(ctx.ncsdot() - ncs) <= 1e-13 * max(1.0, abs(ncs))
        gb = np.array(list(ctx.bulk().values()))
        assert np.allclose(gb, b, rtol=1e-12, atol=1e-15)


def test_golden_gauge_observables(golden_dir):
    for name in ("wilson_n4", "wilson_n465"):
        g = dict(np.load(golden_dir / f"{name}.npz"))
        N = tuple(int(n) for n in g["N"])
        with ctx_with(N, g["links"], g["efield"]) as ctx:
            assert abs(ctx.ncsdot() - float(g["ncsdot0"])) <= 1e-13 * max(1.0, abs(float(g["ncsdot0"])))
            assert np.allclose(np.array(list(ctx.bulk().values())), g["bulk0"], rtol=1e-12, atol=1e-15)
            ctx.set_links(g["links_after"])
            ctx.update_efield(float(g["dt"]))
            assert rel_err(ctx.get_efield(), g["efield_after_update"]) < 1e-13


def test_gauge_leapfrog_keeps_gauss_law():
    N = (6, 6, 6)
    U = random_links(N, 0.8, 9)
    E = np.zeros((volume(N), 3, 3))
    with ctx_with(N, U, E) as ctx:
        e0 = ctx.bulk()["T00"]
        worst = 0.0
        for _ in range(40):
            ctx.update_efield(0.04)
            ctx.update_links(0.04)
            b = ctx.bulk()
            assert b["gauss_avg"] < 1e-13
            worst = max(worst, abs(b["T00"] - e0) / e0)
        assert worst < 0.1


@pytest.mark.skipif(not have_reference("wilson"), reason="reference library not built")
def test_ncsdot_against_reference_n8():
    N = (8, 8, 8)
    U = random_links(N, 1.2, 11)
    E = random_efield(N, 0.7, 12)
    R = reference("wilson")
    R.ovlref_init(*N, 1, 0, 0.1, 1.0, 0.0, 6.0, 0.05, 1.0, 1)
    R.ovlref_set_links(ptr(U))
    R.ovlref_set_efield(ptr(E))
    ref = R.ovlref_ncsdot()
    with ctx_with(N, U, E) as ctx:
        assert abs(ctx.ncsdot() - ref) <= 1e-13 * max(1.0, abs(ref))


@pytest.mark.skipif(not have_reference("wilson"), reason="reference library not built")
def test_cooled_ncs_update_matches_reference_simpson_rule():
    """Delta N_CS between stored and current links (CoolingMethod::GetDeltaNCs(1),
    cooling off) against the reference's GeodesicInterpolation + NCsDot."""
    N = (6, 4, 5)
    U0 = random_links(N, 0.8, 41)
    E = random_efield(N, 0.6, 42)
    p = oracle_params(N)
    U1 = U0.copy()
    for _ in range(5):
        oracle().orc_update_links(C.byref(p), ptr(U1), ptr(E), 0.05)
    R = reference("wilson")
    R.ovlref_init(*N, 1, 0, 0.1, 1.0, 0.0, 6.0, 0.05, 1.0, 1)
    ref = R.ovlref_delta_ncs(ptr(U0), ptr(U1))
    with ctx_with(N, U0, E) as ctx:
        assert ctx.ncs_update() == (0.0, 0.0)
        ctx.set_links(U1)
        d, total = ctx.ncs_update()
        assert abs(d - ref) <= 1e-13 * max(1.0, abs(ref))
        assert total == d
        # U_new became U_old: no further change
        d2, total2 = ctx.ncs_update()
        assert abs(d2) < 1e-15 and abs(total2 - total) < 1e-15
