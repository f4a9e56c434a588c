"""GPU Ritz solver for the overlap spectral bounds (ovl_ritz_bounds) against
the reference's RitzSolver (golden fixtures made by tests/golden/make_golden.py
from FERMIONS/OVERLAP/OPERATOR/RitzSolver.cpp) and the oracle restatement
(orc_ritz), and the overlap leapfrog with bounds computed on the GPU before
every half step (ritz_auto) against the reference, which computes them from
its own random start vectors (OverlapUpdate.cpp:100-125).  The extreme
eigenvalues do not depend on the start vector beyond the iteration's
round-off stagnation (~1e-12 relative)."""
import ctypes as C

import numpy as np
import pytest

from _helpers import current_scale, oracle_params, random_modes, rel_err
from _oracle import have_reference, oracle, ptr, reference
from overlap_b200 import Context
from overlap_b200.inputs import random_efield, random_links, volume

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["ritz_n4", "ritz_n465"])
def test_ritz_matches_golden(golden_dir, name):
    g = dict(np.load(golden_dir / f"{name}.npz"))
    N = tuple(int(n) for n in g["N"])
    with Context(N=N, n_modes=4, fermion="overlap", m_fermion=float(g["m_fermion"]), r_wilson=float(g["r_wilson"]),
                 m_dw=float(g["m_dw"])) as ctx:
        ctx.set_links(g["links"])
        r = ctx.ritz_bounds(g["start"])
    lo, hi = float(g["lambda_min"]), float(g["lambda_max"])
    assert abs(r["raw"][0] - lo) <= 1e-12 * lo
    assert abs(r["raw"][1] - hi) <= 1e-12 * hi
    assert r["bounds"] == pytest.approx((0.95 * r["raw"][0], 1.05 * r["raw"][1]), rel=1e-15)
    assert all(10 < n < 2000 for n in r["iters"])


def test_ritz_random_start_and_u1_background_match_oracle():
    N = (5, 4, 6)
    V = volume(N)
    U = random_links(N, 0.4, 401)
    ph = np.exp(1j * np.random.default_rng(402).uniform(-np.pi, np.pi, (N[1], N[0], 2)))
    p = oracle_params(N, m=0.05, mdw=1.3)
    start = np.random.default_rng(403).uniform(0, 1, (V, 2, 4)) + 1j * np.random.default_rng(404).uniform(0, 1, (V, 2, 4))
    oracle().orc_set_u1(ptr(np.ascontiguousarray(ph).view(np.float64).ravel()))
    try:
        it = C.c_int(0)
        lo = oracle().orc_ritz(C.byref(p), ptr(U), ptr(start.view(np.float64)), 1.0, 2000, 100, 1e-16, C.byref(it))
        hi = -oracle().orc_ritz(C.byref(p), ptr(U), ptr(start.view(np.float64)), -1.0, 2000, 100, 1e-16, C.byref(it))
    finally:
        oracle().orc_set_u1(None)
    with Context(N=N, n_modes=4, fermion="overlap", m_fermion=0.05, m_dw=1.3, ritz_seed=7) as ctx:
        ctx.set_links(U)
        ctx.set_u1(ph)
        same = ctx.ritz_bounds(start)
        r1 = ctx.ritz_bounds()
        r2 = ctx.ritz_bounds()  # the next start vector of the generator
    assert abs(same["raw"][0] - lo) <= 1e-12 * lo and abs(same["raw"][1] - hi) <= 1e-12 * hi
    for r in (r1, r2):
        assert abs(r["raw"][0] - lo) <= 1e-11 * lo and abs(r["raw"][1] - hi) <= 1e-11 * hi
    assert r1["iters"] != r2["iters"] or r1["raw"] != r2["raw"]  # different start vectors


@pytest.mark.skipif(not have_reference("overlap"), reason="reference overlap build not present")
def test_overlap_leapfrog_with_gpu_ritz_bounds_matches_reference():
    N = (4, 4, 4)
    m, r, mdw, dt, steps = 0.1, 1.0, 1.4, 0.05, 2
    U = random_links(N, 0.4, 411)
    E = random_efield(N, 0.2, 412)
    R = reference("overlap")
    nm = R.ovlref_init(*N, 16, 5, m, r, mdw, 1e9, dt, 1.0, 7)
    R.ovlref_set_links(ptr(U))
    R.ovlref_set_efield(ptr(E))
    first = R.ovlref_first_mode()
    R.ovlref_set_free_fermions()
    V = volume(N)
    psi0 = np.zeros((nm, V, 2, 4), np.complex128)
    mid0 = np.zeros_like(psi0)
    R.ovlref_get_modes(ptr(psi0.view(np.float64)), ptr(mid0.view(np.float64)))
    R.ovlref_step(steps)
    rpsi, rmid = np.zeros_like(psi0), np.zeros_like(psi0)
    R.ovlref_get_modes(ptr(rpsi.view(np.float64)), ptr(rmid.view(np.float64)))
    rcur = [np.zeros(4 * V) for _ in range(2)]
    R.ovlref_currents(ptr(rcur[0]), ptr(rcur[1]), None, None, None, None)
    with Context(N=N, n_modes=nm, first_mode=first, fermion="overlap", precision="fp64", m_fermion=m, r_wilson=r,
                 m_dw=mdw, dt=dt, t_sphaleron=1e9, ritz_auto=True, ritz_seed=3) as ctx:
        ctx.set_links(U)
        ctx.set_efield(E)
        ctx.set_modes(psi0, mid0)
        ctx.step(steps)
        psi, mid = ctx.get_modes()
        cur = ctx.currents()
    assert rel_err(psi, rpsi) < 1e-10
    assert rel_err(mid, rmid) < 1e-10
    scale = current_scale(rpsi)
    assert np.max(np.abs(cur["jV"].ravel() - rcur[0])) <= 1e-10 * scale
    assert np.max(np.abs(cur["jA"].ravel() - rcur[1])) <= 1e-10 * scale


def test_overlap_without_bounds_or_ritz_auto_is_an_error():
    from overlap_b200 import OvlError
    with Context(N=(4, 4, 4), n_modes=4, fermion="overlap", m_dw=1.4) as ctx:
        ctx.set_links(random_links((4, 4, 4), 0.3, 1))
        with pytest.raises(OvlError):
            ctx.step(1)


def dense_hw3(N, U, m, mdw, u1=None):
    """h_W of three colours as a dense matrix, column by column from the
    oracle's -i h_W (orc3_wilson_apply), reference layout [V][3][4]."""
    p = oracle_params(N, m=m, mdw=mdw)
    D = 12 * volume(N)
    H = np.zeros((D, D), complex)
    Uf = np.ascontiguousarray(U).view(np.float64)
    if u1 is not None:
        oracle().orc_set_u1(ptr(np.ascontiguousarray(u1).view(np.float64).ravel()))
    try:
        e, out = np.zeros(D, complex), np.zeros(D, complex)
        for k in range(D):
            e[:] = 0.0
            e[k] = 1.0
            oracle().orc3_wilson_apply(C.byref(p), ptr(Uf), ptr(e.view(np.float64)), ptr(out.view(np.float64)))
            H[:, k] = 1j * out
    finally:
        oracle().orc_set_u1(None)
    return H


@pytest.mark.parametrize("with_u1", [False, True])
def test_three_colour_ritz_finds_the_extreme_eigenvalues(with_u1):
    """The Ritz iteration on the three-colour h_W^2 converges to the smallest
    and the largest eigenvalue of the dense matrix."""
    from overlap_b200.inputs import random_links_su3

    N = (4, 3, 4)
    V = volume(N)
    U = random_links_su3(N, 0.6, 501)
    ph = np.exp(1j * np.random.default_rng(502).uniform(-np.pi, np.pi, (N[1], N[0], 2))) if with_u1 else None
    H = dense_hw3(N, U, 0.05, 1.3, ph)
    assert np.max(np.abs(H - H.conj().T)) < 1e-13
    w2 = np.linalg.eigvalsh(H) ** 2
    lo, hi = w2.min(), w2.max()
    rng = np.random.default_rng(503)
    start = rng.uniform(0, 1, (V, 3, 4)) + 1j * rng.uniform(0, 1, (V, 3, 4))
    with Context(N=N, n_colours=3, n_modes=4, fermion="overlap", sign_method="chebyshev", m_fermion=0.05, m_dw=1.3,
                 ritz_seed=9) as ctx:
        ctx.set_links(U)
        if with_u1:
            ctx.set_u1(ph)
        r = ctx.ritz_bounds(start)
        r2 = ctx.ritz_bounds()  # from the context's generator
    for q in (r, r2):
        assert abs(q["raw"][0] - lo) <= 1e-10 * hi and abs(q["raw"][1] - hi) <= 1e-10 * hi
    assert r["bounds"] == pytest.approx((0.95 * r["raw"][0], 1.05 * r["raw"][1]), rel=1e-15)


def test_three_colour_overlap_with_ritz_bounds_before_every_application():
    """ritz_auto on a three-colour Chebyshev overlap context: every application
    scales h_W^2 by 1.05 times the Ritz lambda_max, so it equals a context given
    those bounds as a schedule (to the Ritz iteration's round-off), and differs
    from the analytic bound's scaling."""
    from overlap_b200.inputs import random_links_su3

    N = (4, 4, 4)
    V = volume(N)
    U = random_links_su3(N, 0.5, 601)
    rng = np.random.default_rng(602)
    phi = rng.normal(size=(6, V, 3, 4)) + 1j * rng.normal(size=(6, V, 3, 4))
    kw = dict(N=N, n_colours=3, n_modes=6, fermion="overlap", sign_method="chebyshev", cheb_degree=48, cheb_eps=0.01,
              m_fermion=0.05, m_dw=1.0, precision="fp64")
    with Context(ritz_auto=1, ritz_seed=3, **kw) as a:
        a.set_links(U)
        b = a.ritz_bounds()["bounds"]
        out_a = a.apply(phi)
    with Context(**kw) as c:
        c.set_links(U)
        c.set_spectral_bounds([b])
        out_b = c.apply(phi)
        c.set_spectral_bounds([(0.01 * 25.0, 25.0)])  # the analytic bound (|6r - 2M|/2 + 3)^2 + 2m terms aside
        out_loose = c.apply(phi)
    scale = np.max(np.abs(out_b))
    assert np.max(np.abs(out_a - out_b)) < 1e-9 * scale
    assert np.max(np.abs(out_loose - out_b)) > 1e-6 * scale
    assert b[1] < 25.0
