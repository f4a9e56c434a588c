"""U(1) background in the hopping term (an extension: the reference couples
its U(1) field only into the initial eigenmodes).  Checked against the oracle
with the same phases, and by U(1) gauge covariance: with phases
u'_mu(x) = g(x) u_mu(x) g(x+mu)^* and modes psi' = g psi, the evolution gives
g times the evolution of (u, psi)."""
import ctypes as C

import numpy as np
import pytest

from _helpers import current_scale, oracle_currents, oracle_leapfrog, oracle_params, random_modes, rel_err
from _oracle import oracle, ptr
from overlap_b200 import Context
from overlap_b200.inputs import random_efield, random_links, volume

pytestmark = pytest.mark.gpu

N = (5, 4, 6)


def flux_phases(N, nb):
    p = oracle_params(N)
    out = np.zeros(4 * N[0] * N[1])
    oracle().orc_u1_flux(C.byref(p), nb, ptr(out))
    return out.view(np.complex128).reshape(N[1], N[0], 2)


@pytest.mark.parametrize("precision,form", [("fp64", "plain"), ("fp64", "fused"), ("fp32", "fused")])
def test_u1_leapfrog_and_currents_match_oracle(precision, form):
    n = 40
    U = random_links(N, 0.6, 201)
    E = random_efield(N, 0.3, 202)
    psi0 = random_modes(n, N, 203)
    mid0 = random_modes(n, N, 204)
    u1 = flux_phases(N, 3)
    u1f = np.ascontiguousarray(u1).view(np.float64).ravel()
    oracle().orc_set_u1(ptr(u1f))
    try:
        p = oracle_params(N, m=0.1, mdw=0.0, dt=0.04)
        opsi, omid, oU, _ = oracle_leapfrog(p, U, E, psi0, mid0, 4)
        ocur = oracle_currents(p, oU, opsi, 3)
    finally:
        oracle().orc_set_u1(None)
    with Context(N=N, n_modes=n, first_mode=3, precision=precision, form=form, m_fermion=0.1, m_dw=0.0, dt=0.04,
                 t_sphaleron=1e9) as ctx:
        ctx.set_links(U)
        ctx.set_efield(E)
        ctx.set_u1(u1)
        ctx.set_modes(psi0, mid0)
        ctx.step(4)
        psi, mid = ctx.get_modes()
        tol = 1e-12 if precision == "fp64" else 2e-5
        assert rel_err(psi, opsi) < tol
        assert rel_err(mid, omid) < tol
        cur = ctx.currents()
        scale = current_scale(opsi)
        for k in ocur:
            assert np.max(np.abs(cur[k] - ocur[k])) <= (1e-12 if precision == "fp64" else 1e-5) * scale, k


def test_u1_gauge_covariance():
    n = 32
    U = random_links(N, 0.5, 211)
    psi0 = random_modes(n, N, 212)
    mid0 = random_modes(n, N, 213)
    u1 = flux_phases(N, 2)
    rng = np.random.default_rng(214)
    alpha = rng.uniform(0, 2 * np.pi, size=(N[1], N[0]))  # depends on (x, y) only
    g = np.exp(1j * alpha)
    gp = np.empty_like(u1)
    gp[:, :, 0] = g * u1[:, :, 0] * np.conj(np.roll(g, -1, axis=1))
    gp[:, :, 1] = g * u1[:, :, 1] * np.conj(np.roll(g, -1, axis=0))
    site_g = np.tile(g.ravel(), N[2])  # site = x + N0 (y + N1 z)
    out = {}
    for name, ph, a, b in (("orig", u1, psi0, mid0), ("gauged", gp, psi0 * site_g[None, :, None, None],
                                                    mid0 * site_g[None, :, None, None])):
        with Context(N=N, n_modes=n, precision="fp64", form="fused", m_fermion=0.05, m_dw=0.0, dt=0.05) as ctx:
            ctx.set_links(U)
            ctx.set_u1(ph)
            ctx.set_modes(a, b)
            ctx.step(5)
            out[name] = ctx.get_modes()[0]
            out[name + "_charges"] = ctx.charges()
    assert rel_err(out["gauged"], out["orig"] * site_g[None, :, None, None]) < 1e-12
    for k in ("NV", "N5", "PS", "WA"):
        assert abs(out["gauged_charges"][k] - out["orig_charges"][k]) < 1e-10


def test_u1_unit_phases_change_nothing():
    U = random_links(N, 0.5, 221)
    psi0 = random_modes(8, N, 222)
    res = []
    for ph in (None, np.ones((N[1], N[0], 2), np.complex128)):
        # one fixed hop variant; the phase-dressed kernel is compiled separately
        # (FMA contraction may differ), so agreement is to rounding
        with Context(N=N, n_modes=8, precision="fp64", form="fused", m_fermion=0.05, m_dw=0.0, dt=0.05,
                     hop_variant=0) as ctx:
            ctx.set_links(U)
            ctx.set_u1(ph)
            ctx.set_modes(psi0, psi0)
            ctx.step(3)
            res.append(ctx.get_modes()[0])
    assert rel_err(res[1], res[0]) < 1e-14
