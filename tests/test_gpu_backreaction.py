"""GPU fermion back-reaction and fermion energy against the oracle
(orc_color_force, orc_fermion_energy, orc_coupled_leapfrog), and link
reunitarisation.  The back-reaction has no reference counterpart (the
reference keeps E fixed under the fermions, FERMIONS/WILSON/Update.cpp:48-79);
the oracle's force is pinned on the CPU by finite differences of H_F
(test_backreaction_oracle.py)."""
import ctypes as C

import numpy as np
import pytest

from _helpers import oracle_params, random_modes, rel_err
from _oracle import oracle, ptr
from overlap_b200 import Context, OvlError
from overlap_b200.inputs import random_efield, random_links, volume

pytestmark = pytest.mark.gpu

N = (5, 4, 6)


def force_scale(psi):
    V = psi.shape[1]
    return float(psi.shape[0] * np.max(np.sum(np.abs(psi) ** 2, axis=(2, 3))) / (2.0 * V))


def oracle_force(p, U, psi, first):
    out = np.zeros((volume(p.N), 3, 3))
    oracle().orc_color_force(C.byref(p), ptr(U), ptr(np.ascontiguousarray(psi).view(np.float64)), psi.shape[0], first,
                             ptr(out))
    return out


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_color_force_and_energy_match_oracle(precision):
    n = 70  # three mode blocks, the last one partial
    U = random_links(N, 0.6, 301)
    psi = random_modes(n, N, 302)
    p = oracle_params(N, m=0.15, mdw=0.0, dt=0.04)
    of = oracle_force(p, U, psi, 5)
    oe = oracle().orc_fermion_energy(C.byref(p), ptr(U), ptr(psi.view(np.float64)), n, 5)
    with Context(N=N, n_modes=n, first_mode=5, precision=precision, form="fused", m_fermion=0.15, m_dw=0.0,
                 dt=0.04) as ctx:
        ctx.set_links(U)
        ctx.set_modes(psi, psi)
        f = ctx.color_force()
        e = ctx.fermion_energy()
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert np.max(np.abs(f - of)) <= tol * force_scale(psi)
    assert abs(e - oe) <= tol * force_scale(psi) * volume(N)


def test_color_force_with_u1_background_matches_oracle():
    n = 40
    U = random_links(N, 0.5, 311)
    psi = random_modes(n, N, 312)
    ph = np.exp(1j * np.random.default_rng(313).uniform(-np.pi, np.pi, (N[1], N[0], 2)))
    phf = np.ascontiguousarray(ph).view(np.float64).ravel()
    p = oracle_params(N, m=0.1)
    oracle().orc_set_u1(ptr(phf))
    try:
        of = oracle_force(p, U, psi, 0)
    finally:
        oracle().orc_set_u1(None)
    with Context(N=N, n_modes=n, precision="fp64", m_fermion=0.1, m_dw=0.0) as ctx:
        ctx.set_links(U)
        ctx.set_u1(ph)
        ctx.set_modes(psi, psi)
        f = ctx.color_force()
    assert np.max(np.abs(f - of)) <= 1e-12 * force_scale(psi)


@pytest.mark.parametrize("form", ["plain", "fused"])
def test_coupled_evolution_matches_oracle(form):
    n, steps, g2 = 40, 4, 3.0
    U = random_links(N, 0.5, 321)
    E = random_efield(N, 0.2, 322)
    psi0 = random_modes(n, N, 323)
    mid0 = random_modes(n, N, 324)
    p = oracle_params(N, m=0.1, mdw=0.0, dt=0.04)
    oU, oE, opsi, omid = U.copy(), E.copy(), psi0.copy(), mid0.copy()
    t = C.c_int(0)
    oracle().orc_coupled_leapfrog(C.byref(p), ptr(oU), ptr(oE), ptr(opsi.view(np.float64)), ptr(omid.view(np.float64)),
                                  n, 2, C.byref(t), steps, g2, 1)
    with Context(N=N, n_modes=n, first_mode=2, precision="fp64", form=form, m_fermion=0.1, m_dw=0.0, dt=0.04,
                 t_sphaleron=1e9, gauge_force=True, backreaction=g2) as ctx:
        ctx.set_links(U)
        ctx.set_efield(E)
        ctx.set_modes(psi0, mid0)
        ctx.step(steps)
        psi, mid = ctx.get_modes()
        assert rel_err(psi, opsi) < 1e-12
        assert rel_err(mid, omid) < 1e-12
        assert rel_err(ctx.get_links(), oU) < 1e-13
        assert rel_err(ctx.get_efield(), oE) < 1e-12
    assert rel_err(oE, E) > 1e-3  # the field did move


def test_backreaction_is_rejected_for_overlap_fermions():
    with pytest.raises(OvlError):
        Context(N=(4, 4, 4), n_modes=4, fermion="overlap", backreaction=1.0)


def test_reunitarize_projects_links_onto_su2():
    n = 8
    U = random_links(N, 0.5, 331) * 1.001  # off the group by 1e-3
    E = random_efield(N, 0.2, 332)
    psi0 = random_modes(n, N, 333)
    with Context(N=N, n_modes=n, precision="fp64", form="fused", dt=0.04, t_sphaleron=1e9, reunitarize=True) as ctx:
        ctx.set_links(U)
        ctx.set_efield(E)
        ctx.set_modes(psi0, psi0)
        ctx.step(2)
        b = ctx.bulk()
    assert b["unitarity_max"] < 1e-14
    with Context(N=N, n_modes=n, precision="fp64", form="fused", dt=0.04, t_sphaleron=1e9) as ctx:
        ctx.set_links(U)
        ctx.set_efield(E)
        ctx.step(2)
        assert ctx.bulk()["unitarity_max"] > 1e-4  # the reference keeps the deviation
