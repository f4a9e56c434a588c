"""Three colours on the GPU against the three-colour oracle (orc3_*, itself
pinned through the SU(2) embedding and gauge covariance in
test_oracle_su3.py): the Wilson operator and leapfrog in both forms and
precisions, the link update, the charges, E.B, Delta N_CS, the bulk
observables, the staple force, plane waves, Z2 stochastic modes and the
Chebyshev overlap operator and leapfrog.  Tolerances: 1e-12 relative for FP64
(1e-13 for the links), 2e-5 for FP32 modes (FP32 links and arithmetic)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from _helpers import oracle_params, rel_err
from _oracle import oracle, ptr
from overlap_b200 import Context, OvlError
from overlap_b200.inputs import (embed_su2_efield, embed_su2_links, random_efield_su3, random_links,
                                 random_links_su3, u1_flux, unit_links_su3, volume)

pytestmark = pytest.mark.gpu

N = (4, 3, 5)
M = 40
TOL = {"fp64": 1e-12, "fp32": 2e-5}


def f64(a):
    return np.ascontiguousarray(a).view(np.float64)


def modes3(n, seed):
    rng = np.random.default_rng(seed)
    shape = (n, volume(N), 3, 4)
    return (rng.normal(0, np.sqrt(0.5), shape) + 1j * rng.normal(0, np.sqrt(0.5), shape)).astype(np.complex128)


def ctx3(precision="fp64", form="fused", **kw):
    base = dict(N=N, n_colours=3, n_modes=M, precision=precision, form=form, m_fermion=0.1, m_dw=0.0, dt=0.05,
                t_sphaleron=1e9, device=0)
    base.update(kw)
    return Context(**base)


def oracle_leapfrog3(p, U, E, psi, mid, steps):
    U = f64(U).copy()
    psi = psi.copy()
    mid = mid.copy()
    t = C.c_int(0)
    oracle().orc3_wilson_leapfrog(C.byref(p), ptr(U), ptr(np.ascontiguousarray(E)), ptr(f64(psi)), ptr(f64(mid)),
                                  psi.shape[0], C.byref(t), steps)
    return psi, mid, U.view(np.complex128).reshape(-1, 3, 9)


@pytest.mark.parametrize("precision,variant", [("fp64", 0), ("fp32", 0), ("fp32", 3)])
@pytest.mark.parametrize("u1", [False, True])
def test_wilson_operator(precision, variant, u1):
    """Variant 0: the scalar stencil; 3: the packed-pair FP32 stencil (V = 60:
    a partial last CTA of 8 sites; 40 modes: a half-empty second mode block)."""
    U = random_links_su3(N, 0.8, 1)
    phi = modes3(M, 2)
    p = oracle_params(N, m=0.1)
    ph = u1_flux(N, 2) if u1 else None
    if u1:
        oracle().orc_set_u1(ptr(np.ascontiguousarray(ph).view(np.float64)))
    try:
        want = np.zeros_like(phi)
        for m in range(M):
            oracle().orc3_wilson_apply(C.byref(p), ptr(f64(U)), ptr(f64(phi[m])), ptr(f64(want[m])))
    finally:
        oracle().orc_set_u1(None)
    with ctx3(precision, hop_variant=variant) as ctx:
        ctx.set_links(U)
        if u1:
            ctx.set_u1(ph)
        got = ctx.apply(phi)
        assert ctx.tuning()[0] == variant
    assert rel_err(got, want) < TOL[precision]


@pytest.mark.parametrize("precision,form,variant", [("fp64", "plain", 0), ("fp64", "fused", 0), ("fp32", "fused", 0),
                                                    ("fp32", "plain", 0), ("fp32", "fused", 3), ("fp32", "plain", 3)])
def test_leapfrog_with_moving_links(precision, form, variant):
    U = random_links_su3(N, 0.7, 3)
    E = random_efield_su3(N, 0.4, 4)
    psi, mid = modes3(M, 5), modes3(M, 6)
    p = oracle_params(N, m=0.1, dt=0.05)
    o_psi, o_mid, o_U = oracle_leapfrog3(p, U, E, psi, mid, 4)
    with ctx3(precision, form, plain_chunk_modes=32, hop_variant=variant) as ctx:
        ctx.set_links(U)
        ctx.set_efield(E)
        ctx.set_modes(psi, mid)
        ctx.step(4)
        assert ctx.tuning()[0] == variant
        g_psi, g_mid = ctx.get_modes()
        assert rel_err(ctx.get_links(), o_U) < 1e-13
    assert max(rel_err(g_psi, o_psi), rel_err(g_mid, o_mid)) < TOL[precision]


def test_embedded_su2_leapfrog_equals_two_colour_context():
    """A three-colour run with SU(2) embedded and the third colour empty is the
    two-colour run (whose kernels equal the reference's)."""
    U2 = random_links(N, 0.6, 7)
    E2 = np.random.default_rng(8).normal(0, 0.3, (volume(N), 3, 3))
    rng = np.random.default_rng(9)
    psi2 = rng.normal(size=(M, volume(N), 2, 4)) + 1j * rng.normal(size=(M, volume(N), 2, 4))
    mid2 = rng.normal(size=(M, volume(N), 2, 4)) + 1j * rng.normal(size=(M, volume(N), 2, 4))
    with Context(N=N, n_modes=M, precision="fp64", form="fused", m_fermion=0.1, m_dw=0.0, dt=0.05, t_sphaleron=1e9,
                 hop_variant=0) as c2:
        c2.set_links(U2)
        c2.set_efield(E2)
        c2.set_modes(psi2, mid2)
        c2.step(3)
        a_psi, _ = c2.get_modes()
        a_ch = c2.charges()
    psi3 = np.zeros((M, volume(N), 3, 4), np.complex128)
    mid3 = np.zeros_like(psi3)
    psi3[:, :, :2], mid3[:, :, :2] = psi2, mid2
    with ctx3("fp64") as c3:
        c3.set_links(embed_su2_links(U2))
        c3.set_efield(embed_su2_efield(E2))
        c3.set_modes(psi3, mid3)
        c3.step(3)
        b_psi, _ = c3.get_modes()
        b_ch = c3.charges()
    assert rel_err(b_psi[:, :, :2], a_psi) < 1e-12 and np.abs(b_psi[:, :, 2]).max() == 0.0
    for k in a_ch:
        assert abs(a_ch[k] - b_ch[k]) <= 1e-12 * max(1.0, abs(a_ch[k])), k


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_charges(precision):
    U = random_links_su3(N, 0.9, 10)
    psi = modes3(M, 11)
    p = oracle_params(N, m=0.1)
    want = np.zeros(4)
    oracle().orc3_charges(C.byref(p), ptr(f64(U)), ptr(f64(psi)), M, 0, ptr(want))
    with ctx3(precision) as ctx:
        ctx.set_links(U)
        ctx.set_modes(psi, psi)
        got = ctx.charges()
    scale = M * np.max(np.sum(np.abs(psi) ** 2, axis=(2, 3))) / (2 * volume(N))
    tol = 1e-12 if precision == "fp64" else 1e-6
    for k, key in enumerate(("NV", "N5", "PS", "WA")):
        assert abs(got[key] - want[k]) <= tol * scale, key


def test_ncsdot_delta_ncs_bulk_and_staple_force():
    U0 = random_links_su3(N, 0.8, 12)
    E = random_efield_su3(N, 0.5, 13)
    p = oracle_params(N)
    with ctx3("fp64") as ctx:
        ctx.set_links(U0)
        ctx.set_efield(E)
        want = oracle().orc3_ncsdot(C.byref(p), ptr(f64(U0)), ptr(E))
        assert abs(ctx.ncsdot() - want) <= 1e-12 * max(1.0, abs(want))
        b = np.zeros(10)
        oracle().orc3_bulk(C.byref(p), ptr(f64(U0)), ptr(E), ptr(b))
        got = ctx.bulk()
        vals = np.array([got[k] for k in ("T00", "TXX", "TYY", "TZZ", "electric", "magnetic", "gauss_max",
                                           "gauss_avg", "unitarity_max", "unitarity_avg")])
        assert np.abs(vals[:8] - b[:8]).max() <= 1e-12 * np.abs(b[:6]).max()
        assert abs(vals[8] - b[8]) < 1e-14 and abs(vals[9] - b[9]) < 1e-14
        # Delta N_CS between the stored links and links five half-updates later
        assert ctx.ncs_update() == (0.0, 0.0)
        U1 = f64(U0).copy()
        for _ in range(5):
            oracle().orc3_update_links(C.byref(p), ptr(U1), ptr(E), 0.05)
            ctx.update_links(0.05)
        assert rel_err(ctx.get_links(), U1.view(np.complex128).reshape(-1, 3, 9)) < 1e-13
        d, total = ctx.ncs_update()
        ref = oracle().orc3_delta_ncs(C.byref(p), ptr(f64(U0)), ptr(U1))
        assert abs(d - ref) <= 1e-12 * max(1.0, abs(ref)) and total == d
        # staple force
        E2 = E.copy()
        oracle().orc3_update_efield(C.byref(p), ptr(U1), ptr(E2), 0.03)
        ctx.update_efield(0.03)
        assert rel_err(ctx.get_efield(), E2) < 1e-13


def test_reunitarized_links_stay_special_unitary():
    U = random_links_su3(N, 0.8, 14)
    E = random_efield_su3(N, 2.0, 15)
    with ctx3("fp64", reunitarize=True) as ctx:
        ctx.set_links(U)
        ctx.set_efield(E)
        for _ in range(50):
            ctx.update_links(0.3)
        M3 = np.swapaxes(ctx.get_links().reshape(-1, 3, 3), -1, -2)
    assert np.abs(M3 @ np.conj(np.swapaxes(M3, -1, -2)) - np.eye(3)).max() < 1e-14
    assert np.abs(np.linalg.det(M3) - 1).max() < 1e-14


NE = (4, 4, 6)  # even sizes for plane waves (odd N takes the reference's axis branch at k = (N-1)/2)


def test_plane_waves():
    V = volume(NE)
    n = 12 * V
    p = oracle_params(NE, m=0.1, dt=0.05)
    psi = np.zeros((n, V, 3, 4), np.complex128)
    mid = np.zeros_like(psi)
    assert oracle().orc3_free_fermions(C.byref(p), 0, n, ptr(f64(psi)), ptr(f64(mid))) == 0
    with ctx3("fp64", n_modes=n, N=NE) as ctx:
        assert ctx.set_free_fermions() == 0
        g_psi, g_mid = ctx.get_modes()
    assert rel_err(g_psi, psi) < 1e-13 and rel_err(g_mid, mid) < 1e-13


def _vacuum_energy(ctx, psi):
    """(1/2V) sum_m w_m <psi_m, h psi_m>, h = i D."""
    d = ctx.apply(psi)
    w = np.where(np.arange(psi.shape[0]) % 2 == 0, 1.0, -1.0)
    return float(np.sum(w * np.einsum("msca,msca->m", np.conj(psi), 1j * d).real) / (2 * ctx.V))


def test_stochastic_modes_reproduce_the_vacuum_energy():
    V = volume(NE)
    with ctx3("fp64", n_modes=12 * V, N=NE) as ctx:
        ctx.set_links(unit_links_su3(NE))
        ctx.set_free_fermions()
        e_pw = _vacuum_energy(ctx, ctx.get_modes()[0])
    for pairs in (1, 5):
        with ctx3("fp64", n_modes=2 * pairs, N=NE) as ctx:
            ctx.set_links(unit_links_su3(NE))
            ctx.set_stochastic_modes(seed=21)
            psi, mid = ctx.get_modes()
            assert abs(_vacuum_energy(ctx, psi) - e_pw) <= 1e-12 * abs(e_pw)
            assert np.allclose(np.sum(np.abs(psi) ** 2, axis=(1, 2, 3)), np.sum(np.abs(mid) ** 2, axis=(1, 2, 3)))


def _overlap_kw(precision):
    return dict(fermion="overlap", sign_method="chebyshev", cheb_degree=48, cheb_eps=0.01, m_fermion=0.05, m_dw=1.0,
                precision=precision, form="fused")


@pytest.mark.parametrize("precision,variant", [("fp64", 0), ("fp32", 0), ("fp32", 3)])
def test_chebyshev_overlap_operator_and_leapfrog(precision, variant):
    U = random_links_su3(N, 0.6, 16)
    E = random_efield_su3(N, 0.3, 17)
    phi = modes3(40, 18)  # two mode blocks: the split recurrence
    mid = modes3(40, 19)
    p = oracle_params(N, m=0.05, mdw=1.0, dt=0.05)
    lmax = (0.5 * abs(6 + 2 * 0.05 - 2 * 1.0) + 3.0) ** 2  # the context's default bound on h_W^2
    want = np.zeros_like(phi)
    for m in range(40):
        oracle().orc3_overlap_apply(C.byref(p), ptr(f64(U)), ptr(f64(phi[m])), ptr(f64(want[m])), 48, 0.01, lmax)
    t = C.c_int(0)
    o_psi, o_mid, o_U = phi.copy(), mid.copy(), f64(U).copy()
    oracle().orc3_overlap_leapfrog(C.byref(p), ptr(o_U), ptr(E), ptr(f64(o_psi)), ptr(f64(o_mid)), 40, C.byref(t), 2, 48,
                                   0.01, lmax)
    tol = 1e-11 if precision == "fp64" else 1e-4
    with ctx3(n_modes=40, hop_variant=variant, **_overlap_kw(precision)) as ctx:
        ctx.set_links(U)
        ctx.set_efield(E)
        assert rel_err(ctx.apply(phi), want) < tol
        ctx.set_modes(phi, mid)
        ctx.step(2)
        g_psi, g_mid = ctx.get_modes()
        ch = ctx.charges()
        assert rel_err(ctx.get_links(), o_U.view(np.complex128).reshape(-1, 3, 9)) < 1e-13
    assert max(rel_err(g_psi, o_psi), rel_err(g_mid, o_mid)) < tol
    # overlap N_5: local bilinears with O = -i h_ov psi (OverlapCurrents.cpp:35-212, three colours)
    O = np.zeros_like(o_psi)
    for m in range(40):
        oracle().orc3_overlap_apply(C.byref(p), ptr(o_U), ptr(f64(o_psi[m])), ptr(f64(O[m])), 48, 0.01, lmax)
    g5 = np.array([[0, 0, 1, 0], [0, 0, 0, 1], [1, 0, 0, 0], [0, 1, 0, 0]], complex)
    g0 = np.diag([1, 1, -1, -1]).astype(complex)
    w = np.where(np.arange(40) % 2 == 0, 1.0, -1.0)
    a1 = np.einsum("msca,ab,mscb->m", np.conj(o_psi), g5, o_psi).real
    a2 = np.einsum("msca,ab,mscb->m", np.conj(o_psi), g5 @ g0, O).imag
    n5 = float(np.sum(w * (a1 + 0.5 * a2)) / (2 * volume(N)))
    assert abs(ch["N5"] - n5) <= (1e-10 if precision == "fp64" else 1e-4) * max(1.0, abs(n5))


def test_packed_stencil_beyond_one_cta_row_of_mode_blocks():
    """300 modes = 10 mode blocks (the last 12 of 32 lanes): a CTA of the packed
    three-colour kernel runs 8 mode blocks, so a second row of CTAs holds blocks
    8 and 9.  Fused leapfrog with moving links and a U(1) background against
    the oracle with the same phases."""
    n = 300
    U = random_links_su3(N, 0.7, 31)
    E = random_efield_su3(N, 0.4, 32)
    psi, mid = modes3(n, 33), modes3(n, 34)
    ph = u1_flux(N, 2)
    p = oracle_params(N, m=0.1, dt=0.05)
    oracle().orc_set_u1(ptr(np.ascontiguousarray(ph).view(np.float64)))
    try:
        o_psi, o_mid, o_U = oracle_leapfrog3(p, U, E, psi, mid, 3)
    finally:
        oracle().orc_set_u1(None)
    with ctx3("fp32", "fused", n_modes=n, hop_variant=3) as ctx:
        ctx.set_links(U)
        ctx.set_efield(E)
        ctx.set_u1(ph)
        ctx.set_modes(psi, mid)
        ctx.step(3)
        g_psi, g_mid = ctx.get_modes()
    assert max(rel_err(g_psi, o_psi), rel_err(g_mid, o_mid)) < TOL["fp32"]


@pytest.mark.parametrize("fermion", ["wilson", "overlap"])
def test_autotune_chooses_between_the_three_colour_stencils(fermion):
    """FP32 three-colour contexts time the scalar (0) and packed (3) stencils;
    the state is kept, and FP64 contexts have the scalar stencil only."""
    kw = _overlap_kw("fp32") if fermion == "overlap" else dict(precision="fp32", form="fused")
    with ctx3(n_modes=40, **kw) as ctx:
        U = random_links_su3(N, 0.5, 41)
        ctx.set_links(U)
        ctx.set_modes(modes3(40, 42), modes3(40, 43))
        before = ctx.get_modes()
        v, ms = ctx.autotune()
        assert v in (0, 3) and ms[0] > 0 and ms[3] > 0 and ms[1] == ms[2] == 0
        assert ctx.tuning()[0] == v
        after = ctx.get_modes()
        assert np.array_equal(before[0], after[0]) and np.array_equal(before[1], after[1])
    with ctx3("fp64", "fused") as ctx:
        ctx.set_links(random_links_su3(N, 0.5, 44))
        v, ms = ctx.autotune()
        assert v == 0


def test_three_colour_limits_are_reported():
    for kw in (dict(precision="fp40"), dict(fermion="overlap", sign_method="zolotarev"), dict(n_colours=4)):
        with pytest.raises(OvlError):
            ctx3(**kw)



def test_gauss_restore():
    """GaussLawRestoration::Restore for three colours against the oracle, on
    quasi-particle fields (SetQuasiParticles restores Gauss's law after the
    transform)."""
    from overlap_b200.inputs import quasi_particles

    U, E = quasi_particles(N, 4.0, 1.0, seed=22, n_colours=3)
    p = oracle_params(N)
    Eo = E.copy()
    out = np.zeros(2)
    n = oracle().orc3_gauss_restore(C.byref(p), ptr(f64(U)), ptr(Eo), 10000, 1e-14, ptr(out))
    with ctx3("fp64") as ctx:
        ctx.set_links(U)
        ctx.set_efield(E)
        r = ctx.gauss_restore(10000, 1e-14)
        assert r["iterations"] == n and r["max"] <= 1e-14
        assert rel_err(ctx.get_efield(), Eo) < 1e-12
        assert ctx.bulk()["gauss_max"] <= 1e-14


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_back_reaction_force_energy_and_coupled_leapfrog(precision):
    """The fermion force on E, the fermion energy and the coupled step (gauge
    force and back-reaction g^2 = 0.7) against the three-colour oracle."""
    U = random_links_su3(N, 0.6, 40)
    E = random_efield_su3(N, 0.3, 41)
    psi, mid = modes3(M, 42), modes3(M, 43)
    p = oracle_params(N, m=0.1, dt=0.05)
    F = np.zeros((volume(N), 3, 8))
    oracle().orc3_color_force(C.byref(p), ptr(f64(U)), ptr(f64(psi)), M, 0, ptr(F))
    h = oracle().orc3_fermion_energy(C.byref(p), ptr(f64(U)), ptr(f64(psi)), M, 0)
    o_U, o_E, o_psi, o_mid = f64(U).copy(), E.copy(), psi.copy(), mid.copy()
    t = C.c_int(0)
    oracle().orc3_coupled_leapfrog(C.byref(p), ptr(o_U), ptr(o_E), ptr(f64(o_psi)), ptr(f64(o_mid)), M, 0, C.byref(t),
                                   3, 0.7, 1)
    tol = TOL[precision]
    with ctx3(precision, gauge_force=True, backreaction=0.7) as ctx:
        ctx.set_links(U)
        ctx.set_efield(E)
        ctx.set_modes(psi, mid)
        assert rel_err(ctx.color_force(), F) < (1e-12 if precision == "fp64" else 1e-5)
        assert abs(ctx.fermion_energy() - h) <= (1e-12 if precision == "fp64" else 1e-6) * abs(h)
        ctx.step(3)
        assert rel_err(ctx.get_efield(), o_E) < (1e-12 if precision == "fp64" else 1e-5)
        assert rel_err(ctx.get_modes()[0], o_psi) < tol


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_currents_embed_su2_and_sum_to_the_charges(precision):
    """Per-site Wilson currents for three colours: with SU(2) embedded and the
    third colour empty they are the two-colour context's (pinned to the
    reference); for SU(3) fields their lattice sums are the oracle's charges."""
    U2 = random_links(N, 0.6, 44)
    rng = np.random.default_rng(45)
    psi2 = rng.normal(size=(M, volume(N), 2, 4)) + 1j * rng.normal(size=(M, volume(N), 2, 4))
    with Context(N=N, n_modes=M, first_mode=1, precision=precision, form="fused", m_fermion=0.1, m_dw=0.0,
                 dt=0.05, t_sphaleron=1e9, hop_variant=0) as c2:
        c2.set_links(U2)
        c2.set_u1(u1_flux(N, 2))
        c2.set_modes(psi2, psi2)
        cur2 = c2.currents()
    psi3 = np.zeros((M, volume(N), 3, 4), np.complex128)
    psi3[:, :, :2] = psi2
    with ctx3(precision, first_mode=1) as c3:
        c3.set_links(embed_su2_links(U2))
        c3.set_u1(u1_flux(N, 2))
        c3.set_modes(psi3, psi3)
        cur3 = c3.currents()
    for k in cur2:
        scale = max(1.0, np.abs(cur2[k]).max())
        assert np.abs(cur3[k] - cur2[k]).max() <= (1e-12 if precision == "fp64" else 1e-6) * scale, k
    U = random_links_su3(N, 0.8, 46)
    psi = modes3(M, 47)
    want = np.zeros(4)
    oracle().orc3_charges(C.byref(oracle_params(N, m=0.1)), ptr(f64(U)), ptr(f64(psi)), M, 0, ptr(want))
    with ctx3(precision) as ctx:
        ctx.set_links(U)
        ctx.set_modes(psi, psi)
        cur = ctx.currents()
    got = [cur["jV"][:, 0].sum(), cur["jA"][:, 0].sum(), cur["PS"].sum(), cur["WA"].sum()]
    scale = M * np.max(np.sum(np.abs(psi) ** 2, axis=(2, 3))) / (2 * volume(N))
    # FP32 contexts store the modes rounded to FP32: the oracle's FP64 modes differ by that
    assert np.abs(np.array(got) - want).max() <= (1e-11 if precision == "fp64" else 1e-6) * scale
