"""GPU parity of the overlap operator (batched multi-shift CG, FP64) with the
reference's overlap code compiled from source (oracle/_ref/libovlref_overlap.so).

The reference draws the start vector of its Ritz bound estimate from its RNG
(FERMIONS/OVERLAP/OverlapUpdate.cpp:66-84); the tests replay the bounds the
reference used, through ovl_set_spectral_bounds.  The reference's Zolotarev
approximation is accurate to ~1e-7 (single-precision square roots in its
coefficients) and its CG stops at a relative residual ~1e-8: both sides run the
same coefficients and the same per-mode stopping rule, and agree to 1e-11."""
import functools

import numpy as np
import pytest

from _helpers import current_scale, random_modes, rel_err
from _oracle import have_reference, ptr, reference
from overlap_b200 import Context
from overlap_b200.inputs import random_efield, random_links, volume

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not have_reference("overlap"), reason="reference overlap build not present")]

TOL = 1e-11


def ref_setup(N, nranks, rank, m, r, mdw, tsph, dt, U, E):
    R = reference("overlap")
    nm = R.ovlref_init(*N, nranks, rank, m, r, mdw, tsph, dt, 1.0, 7)
    R.ovlref_set_links(ptr(U))
    R.ovlref_set_efield(ptr(E))
    return R, nm


def test_overlap_operator_matches_reference():
    N = (4, 4, 4)
    U = random_links(N, 0.5, 101)
    E = np.zeros((volume(N), 3, 3))
    R, _ = ref_setup(N, 16, 0, 0.1, 1.0, 1.4, 6.0, 0.05, U, E)
    b = np.zeros(2)
    R.ovlref_ritz_bounds(ptr(b))
    phis = random_modes(20, N, 102)
    ref = np.zeros_like(phis)
    for i in range(phis.shape[0]):
        R.ovlref_apply(ptr(phis[i].view(np.float64)), ptr(ref[i].view(np.float64)), b[0], b[1])
    with Context(N=N, n_modes=20, fermion="overlap", precision="fp64", m_fermion=0.1, r_wilson=1.0, m_dw=1.4,
                 dt=0.05) as ctx:
        ctx.set_links(U)
        ctx.set_spectral_bounds([b])
        out = ctx.apply(phis)
        st = ctx.solver_stats()
    assert st["not_converged"] == 0 and st["iterations"] > 5
    assert rel_err(out, ref) < TOL


def test_overlap_operator_is_anti_hermitian():
    """D = -i h_ov with h_ov hermitian: <a, D b> = -<D a, b>."""
    N = (4, 4, 4)
    U = random_links(N, 0.6, 111)
    R, _ = ref_setup(N, 16, 0, 0.0, 1.0, 1.4, 6.0, 0.05, U, np.zeros((volume(N), 3, 3)))
    b = np.zeros(2)
    R.ovlref_ritz_bounds(ptr(b))
    ab = random_modes(2, N, 112)
    with Context(N=N, n_modes=2, fermion="overlap", m_fermion=0.0, m_dw=1.4) as ctx:
        ctx.set_links(U)
        ctx.set_spectral_bounds([b])
        d = ctx.apply(ab)
    lhs = np.vdot(ab[0], d[1])
    rhs = -np.vdot(d[0], ab[1])
    assert abs(lhs - rhs) <= 1e-7 * np.linalg.norm(ab[0]) * np.linalg.norm(d[1])


def test_overlap_leapfrog_and_currents_match_reference():
    N = (4, 4, 4)
    m, r, mdw, dt, tsph, steps = 0.1, 1.0, 1.4, 0.05, 1e9, 2
    U = random_links(N, 0.4, 121)
    E = random_efield(N, 0.2, 122)
    R, nm = ref_setup(N, 16, 5, m, r, mdw, tsph, dt, U, E)
    first = R.ovlref_first_mode()
    R.ovlref_set_free_fermions()  # free overlap spinors (GetOverlapDiracSpinor, FermionField.cpp:331-517)
    V = volume(N)
    psi0 = np.zeros((nm, V, 2, 4), np.complex128)
    mid0 = np.zeros_like(psi0)
    R.ovlref_get_modes(ptr(psi0.view(np.float64)), ptr(mid0.view(np.float64)))
    scratch = np.zeros(64)
    R.ovlref_take_bounds(ptr(scratch), 32)  # clear
    R.ovlref_step(steps)
    bounds = np.zeros(64)
    nb = R.ovlref_take_bounds(ptr(bounds), 64)
    assert nb == 4 * steps  # (min, max) after each of the 2*steps half steps
    rpsi = np.zeros_like(psi0)
    rmid = np.zeros_like(psi0)
    R.ovlref_get_modes(ptr(rpsi.view(np.float64)), ptr(rmid.view(np.float64)))
    rU = np.zeros_like(U)
    R.ovlref_get_links(ptr(rU))
    rcur = [np.zeros(4 * V) for _ in range(2)]
    assert R.ovlref_currents(ptr(rcur[0]), ptr(rcur[1]), None, None, None, None) == 2
    cb = np.zeros(2)
    R.ovlref_last_bounds(ptr(cb))

    with Context(N=N, n_modes=nm, first_mode=first, fermion="overlap", precision="fp64", m_fermion=m, r_wilson=r,
                 m_dw=mdw, dt=dt, t_sphaleron=tsph) as ctx:
        ctx.set_links(U)
        ctx.set_efield(E)
        ctx.set_modes(psi0, mid0)
        ctx.set_spectral_bounds(bounds[:nb].reshape(-1, 2))
        ctx.step(steps)
        psi, mid = ctx.get_modes()
        assert rel_err(psi, rpsi) < TOL
        assert rel_err(mid, rmid) < TOL
        assert rel_err(ctx.get_links(), rU) < 1e-13
        ctx.set_spectral_bounds([cb])
        cur = ctx.currents()
    scale = current_scale(rpsi)
    assert np.max(np.abs(cur["jV"].ravel() - rcur[0])) <= TOL * scale
    assert np.max(np.abs(cur["jA"].ravel() - rcur[1])) <= TOL * scale


def test_chebyshev_sign_agrees_with_zolotarev_form():
    """Chebyshev series of x^(-1/2) (degree 200 on [0.9 lambda_min / lambda_max, 1])
    against the reference's Zolotarev form on the same links and bounds; the
    Zolotarev coefficients are accurate to ~1e-7, so the forms agree to 1e-6.
    FP32 Chebyshev agrees with FP64 Chebyshev to 1e-5, also with the D passes
    in the packed-pair kernel (hop variant 3)."""
    N = (4, 4, 4)
    U = random_links(N, 0.5, 131)
    R, _ = ref_setup(N, 16, 0, 0.1, 1.0, 1.4, 6.0, 0.05, U, np.zeros((volume(N), 3, 3)))
    b = np.zeros(2)
    R.ovlref_ritz_bounds(ptr(b))
    eps = 0.9 * b[0] / b[1]
    phis = random_modes(12, N, 132)
    outs = {}
    for name, kw in (("zolo", dict(precision="fp64")),
                     ("cheb64", dict(precision="fp64", sign_method="chebyshev", cheb_degree=200, cheb_eps=eps)),
                     ("cheb32", dict(precision="fp32", sign_method="chebyshev", cheb_degree=200, cheb_eps=eps)),
                     ("cheb32p", dict(precision="fp32", sign_method="chebyshev", cheb_degree=200, cheb_eps=eps,
                                      hop_variant=3))):
        with Context(N=N, n_modes=12, fermion="overlap", m_fermion=0.1, m_dw=1.4, dt=0.05, **kw) as ctx:
            ctx.set_links(U)
            ctx.set_spectral_bounds([b])
            outs[name] = ctx.apply(phis)
            if name != "zolo":
                assert ctx.solver_stats()["not_converged"] == 0
    assert rel_err(outs["cheb64"], outs["zolo"]) < 1e-6
    assert rel_err(outs["cheb32"], outs["cheb64"]) < 1e-5
    assert rel_err(outs["cheb32p"], outs["cheb64"]) < 1e-5


def test_chebyshev_overlap_leapfrog_fp32_runs_and_conserves_norm():
    """FP32 Chebyshev overlap leapfrog: h_ov is hermitian, so the leapfrog keeps
    the mode norms bounded; the charges stay finite."""
    N = (4, 4, 4)
    U = random_links(N, 0.4, 141)
    R, _ = ref_setup(N, 16, 0, 0.1, 1.0, 1.4, 6.0, 0.05, U, np.zeros((volume(N), 3, 3)))
    b = np.zeros(2)
    R.ovlref_ritz_bounds(ptr(b))
    psi0 = random_modes(32, N, 142)
    with Context(N=N, n_modes=32, fermion="overlap", precision="fp32", sign_method="chebyshev", cheb_degree=96,
                 cheb_eps=0.9 * b[0] / b[1], m_fermion=0.1, m_dw=1.4, dt=0.05) as ctx:
        ctx.set_links(U)
        ctx.set_spectral_bounds([b])
        ctx.set_modes(psi0, psi0)
        n0 = np.sum(np.abs(psi0) ** 2)
        ctx.step(10)
        psi, _ = ctx.get_modes()
        assert abs(np.sum(np.abs(psi) ** 2) / n0 - 1.0) < 0.2
        assert np.isfinite(ctx.charges()["N5"])


def _embedded_chebyshev_oracle(N, U, E, psi, mid, steps, K, eps, lmax, m, mdw, dt):
    """The FP64 Chebyshev overlap leapfrog of two colours: the three-colour
    oracle (orc3_overlap_leapfrog) on the fields embedded in the upper-left
    colour block, where the third colour is free and stays empty (the
    embedding reproduces every two-colour oracle function, tests/test_oracle_su3.py).
    Returns the two-colour modes, the links and N_5 of the final modes."""
    import ctypes as C

    from _helpers import oracle_params
    from _oracle import oracle
    from overlap_b200.inputs import embed_su2_efield, embed_su2_links

    def f64(a):
        return np.ascontiguousarray(a).view(np.float64)

    def embed(q):
        out = np.zeros(q.shape[:2] + (3, 4), complex)
        out[:, :, :2, :] = q
        return out

    p = oracle_params(N, m=m, mdw=mdw, dt=dt)
    U3, E3 = embed_su2_links(U).copy(), embed_su2_efield(E)
    o_psi, o_mid = embed(psi), embed(mid)
    t = C.c_int(0)
    oracle().orc3_overlap_leapfrog(C.byref(p), ptr(f64(U3)), ptr(f64(E3)), ptr(f64(o_psi)), ptr(f64(o_mid)),
                                   psi.shape[0], C.byref(t), steps, K, eps, lmax)
    O = np.zeros_like(o_psi)
    for k in range(psi.shape[0]):
        oracle().orc3_overlap_apply(C.byref(p), ptr(f64(U3)), ptr(f64(o_psi[k])), ptr(f64(O[k])), K, eps, lmax)
    # overlap N_5 (OverlapCurrents.cpp:35-212): local bilinears with O = -i h_ov psi
    g5 = np.array([[0, 0, 1, 0], [0, 0, 0, 1], [1, 0, 0, 0], [0, 1, 0, 0]], complex)
    g0 = np.diag([1, 1, -1, -1]).astype(complex)
    w = np.where(np.arange(psi.shape[0]) % 2 == 0, 1.0, -1.0)
    a1 = np.einsum("msca,ab,mscb->m", np.conj(o_psi), g5, o_psi).real
    a2 = np.einsum("msca,ab,mscb->m", np.conj(o_psi), g5 @ g0, O).imag
    n5 = float(np.sum(w * (a1 + 0.5 * a2)) / (2 * volume(N)))
    scale = float(np.sum(np.abs(a1 + 0.5 * a2)) / (2 * volume(N)))  # the size of the summed mode terms
    assert np.max(np.abs(o_psi[:, :, 2, :])) == 0.0
    return o_psi[:, :, :2, :], o_mid[:, :, :2, :], n5, scale


_CHEB_CASE = dict(N=(4, 4, 4), m=0.05, mdw=1.0, dt=0.05, K=96, eps=0.01, steps=100, modes=16)


@functools.lru_cache(maxsize=1)
def _cheb_case():
    c = _CHEB_CASE
    N = c["N"]
    lmax = (0.5 * abs(6 + 2 * c["m"] - 2 * c["mdw"]) + 3.0) ** 2  # the context's bound without a schedule
    U, E = random_links(N, 0.5, 151), random_efield(N, 0.2, 152)
    psi0, mid0 = random_modes(c["modes"], N, 153), random_modes(c["modes"], N, 154)
    want = _embedded_chebyshev_oracle(N, U, E, psi0, mid0, c["steps"], c["K"], c["eps"], lmax, c["m"], c["mdw"], c["dt"])
    return U, E, psi0, mid0, want


@pytest.mark.parametrize("precision,variant", [("fp64", 0), ("fp32", 0), ("fp32", 3)])
def test_chebyshev_overlap_leapfrog_matches_the_fp64_oracle(precision, variant):
    """Two colours, 100 leapfrog steps with moving links, Chebyshev degree 96
    on the analytic bound: the modes and N_5 against the FP64 Chebyshev
    oracle leapfrog.  FP64 to 1e-10; FP32 (the serving and bench form) to
    1e-4 in the fields and, in the axial charge, 1e-5 of the summed size of
    the modes' terms (N_5 sums terms of alternating sign, which cancel: the
    error is measured against the terms, not against their small sum;
    measured: fields 1.2e-6, N_5 7e-7 absolute)."""
    c = _CHEB_CASE
    N, m, mdw, dt, K, eps, steps = c["N"], c["m"], c["mdw"], c["dt"], c["K"], c["eps"], c["steps"]
    U, E, psi0, mid0, (o_psi, o_mid, n5, n5_scale) = _cheb_case()
    with Context(N=N, n_modes=c["modes"], fermion="overlap", sign_method="chebyshev", cheb_degree=K, cheb_eps=eps,
                 m_fermion=m, m_dw=mdw, dt=dt, precision=precision, hop_variant=variant) as ctx:
        ctx.set_links(U)
        ctx.set_efield(E)
        ctx.set_modes(psi0, mid0)
        ctx.step(steps)
        g_psi, g_mid = ctx.get_modes()
        g_n5 = ctx.charges()["N5"]
    err = max(rel_err(g_psi, o_psi), rel_err(g_mid, o_mid))
    n5_err = abs(g_n5 - n5) / n5_scale
    print(f"{precision} v{variant}: fields {err:.2e}, N5 {g_n5:.12e} vs {n5:.12e} (of the terms {n5_err:.2e})")
    if precision == "fp64":
        assert err < 1e-10 and n5_err < 1e-10
    else:
        assert err < 1e-4 and n5_err < 1e-5


@pytest.mark.skipif(not have_reference("overlap"), reason="reference overlap build absent")
@pytest.mark.parametrize("precision,sign", [("fp64", "zolotarev"), ("fp32", "chebyshev")])
def test_overlap_plane_waves_match_reference(precision, sign):
    """ovl_set_free_fermions on an overlap context gives the reference's
    overlap plane waves (GetOverlapDiracSpinor, FermionField.cpp:331-517)."""
    N = (4, 5, 6)
    R = reference("overlap")
    m = R.ovlref_init(*N, 4, 2, 0.05, 1.0, 1.2, 1e9, 0.05, 1.0, 1)
    first = R.ovlref_first_mode()
    R.ovlref_set_free_fermions()
    V = volume(N)
    rpsi = np.zeros((m, V, 2, 4), np.complex128)
    rmid = np.zeros_like(rpsi)
    R.ovlref_get_modes(ptr(rpsi.view(np.float64)), ptr(rmid.view(np.float64)))
    with Context(N=N, n_modes=m, first_mode=first, fermion="overlap", sign_method=sign, precision=precision,
                 m_fermion=0.05, m_dw=1.2, dt=0.05, t_sphaleron=1e9) as ctx:
        ctx.set_free_fermions()  # N1 = 5 odd: some axis-branch spinors fail the eigen check, as the reference's
        psi, mid = ctx.get_modes()
    tol = 1e-14 if precision == "fp64" else 1e-7
    assert rel_err(psi, rpsi) < tol and rel_err(mid, rmid) < tol


def test_overlap_beyond_one_cta_row_of_mode_blocks():
    """300 modes = 10 mode blocks (the last 12 of 32 lanes) on N = (4, 5, 5),
    V = 100, whose last CTA of 8 sites holds 4: the Zolotarev form against the
    reference's own application on modes of both rows of mode blocks (the
    stopping rule leaves 3e-11 here), the Chebyshev form (a recurrence per mode)
    on the last modes against a context that holds only those, and against the
    reference to the Zolotarev approximation's 1e-6."""
    N = (4, 5, 5)
    U = random_links(N, 0.5, 151)
    R, _ = ref_setup(N, 16, 0, 0.1, 1.0, 1.4, 6.0, 0.05, U, np.zeros((volume(N), 3, 3)))
    b = np.zeros(2)
    R.ovlref_ritz_bounds(ptr(b))
    phis = random_modes(300, N, 152)
    pick = list(range(0, 256, 51)) + list(range(256, 300, 9))
    ref = np.zeros((len(pick),) + phis.shape[1:], phis.dtype)
    for j, i in enumerate(pick):
        R.ovlref_apply(ptr(np.ascontiguousarray(phis[i]).view(np.float64)), ptr(ref[j].view(np.float64)), b[0], b[1])
    with Context(N=N, n_modes=300, fermion="overlap", precision="fp64", m_fermion=0.1, r_wilson=1.0, m_dw=1.4,
                 dt=0.05) as ctx:
        ctx.set_links(U)
        ctx.set_spectral_bounds([b])
        out = ctx.apply(phis)
        assert ctx.solver_stats()["not_converged"] == 0
    assert rel_err(out[pick], ref) < 5e-11
    eps = 0.9 * b[0] / b[1]
    cheb = dict(fermion="overlap", precision="fp64", sign_method="chebyshev", cheb_degree=200, cheb_eps=eps,
                m_fermion=0.1, r_wilson=1.0, m_dw=1.4, dt=0.05)
    with Context(N=N, n_modes=300, **cheb) as ctx:
        ctx.set_links(U)
        ctx.set_spectral_bounds([b])
        outc = ctx.apply(phis)
    with Context(N=N, n_modes=44, **cheb) as ctx:
        ctx.set_links(U)
        ctx.set_spectral_bounds([b])
        outs = ctx.apply(phis[256:])
    assert rel_err(outc[256:], outs) < 1e-13
    assert rel_err(outc[pick], ref) < 1e-6


@pytest.mark.parametrize("method", ["zolotarev", "chebyshev"])
def test_overlap_link_table_mode_blocks_per_cta(method):
    """In FP64 the stencils of both sign methods run up to 8 mode blocks per CTA
    on links gathered once in shared memory (fewer while the grid would hold
    under 4 CTAs per SM).  On N = (7, 7, 7), V = 343, 3400 modes (107 mode
    blocks) give 8 per CTA on a 148-SM B200, 72 modes one: the last 72 modes of
    the large context against a context that holds only them.  Each mode's
    Chebyshev recurrence is its own (1e-13); the multi-shift CG stops each mode
    by its own residual (1e-11)."""
    N = (7, 7, 7)
    U = random_links(N, 0.5, 161)
    phis = random_modes(3400, N, 162)
    kw = dict(fermion="overlap", precision="fp64", m_fermion=0.1, r_wilson=1.0, m_dw=1.4, dt=0.05)
    with Context(N=N, n_modes=1, **kw) as ctx:
        ctx.set_links(U)
        b = np.array(ctx.ritz_bounds(phis[0])["bounds"])
    if method == "chebyshev":
        kw.update(sign_method="chebyshev", cheb_degree=120, cheb_eps=0.9 * b[0] / b[1])
    with Context(N=N, n_modes=3400, **kw) as ctx:
        ctx.set_links(U)
        ctx.set_spectral_bounds([b])
        out = ctx.apply(phis)
    with Context(N=N, n_modes=72, **kw) as ctx:
        ctx.set_links(U)
        ctx.set_spectral_bounds([b])
        sub = ctx.apply(phis[3328:])
    assert rel_err(out[3328:], sub) < (1e-13 if method == "chebyshev" else 1e-11)
