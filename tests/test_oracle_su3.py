"""The three-colour oracle (oracle/ovl_oracle.c, orc3_*) on the CPU.

The reference has no three-colour fermions and its SU(3) group code does not
build, so the SU(3) oracle is pinned in two ways: (1) with SU(2) embedded in
the upper-left colour block every orc3_* function reproduces its two-colour
counterpart, which is pinned to the reference compiled from source; (2)
properties that hold for any SU(3) field -- gauge covariance of the Wilson
operator, unitarity of the link exponential against numpy's eigensolver,
plane waves as eigenmodes of the free operator, and the Chebyshev overlap
operator against a dense evaluation of the same polynomial.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from _helpers import oracle_leapfrog, oracle_params, random_modes, rel_err
from _oracle import have_reference, oracle, ptr, reference
from overlap_b200.inputs import (embed_su2_efield, embed_su2_links, random_efield, random_efield_su3, random_links,
                                 random_links_su3, su3_exp, su3_pack, su3_unpack, unit_links_su3, volume)


def f64(a):
    return np.ascontiguousarray(a).view(np.float64)


def random_modes3(n, N, seed):
    rng = np.random.default_rng(seed)
    shape = (n, volume(N), 3, 4)
    return (rng.normal(0, np.sqrt(0.5), shape) + 1j * rng.normal(0, np.sqrt(0.5), shape)).astype(np.complex128)


def embed_modes(psi2):
    out = np.zeros(psi2.shape[:2] + (3, 4), dtype=np.complex128)
    out[:, :, :2, :] = psi2
    return out


def test_exp_matches_eigh_and_is_special_unitary():
    rng = np.random.default_rng(1)
    for k in range(20):
        alpha = rng.normal(0, 1.5, 8)
        c = float(rng.normal())
        out = np.zeros(18)
        oracle().orc3_exp(c, ptr(alpha), ptr(out))
        M = su3_unpack(out.view(np.complex128))
        assert np.abs(M - su3_exp(alpha, c)).max() < 1e-13
        assert np.abs(M @ M.conj().T - np.eye(3)).max() < 1e-13
        assert abs(np.linalg.det(M) - 1) < 1e-13
    # degenerate spectrum (alpha along lambda_8) and zero
    for alpha in (np.eye(8)[7] * 0.9, np.zeros(8)):
        out = np.zeros(18)
        oracle().orc3_exp(0.4, ptr(alpha), ptr(out))
        assert np.abs(su3_unpack(out.view(np.complex128)) - su3_exp(alpha, 0.4)).max() < 1e-14


def test_embedded_su2_link_update_and_staple_force():
    N = (3, 4, 5)
    U2 = random_links(N, 0.8, 2)
    E2 = random_efield(N, 0.5, 3)
    p = oracle_params(N)
    U3 = f64(embed_su2_links(U2)).copy()
    E3 = embed_su2_efield(E2)
    oracle().orc_update_links(C.byref(p), ptr(U2), ptr(E2), 0.07)
    oracle().orc3_update_links(C.byref(p), ptr(U3), ptr(E3), 0.07)
    assert np.abs(U3.view(np.complex128).reshape(-1, 3, 9) - embed_su2_links(U2)).max() < 1e-14
    oracle().orc_update_efield(C.byref(p), ptr(U2), ptr(E2), 0.03)
    oracle().orc3_update_efield(C.byref(p), ptr(U3), ptr(E3), 0.03)
    assert np.abs(E3[..., :3] - E2).max() < 1e-14 and np.abs(E3[..., 3:]).max() < 1e-14


def test_embedded_su2_wilson_leapfrog_and_charges():
    N = (4, 3, 4)
    U2 = random_links(N, 0.6, 4)
    E2 = random_efield(N, 0.4, 5)
    psi2 = random_modes(6, N, 6)
    mid2 = random_modes(6, N, 7)
    p = oracle_params(N, m=0.1)
    o_psi, o_mid, o_U, _ = oracle_leapfrog(p, U2, E2, psi2, mid2, 3)
    U3 = f64(embed_su2_links(U2)).copy()
    psi3 = embed_modes(psi2)
    mid3 = embed_modes(mid2)
    t = C.c_int(0)
    oracle().orc3_wilson_leapfrog(C.byref(p), ptr(U3), ptr(embed_su2_efield(E2)), ptr(f64(psi3)), ptr(f64(mid3)), 6,
                                  C.byref(t), 3)
    assert rel_err(psi3[:, :, :2], o_psi) < 1e-13 and np.abs(psi3[:, :, 2]).max() == 0.0
    assert rel_err(mid3[:, :, :2], o_mid) < 1e-13
    assert np.abs(U3.view(np.complex128).reshape(-1, 3, 9) - embed_su2_links(o_U)).max() < 1e-13
    # charges: lattice sums of the two-colour currents
    V = volume(N)
    cur = [np.zeros(4 * V) for _ in range(4)] + [np.zeros(V), np.zeros(V)]
    oracle().orc_wilson_currents(C.byref(p), ptr(o_U), ptr(f64(o_psi)), 6, 1, *[ptr(a) for a in cur])
    want = [cur[0].reshape(V, 4)[:, 0].sum(), cur[1].reshape(V, 4)[:, 0].sum(), cur[4].sum(), cur[5].sum()]
    got = np.zeros(4)
    oracle().orc3_charges(C.byref(p), ptr(U3), ptr(f64(psi3)), 6, 1, ptr(got))
    assert np.abs(got - want).max() < 1e-13 * max(1.0, np.abs(want).max())


def test_embedded_su2_ncsdot_bulk_and_delta_ncs():
    N = (4, 5, 3)
    U2 = random_links(N, 0.9, 8)
    E2 = random_efield(N, 0.7, 9)
    p = oracle_params(N)
    U3 = f64(embed_su2_links(U2))
    E3 = embed_su2_efield(E2)
    a = oracle().orc_ncsdot(C.byref(p), ptr(U2), ptr(E2))
    b = oracle().orc3_ncsdot(C.byref(p), ptr(U3), ptr(E3))
    assert abs(a - b) < 1e-13 * max(1.0, abs(a))
    o2 = np.zeros(10)
    o3 = np.zeros(10)
    oracle().orc_bulk(C.byref(p), ptr(U2), ptr(E2), ptr(o2))
    oracle().orc3_bulk(C.byref(p), ptr(U3), ptr(E3), ptr(o3))
    o3[7] *= np.sqrt(8.0 / 3.0)  # the Gauss rms runs over the Nc^2 - 1 components (GaussLawViolation.cpp:64)
    assert np.abs(o2[:8] - o3[:8]).max() < 1e-13 * np.abs(o2[:8]).max()
    # Gauss restoration: the embedded run is the two-colour one
    E2r, E3r = E2.copy(), E3.copy()
    n2 = oracle().orc_gauss_restore(C.byref(p), ptr(U2), ptr(E2r), 10000, 1e-14, ptr(np.zeros(2)))
    n3 = oracle().orc3_gauss_restore(C.byref(p), ptr(U3), ptr(E3r), 10000, 1e-14, ptr(np.zeros(2)))
    assert n2 == n3 and np.abs(E3r[..., :3] - E2r).max() < 1e-13 and np.abs(E3r[..., 3:]).max() < 1e-14
    if have_reference("wilson"):
        U2b = U2.copy()
        for _ in range(5):
            oracle().orc_update_links(C.byref(p), ptr(U2b), ptr(E2), 0.05)
        R = reference("wilson")
        R.ovlref_init(*N, 1, 0, 0.1, 1.0, 0.0, 6.0, 0.05, 1.0, 1)
        ref = R.ovlref_delta_ncs(ptr(U2), ptr(U2b))
        d = oracle().orc3_delta_ncs(C.byref(p), ptr(U3), ptr(f64(embed_su2_links(U2b))))
        assert abs(d - ref) < 1e-12 * max(1.0, abs(ref))


def test_delta_ncs_follows_the_link_update_path():
    """With E fixed the links move along exp(i c E t) U: the geodesic between two
    configurations is that path, so Delta N_CS is the Simpson sum of NCsDot at
    the two ends and the midpoint of the actual trajectory."""
    N = (3, 3, 4)
    U0 = f64(random_links_su3(N, 0.7, 10)).copy()
    E = random_efield_su3(N, 0.5, 11)
    p = oracle_params(N)
    Um = U0.copy()
    oracle().orc3_update_links(C.byref(p), ptr(Um), ptr(E), 0.1)
    U1 = Um.copy()
    oracle().orc3_update_links(C.byref(p), ptr(U1), ptr(E), 0.1)
    d = oracle().orc3_delta_ncs(C.byref(p), ptr(U0), ptr(U1))
    # E_mid of the geodesic = 0.2 E (cU = -dt), NCsDot is linear in E
    f = [oracle().orc3_ncsdot(C.byref(p), ptr(u), ptr(np.ascontiguousarray(0.2 * E))) for u in (U0, Um, U1)]
    assert abs(d - (f[0] + 4 * f[1] + f[2]) / 6) < 1e-12 * max(1.0, abs(d))


def _gauge_transform(U, psi, N, seed):
    V = volume(N)
    g = su3_exp(np.random.default_rng(seed).normal(0, 2.0, (V, 8)))
    M = su3_unpack(U.reshape(V, 3, 9))
    n0, n1 = N[0], N[0] * N[1]
    idx = np.arange(V)
    x, y, z = idx % N[0], (idx // N[0]) % N[1], idx // n1
    fwd = [((x + 1) % N[0]) + n0 * y + n1 * z, x + n0 * ((y + 1) % N[1]) + n1 * z, x + n0 * y + n1 * ((z + 1) % N[2])]
    Mg = np.stack([g @ M[:, mu] @ np.conj(np.swapaxes(g[fwd[mu]], -1, -2)) for mu in range(3)], axis=1)
    psig = np.einsum("sij,msja->msia", g, psi)
    return su3_pack(Mg), psig, g


def test_wilson_operator_is_gauge_covariant():
    N = (3, 4, 3)
    U = random_links_su3(N, 1.0, 12)
    psi = random_modes3(1, N, 13)
    p = oracle_params(N, m=0.2, mdw=0.3)
    out = np.zeros_like(psi)
    oracle().orc3_wilson_apply(C.byref(p), ptr(f64(U)), ptr(f64(psi)), ptr(f64(out)))
    Ug, psig, g = _gauge_transform(U, psi, N, 14)
    outg = np.zeros_like(psi)
    oracle().orc3_wilson_apply(C.byref(p), ptr(f64(Ug)), ptr(f64(psig)), ptr(f64(outg)))
    assert rel_err(outg, np.einsum("sij,msja->msia", g, out)) < 1e-13


def test_plane_waves_are_free_eigenmodes():
    N = (4, 4, 4)
    V = volume(N)
    p = oracle_params(N, m=0.1, dt=0.05)
    n = 12 * V
    psi = np.zeros((n, V, 3, 4), dtype=np.complex128)
    mid = np.zeros_like(psi)
    assert oracle().orc3_free_fermions(C.byref(p), 0, n, ptr(f64(psi)), ptr(f64(mid))) == 0
    U = f64(unit_links_su3(N))
    for m in (0, 1, 5, 77, n - 1):
        out = np.zeros((V, 3, 4), dtype=np.complex128)
        oracle().orc3_wilson_apply(C.byref(p), ptr(U), ptr(f64(psi[m])), ptr(f64(out)))
        # D psi = -i omega psi, psimid = e^{-i omega dt / 2} psi
        lam = np.vdot(psi[m], out) / np.vdot(psi[m], psi[m])
        assert abs(lam.real) < 1e-13 and np.abs(out - lam * psi[m]).max() < 1e-12
        assert np.abs(mid[m] - np.exp(0.5 * lam * 0.05) * psi[m]).max() < 1e-13
    # every colour carries the same spectrum: the basis is complete
    norms = np.einsum("msca,msca->mc", np.conj(psi), psi).real
    assert np.allclose(norms.sum(0), [4 * V * V] * 3)


def _dense_wilson(p, U, N):
    V = volume(N)
    dim = 12 * V
    D = np.zeros((dim, dim), dtype=np.complex128)
    for k in range(dim):
        e = np.zeros(dim, dtype=np.complex128)
        e[k] = 1.0
        out = np.zeros(dim, dtype=np.complex128)
        oracle().orc3_wilson_apply(C.byref(p), ptr(f64(U)), ptr(e.view(np.float64)), ptr(out.view(np.float64)))
        D[:, k] = out
    return D


def test_chebyshev_overlap_against_dense_polynomial():
    N = (2, 2, 3)
    U = random_links_su3(N, 0.8, 15)
    p = oracle_params(N, m=0.05, mdw=1.0)
    K, eps, lmax = 40, 0.01, 25.0
    D = _dense_wilson(p, U, N)
    h2 = -(D @ D)  # h_W^2, hermitian
    lam, vec = np.linalg.eigh(0.5 * (h2 + h2.conj().T))
    assert lam.max() <= lmax  # ||h_W|| <= |6r + 2m - 2M| / 2 + 3r
    c = np.zeros(K + 1)
    oracle().orc_chebyshev_coeffs(K, eps, ptr(c))
    t = (2 * lam / lmax - 1 - eps) / (1 - eps)
    poly = np.polynomial.chebyshev.chebval(t, np.concatenate([[0.5 * c[0]], c[1:]])) / np.sqrt(lmax)
    dim = D.shape[0]
    phi = np.random.default_rng(16).normal(size=dim) + 1j * np.random.default_rng(17).normal(size=dim)
    chi = vec @ (poly * (vec.conj().T @ phi))
    spin = np.arange(dim) % 4
    g = np.where(spin < 2, -1j, 1j) * (1 + 0.5 * p.m_fermion) * phi
    want = p.m_dw * (g + (1 - 0.5 * p.m_fermion) * (D @ chi))
    out = np.zeros(dim, dtype=np.complex128)
    oracle().orc3_overlap_apply(C.byref(p), ptr(f64(U)), ptr(phi.view(np.float64)), ptr(out.view(np.float64)), K, eps,
                                lmax)
    assert rel_err(out, want) < 1e-12
    # the series approximates (h^2)^(-1/2) where h^2 >= eps lambda_max
    ok = lam >= eps * lmax
    assert np.abs(poly[ok] * np.sqrt(lam[ok]) - 1).max() < 0.05


def test_color_force_is_the_energy_gradient_and_embeds_su2():
    """dH_F/dtheta^a against a central difference of H_F along the link update
    exp(i theta t^a) U of one link, and the SU(2) embedding against
    orc_color_force (itself checked the same way)."""
    N = (3, 4, 3)
    V = volume(N)
    U = f64(random_links_su3(N, 0.7, 30)).copy()
    psi = random_modes3(6, N, 31)
    p = oracle_params(N, m=0.1)
    F = np.zeros((V, 3, 8))
    oracle().orc3_color_force(C.byref(p), ptr(U), ptr(f64(psi)), 6, 0, ptr(F))
    h = 1e-5
    for (s, mu, a) in ((0, 0, 0), (5, 1, 4), (17, 2, 7), (30, 0, 2)):
        vals = []
        for sign in (+1, -1):
            Ut = U.copy()
            E = np.zeros((V, 3, 8))
            E[s, mu, a] = 1.0
            # exp(i cU E t) with cU = -dt_step: dt_step = -sign h moves theta^a by sign h
            oracle().orc3_update_links(C.byref(p), ptr(Ut), ptr(E), -sign * h)
            vals.append(oracle().orc3_fermion_energy(C.byref(p), ptr(Ut), ptr(f64(psi)), 6, 0))
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - F[s, mu, a]) < 1e-7 * max(1.0, np.abs(F).max()), (s, mu, a)
    U2 = random_links(N, 0.6, 32)
    psi2 = random_modes(6, N, 33)
    F2 = np.zeros((V, 3, 3))
    oracle().orc_color_force(C.byref(p), ptr(U2), ptr(f64(psi2)), 6, 1, ptr(F2))
    F3 = np.zeros((V, 3, 8))
    oracle().orc3_color_force(C.byref(p), ptr(f64(embed_su2_links(U2))), ptr(f64(embed_modes(psi2))), 6, 1, ptr(F3))
    assert np.abs(F3[..., :3] - F2).max() < 1e-14 * max(1.0, np.abs(F2).max())
