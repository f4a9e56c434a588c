"""Pins the CPU oracle (oracle/ovl_oracle.c) to the reference's own code.

Always: against the golden vectors in tests/golden, which the reference
compiled from source produced (tests/golden/make_golden.py).
Where oracle/_ref was built: against the live reference on fresh seeded inputs.
"""
import ctypes as C

import numpy as np
import pytest

from _helpers import current_scale, oracle_currents, oracle_leapfrog, oracle_params, random_modes, rel_err
from _oracle import have_reference, oracle, ptr, reference
from overlap_b200.inputs import random_efield, random_links, volume

CASES = ["wilson_n4", "wilson_n465"]


def load(golden_dir, name):
    g = dict(np.load(golden_dir / f"{name}.npz"))
    g["N"] = tuple(int(n) for n in g["N"])
    return g


def params_of(g):
    return oracle_params(g["N"], m=float(g["m_fermion"]), r=float(g["r_wilson"]), mdw=float(g["m_dw"]),
                         dt=float(g["dt"]), t_sph=float(g["t_sphaleron"]))


@pytest.mark.parametrize("name", CASES)
def test_free_fermions_match_golden(golden_dir, name):
    g = load(golden_dir, name)
    p = params_of(g)
    psi = np.zeros_like(g["psi0"])
    mid = np.zeros_like(g["psi0"])
    bad = oracle().orc_free_fermions(C.byref(p), int(g["first_mode"]), psi.shape[0], ptr(psi.view(np.float64)),
                                     ptr(mid.view(np.float64)))
    assert bad == 0
    assert np.max(np.abs(psi - g["psi0"])) < 1e-13
    assert np.max(np.abs(mid - g["psimid0"])) < 1e-13


@pytest.mark.parametrize("name", CASES)
def test_leapfrog_matches_golden(golden_dir, name):
    g = load(golden_dir, name)
    psi, mid, U, t = oracle_leapfrog(params_of(g), g["links"], g["efield"], g["psi0"], g["psimid0"], int(g["steps"]))
    assert t == int(g["steps"])
    assert rel_err(psi, g["psi"]) < 1e-12
    assert rel_err(mid, g["psimid"]) < 1e-12
    assert rel_err(U, g["links_after"]) < 1e-13


@pytest.mark.parametrize("name", CASES)
def test_currents_match_golden(golden_dir, name):
    g = load(golden_dir, name)
    p = params_of(g)
    cur = oracle_currents(p, g["links_after"], g["psi"], int(g["first_mode"]))
    scale = current_scale(g["psi"])
    for k in ("jV", "jA", "jVw", "jAw", "PS", "WA"):
        ref = g[k].reshape(cur[k].shape)
        assert np.max(np.abs(cur[k] - ref)) <= 1e-12 * scale, k


@pytest.mark.parametrize("name", CASES)
def test_gauge_observables_match_golden(golden_dir, name):
    g = load(golden_dir, name)
    p = params_of(g)
    ncs = oracle().orc_ncsdot(C.byref(p), ptr(g["links"]), ptr(g["efield"]))
    assert abs(ncs - float(g["ncsdot0"])) <= 1e-13 * max(1.0, abs(float(g["ncsdot0"])))
    bulk = np.zeros(10)
    oracle().orc_bulk(C.byref(p), ptr(g["links"]), ptr(g["efield"]), ptr(bulk))
    assert np.allclose(bulk, g["bulk0"], rtol=1e-12, atol=1e-14)
    E = g["efield"].copy()
    oracle().orc_update_efield(C.byref(p), ptr(g["links_after"]), ptr(E), float(g["dt"]))
    assert rel_err(E, g["efield_after_update"]) < 1e-13


def test_u1_flux_formula():
    """QED::SetConstantMagneticField (QED.cpp:62-84): every plaquette carries the
    same flux, and the total winds n_B times around the (x, y) torus."""
    N = (6, 5, 4)
    p = oracle_params(N)
    out = np.zeros(2 * N[0] * N[1] * 2)
    oracle().orc_u1_flux(C.byref(p), 3, ptr(out))
    u = out.view(np.complex128).reshape(N[1], N[0], 2)  # [y][x][mu]
    ph = []
    for y in range(N[1]):
        for x in range(N[0]):
            box = u[y, x, 0] * u[y, (x + 1) % N[0], 1] * np.conj(u[(y + 1) % N[1], x, 0]) * np.conj(u[y, x, 1])
            ph.append(np.angle(box))
    ph = np.array(ph)
    assert np.allclose(ph, ph[0], atol=1e-12)
    assert abs(ph.sum() / (2 * np.pi) + 3) < 1e-9 or abs(ph.sum() / (2 * np.pi) - 3) < 1e-9


needs_ref = pytest.mark.skipif(not have_reference("wilson"), reason="reference not built here (oracle/_ref)")


@needs_ref
def test_live_reference_random_modes_and_links():
    """Random (non-eigen) modes, moving links, odd first mode: oracle == reference."""
    R = reference("wilson")
    N = (4, 4, 4)
    V = volume(N)
    m = R.ovlref_init(*N, 8, 5, 0.2, 1.0, 0.3, 0.1, 0.04, 1.0, 1)
    first = R.ovlref_first_mode()
    U = random_links(N, 0.7, 5)
    E = random_efield(N, 0.3, 6)
    psi = random_modes(m, N, 7)
    mid = random_modes(m, N, 8)
    R.ovlref_set_links(ptr(U))
    R.ovlref_set_efield(ptr(E))
    R.ovlref_set_modes(ptr(psi.view(np.float64)), ptr(mid.view(np.float64)))
    R.ovlref_step(5)
    rpsi = np.zeros_like(psi)
    rmid = np.zeros_like(psi)
    R.ovlref_get_modes(ptr(rpsi.view(np.float64)), ptr(rmid.view(np.float64)))
    p = oracle_params(N, m=0.2, r=1.0, mdw=0.3, dt=0.04, t_sph=0.1)
    opsi, omid, oU, _ = oracle_leapfrog(p, U, E, psi, mid, 5)
    assert rel_err(opsi, rpsi) < 1e-12
    assert rel_err(omid, rmid) < 1e-12
    rU = np.zeros_like(U)
    R.ovlref_get_links(ptr(rU))
    assert rel_err(oU, rU) < 1e-13
    cur = [np.zeros(4 * V) for _ in range(4)] + [np.zeros(V), np.zeros(V)]
    R.ovlref_currents(*[ptr(a) for a in cur])
    ocur = oracle_currents(p, oU, opsi, first)
    scale = current_scale(opsi)
    for k, ref in zip(("jV", "jA", "jVw", "jAw", "PS", "WA"), cur):
        assert np.max(np.abs(ocur[k].ravel() - ref)) <= 1e-12 * scale, k


@needs_ref
def test_live_reference_wilson_operator():
    R = reference("wilson")
    N = (5, 4, 6)
    R.ovlref_init(*N, 240, 0, 0.1, 1.0, 0.0, 0.0, 0.05, 1.0, 1)
    U = random_links(N, 1.0, 21)
    R.ovlref_set_links(ptr(U))
    phi = random_modes(1, N, 22)[0]
    out_r = np.zeros_like(phi)
    R.ovlref_apply(ptr(phi.view(np.float64)), ptr(out_r.view(np.float64)), 0.0, 0.0)
    out_o = np.zeros_like(phi)
    oracle().orc_wilson_apply(C.byref(oracle_params(N, m=0.1)), ptr(U), ptr(phi.view(np.float64)),
                              ptr(out_o.view(np.float64)))
    assert rel_err(out_o, out_r) < 1e-14


def test_gauge_leapfrog_preserves_gauss_law_and_energy():
    """Coupled E/U leapfrog with the restated staple force: Gauss's law holds to
    round-off and the energy error is bounded and shrinks with dt."""
    N = (4, 4, 4)
    spreads = []
    for dt in (0.04, 0.02):
        p = oracle_params(N, dt=dt)
        U = random_links(N, 0.8, 3)
        E = np.zeros((volume(N), 3, 3))
        b = np.zeros(10)
        oracle().orc_bulk(C.byref(p), ptr(U), ptr(E), ptr(b))
        e0 = b[0]
        energies = []
        for _ in range(int(round(1.0 / dt))):
            oracle().orc_update_efield(C.byref(p), ptr(U), ptr(E), dt)
            oracle().orc_update_links(C.byref(p), ptr(U), ptr(E), dt)
            oracle().orc_bulk(C.byref(p), ptr(U), ptr(E), ptr(b))
            energies.append(b[0])
            assert b[7] < 1e-13  # Gauss-law violation (rms)
        spreads.append(max(abs(e - e0) for e in energies) / e0)
    assert spreads[0] < 0.1
    assert spreads[1] < 0.6 * spreads[0]


@pytest.mark.parametrize("name", ["ritz_n4", "ritz_n465"])
def test_ritz_matches_golden(golden_dir, name):
    """RitzSolver (RitzSolver.cpp:91-292) restated: the smallest and largest
    eigenvalues of h_W^2 from the reference's start vector agree with the
    reference's to 1e-12 (the iteration stops at round-off, so the last few
    iterates may differ)."""
    g = dict(np.load(golden_dir / f"{name}.npz"))
    N = tuple(int(n) for n in g["N"])
    p = oracle_params(N, m=float(g["m_fermion"]), r=float(g["r_wilson"]), mdw=float(g["m_dw"]))
    it = C.c_int(0)
    lo = oracle().orc_ritz(C.byref(p), ptr(g["links"]), ptr(g["start"].view(np.float64)), 1.0, 2000, 100, 1e-16,
                           C.byref(it))
    assert 10 < it.value < 2000
    hi = -oracle().orc_ritz(C.byref(p), ptr(g["links"]), ptr(g["start"].view(np.float64)), -1.0, 2000, 100, 1e-16,
                            C.byref(it))
    assert abs(lo - float(g["lambda_min"])) <= 1e-12 * abs(float(g["lambda_min"]))
    assert abs(hi - float(g["lambda_max"])) <= 1e-12 * abs(float(g["lambda_max"]))


def test_gauss_restore_matches_golden(golden_dir):
    """GaussLawRestoration::Restore (GaussRestore.cpp:132-168) restated: the
    restored E equals the reference's (whose Gauss-violation macro is itself a
    restatement, see oracle/ref/ovl_calc_macros.h) and the violation ends
    below 1e-14."""
    g = dict(np.load(golden_dir / "gauss_n465.npz"))
    N = tuple(int(n) for n in g["N"])
    p = oracle_params(N)
    E = g["efield"].copy()
    out = np.zeros(2)
    n = oracle().orc_gauss_restore(C.byref(p), ptr(g["links"]), ptr(E), 10000, 1e-14, ptr(out))
    assert 5 < n < 10000
    assert out[0] <= 1e-14
    assert rel_err(E, g["efield_restored"]) < 1e-12


def test_u1_flux_input_matches_oracle():
    """inputs.u1_flux (the package's restatement of QED.cpp:62-84 for bench
    inputs) equals the oracle's phases."""
    from overlap_b200.inputs import u1_flux
    for N, nb in (((4, 6, 5), 3), ((8, 8, 8), 4)):
        p = oracle_params(N)
        out = np.zeros(4 * N[0] * N[1])
        oracle().orc_u1_flux(C.byref(p), nb, ptr(out))
        ref = out.view(np.complex128).reshape(N[1], N[0], 2)
        assert np.max(np.abs(u1_flux(N, nb) - ref)) < 1e-15


@pytest.mark.skipif(not have_reference("overlap"), reason="reference overlap build absent")
@pytest.mark.parametrize("mdw,N", [(1.4, (4, 4, 4)), (1.0, (4, 5, 6))])
def test_overlap_plane_waves_match_reference(mdw, N):
    """SetFreeFermions in the overlap build (GetOverlapDiracSpinor,
    FermionField.cpp:331-517) against the oracle's overlap spinors, for the
    slice of one emulated MPI rank."""
    R = reference("overlap")
    m = R.ovlref_init(*N, 4, 1, 0.05, 1.0, mdw, 1e9, 0.05, 1.0, 1)
    first = R.ovlref_first_mode()
    R.ovlref_set_free_fermions()
    V = volume(N)
    rpsi = np.zeros((m, V, 2, 4), np.complex128)
    rmid = np.zeros_like(rpsi)
    R.ovlref_get_modes(ptr(rpsi.view(np.float64)), ptr(rmid.view(np.float64)))
    p = oracle_params(N, m=0.05, mdw=mdw, dt=0.05)
    psi = np.zeros_like(rpsi)
    mid = np.zeros_like(rpsi)
    oracle().orc_set_free_kind(1)
    try:
        bad = oracle().orc_free_fermions(C.byref(p), first, m, ptr(psi.view(np.float64)), ptr(mid.view(np.float64)))
    finally:
        oracle().orc_set_free_kind(0)
    # odd N: the momentum index (N-1)/2 takes the reference's axis branch
    # (k == N/2 in integer division), whose spinors fail its own eigen check
    assert (bad == 0) == all(n % 2 == 0 for n in N)
    assert rel_err(psi, rpsi) < 1e-14 and rel_err(mid, rmid) < 1e-14
