"""The oracle's fermion back-reaction (orc_color_force, orc_coupled_leapfrog),
an extension without reference counterpart, checked by its defining
properties on the CPU:

* the force is the derivative of H_F = (1/2V) sum_m w_m Re <psi_m, h_W psi_m>
  along the reference's own link update (U <- exp(-i dt E^a t^a) U,
  DYNAMICS/Dynamics.cpp:97-138), by central finite differences;
* the coupled evolution conserves H_gauge + g^2 H_F at second order in dt
  (E at half-integer times, measured as the average of its neighbours);
* with no coupling it is the reference step, E untouched."""
import ctypes as C

import numpy as np

from _helpers import oracle_leapfrog, oracle_params, random_modes
from _oracle import oracle, ptr
from overlap_b200.inputs import random_efield, random_links, volume


def force(p, U, psi, first):
    out = np.zeros((volume(p.N), 3, 3))
    oracle().orc_color_force(C.byref(p), ptr(U), ptr(psi.view(np.float64)), psi.shape[0], first, ptr(out))
    return out


def fermion_energy(p, U, psi, first):
    return oracle().orc_fermion_energy(C.byref(p), ptr(U), ptr(psi.view(np.float64)), psi.shape[0], first)


def test_force_is_the_derivative_of_the_fermion_energy():
    N = (3, 4, 3)
    V = volume(N)
    p = oracle_params(N, m=0.1)
    U = random_links(N, 0.5, 3)
    psi = random_modes(6, N, 4)
    f = force(p, U, psi, 1)
    eps = 1e-5
    for s, mu, a in [(0, 0, 0), (5, 1, 2), (17, 2, 1), (30, 0, 1), (11, 2, 2), (35, 1, 0)]:
        h = []
        for sg in (1, -1):
            Ux = U.copy()
            E = np.zeros((V, 3, 3))
            E[s, mu, a] = 1.0
            oracle().orc_update_links(C.byref(p), ptr(Ux), ptr(E), -sg * eps)  # theta^a = sg eps
            h.append(fermion_energy(p, Ux, psi, 1))
        fd = (h[0] - h[1]) / (2 * eps)
        assert abs(fd - f[s, mu, a]) <= 1e-7 * max(abs(f[s, mu, a]), 1e-3)


def _energy_drift(dt, g2):
    N = (3, 4, 3)
    V = volume(N)
    n = 8
    p = oracle_params(N, m=0.1, dt=dt)
    U = random_links(N, 0.4, 3)
    E = random_efield(N, 0.3, 5)
    psi = random_modes(n, N, 4)
    psi *= np.sqrt(V) / np.sqrt(np.sum(np.abs(psi) ** 2, axis=(1, 2, 3), keepdims=True))
    # psimid at t = dt/2 to first order, so that the modes start consistently
    mid = np.empty_like(psi)
    for i in range(n):
        w = np.zeros_like(psi[i])
        oracle().orc_wilson_apply(C.byref(p), ptr(U), ptr(psi[i].view(np.float64)), ptr(w.view(np.float64)))
        mid[i] = psi[i] + 0.5 * dt * w

    def total(U, E, psi):
        F = np.zeros((V, 3, 3))
        oracle().orc_update_efield(C.byref(p), ptr(U), ptr(F), 1.0)
        F += g2 * force(p, U, psi, 0)
        Ei = np.ascontiguousarray(E - 0.5 * dt * F)  # E at the integer time
        b = np.zeros(10)
        oracle().orc_bulk(C.byref(p), ptr(U), ptr(Ei), ptr(b))
        return b[0] * V + g2 * fermion_energy(p, U, psi, 0)

    h0 = total(U, E, psi)
    t = C.c_int(0)
    oracle().orc_coupled_leapfrog(C.byref(p), ptr(U), ptr(E), ptr(psi.view(np.float64)), ptr(mid.view(np.float64)), n,
                                  0, C.byref(t), int(round(0.5 / dt)), g2, 1)
    return abs(total(U, E, psi) - h0), abs(h0)


def test_coupled_evolution_conserves_total_energy_at_second_order():
    (d1, _), (d2, h) = _energy_drift(0.04, 4.0), _energy_drift(0.02, 4.0)
    assert d2 < 0.35 * d1  # second order: a ratio of 1/4
    assert d2 < 1e-3 * h


def test_uncoupled_evolution_is_the_reference_step():
    N = (4, 3, 4)
    p = oracle_params(N, m=0.2, dt=0.05)
    U = random_links(N, 0.5, 7)
    E = random_efield(N, 0.2, 8)
    psi = random_modes(5, N, 9)
    mid = random_modes(5, N, 10)
    rpsi, rmid, rU, _ = oracle_leapfrog(p, U, E, psi, mid, 3)
    Uc, Ec, pc, mc = U.copy(), E.copy(), psi.copy(), mid.copy()
    t = C.c_int(0)
    oracle().orc_coupled_leapfrog(C.byref(p), ptr(Uc), ptr(Ec), ptr(pc.view(np.float64)), ptr(mc.view(np.float64)), 5,
                                  0, C.byref(t), 3, 0.0, 0)
    assert np.array_equal(pc, rpsi) and np.array_equal(mc, rmid) and np.array_equal(Uc, rU)
    assert np.array_equal(Ec, E)
