"""Shared test utilities: seeded mode sets, oracle runs, error norms."""
from __future__ import annotations

import ctypes as C

import numpy as np

from _oracle import oracle, orc_params, ptr
from overlap_b200.inputs import volume


def random_modes(n_modes: int, N, seed: int) -> np.ndarray:
    """complex128[n_modes, V, 2, 4], entries ~ N(0, 1/2) + i N(0, 1/2)."""
    rng = np.random.default_rng(seed)
    shape = (n_modes, volume(N), 2, 4)
    return (rng.normal(0, np.sqrt(0.5), shape) + 1j * rng.normal(0, np.sqrt(0.5), shape)).astype(np.complex128)


def oracle_params(N, m=0.1, r=1.0, mdw=0.0, dt=0.05, qs=1.0, t_sph=1e300):
    return orc_params(tuple(int(n) for n in N), r=r, m=m, mdw=mdw, dt=dt, qs=qs, t_sph=t_sph)


def oracle_leapfrog(p, U, E, psi, psimid, steps, tsteps=0):
    """Runs the oracle on copies; returns (psi, psimid, links, tsteps)."""
    U = np.ascontiguousarray(U.copy())
    psi = np.ascontiguousarray(psi.copy())
    mid = np.ascontiguousarray(psimid.copy())
    t = C.c_int(tsteps)
    oracle().orc_wilson_leapfrog(C.byref(p), ptr(U), ptr(np.ascontiguousarray(E)), ptr(psi.view(np.float64)),
                                 ptr(mid.view(np.float64)), psi.shape[0], C.byref(t), steps)
    return psi, mid, U, t.value


def oracle_currents(p, U, psi, first):
    V = psi.shape[1]
    out = [np.zeros(4 * V) for _ in range(4)] + [np.zeros(V), np.zeros(V)]
    oracle().orc_wilson_currents(C.byref(p), ptr(U), ptr(np.ascontiguousarray(psi).view(np.float64)), psi.shape[0],
                                 first, *[ptr(a) for a in out])
    names = ("jV", "jA", "jVw", "jAw", "PS", "WA")
    return {k: (a.reshape(V, 4) if a.size == 4 * V else a) for k, a in zip(names, out)}


def rel_err(a, b) -> float:
    """max |a - b| / max |b| (b the reference value)."""
    a = np.asarray(a)
    b = np.asarray(b)
    scale = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (scale if scale > 0 else 1.0))


def current_scale(psi: np.ndarray) -> float:
    """Size of one mode's contribution to a current density: the bound used to
    normalise current errors, since the vacuum-weighted mode sum cancels."""
    V = psi.shape[1]
    return float(psi.shape[0] * np.max(np.sum(np.abs(psi) ** 2, axis=(2, 3))) / (2.0 * V))
