"""Generates tests/golden/*.npz from the reference's own code.

Runs the reference hot path compiled from source (oracle/_ref/libovlref_*.so,
built by `make -C oracle ref` where the reference tree is available) on small
seeded inputs and stores inputs and outputs.  The fixtures pin the oracle
restatement (tests/test_oracle_pin.py) and the GPU path (tests/test_gpu_*.py)
on machines without the reference.

    python tests/golden/make_golden.py [case names]
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE.parents[1]))

from _oracle import ptr, reference  # noqa: E402
from overlap_b200.inputs import random_efield, random_links, volume  # noqa: E402

# name: lattice, MPI emulation (nranks, rank), physics, steps, seeds
CASES = {
    "wilson_n4": dict(N=(4, 4, 4), nranks=16, rank=3, m=0.1, r=1.0, mdw=0.0, dt=0.05, steps=4,
                      link_sigma=0.3, e_sigma=0.1, seed=11, t_sph=1e300),
    "wilson_n465": dict(N=(4, 6, 5), nranks=30, rank=5, m=0.05, r=1.0, mdw=0.0, dt=0.05, steps=3,
                        link_sigma=0.5, e_sigma=0.2, seed=12, t_sph=0.08),
}


def run_case(name: str, c: dict) -> dict:
    R = reference("wilson")
    N = c["N"]
    V = volume(N)
    m = R.ovlref_init(*N, c["nranks"], c["rank"], c["m"], c["r"], c["mdw"], c["t_sph"], c["dt"], 1.0, 1)
    assert m > 0
    U = random_links(N, c["link_sigma"], c["seed"])
    E = random_efield(N, c["e_sigma"], c["seed"] + 1000)
    R.ovlref_set_links(ptr(U))
    R.ovlref_set_efield(ptr(E))
    R.ovlref_set_free_fermions()
    psi0 = np.zeros((m, V, 2, 4), np.complex128)
    mid0 = np.zeros_like(psi0)
    R.ovlref_get_modes(ptr(psi0.view(np.float64)), ptr(mid0.view(np.float64)))
    ncs0 = R.ovlref_ncsdot()
    bulk0 = np.zeros(10)
    R.ovlref_bulk(ptr(bulk0))
    R.ovlref_step(c["steps"])
    psi = np.zeros_like(psi0)
    mid = np.zeros_like(psi0)
    R.ovlref_get_modes(ptr(psi.view(np.float64)), ptr(mid.view(np.float64)))
    U1 = np.zeros_like(U)
    R.ovlref_get_links(ptr(U1))
    cur = [np.zeros(4 * V) for _ in range(4)] + [np.zeros(V), np.zeros(V)]
    assert R.ovlref_currents(*[ptr(a) for a in cur]) == 6
    E1 = E.copy()
    R.ovlref_update_efield(c["dt"])
    R.ovlref_get_efield(ptr(E1))
    first = R.ovlref_first_mode()
    return dict(N=np.array(N), first_mode=first, n_modes=m, m_fermion=c["m"], r_wilson=c["r"], m_dw=c["mdw"],
                dt=c["dt"], steps=c["steps"], t_sphaleron=c["t_sph"], links=U, efield=E, psi0=psi0, psimid0=mid0,
                ncsdot0=ncs0, bulk0=bulk0, psi=psi, psimid=mid, links_after=U1, jV=cur[0], jA=cur[1], jVw=cur[2],
                jAw=cur[3], PS=cur[4], WA=cur[5], efield_after_update=E1)


# Ritz extreme eigenvalues of h_W^2 (FERMIONS/OVERLAP/OPERATOR/RitzSolver.cpp) from a
# seeded start vector with the reference's distribution (Re, Im uniform in [0, 1),
# OverlapUpdate.cpp:69-84).
RITZ_CASES = {
    "ritz_n4": dict(N=(4, 4, 4), m=0.1, r=1.0, mdw=1.4, link_sigma=0.5, seed=21),
    "ritz_n465": dict(N=(4, 6, 5), m=0.0, r=1.0, mdw=1.2, link_sigma=0.4, seed=22),
}


def run_ritz_case(name: str, c: dict) -> dict:
    R = reference("overlap")
    N = c["N"]
    V = volume(N)
    R.ovlref_init(*N, 16, 0, c["m"], c["r"], c["mdw"], 6.0, 0.05, 1.0, 1)
    U = random_links(N, c["link_sigma"], c["seed"])
    R.ovlref_set_links(ptr(U))
    rng = np.random.default_rng(c["seed"] + 1000)
    start = rng.uniform(0.0, 1.0, (V, 2, 4)) + 1j * rng.uniform(0.0, 1.0, (V, 2, 4))
    start = np.ascontiguousarray(start / np.linalg.norm(start))
    lam_min = R.ovlref_ritz_solve(ptr(start.view(np.float64)), 1.0)
    lam_max = -R.ovlref_ritz_solve(ptr(start.view(np.float64)), -1.0)
    return dict(N=np.array(N), m_fermion=c["m"], r_wilson=c["r"], m_dw=c["mdw"], links=U, start=start,
                lambda_min=lam_min, lambda_max=lam_max)


# Gauss-law restoration (GAUSSLAWFIXING/GaussRestore.cpp:132-168) of a random E
# on random links.
GAUSS_CASES = {"gauss_n465": dict(N=(4, 6, 5), link_sigma=0.5, e_sigma=0.3, seed=31)}


def run_gauss_case(name: str, c: dict) -> dict:
    R = reference("wilson")
    N = c["N"]
    R.ovlref_init(*N, 1, 0, 0.1, 1.0, 0.0, 6.0, 0.05, 1.0, 1)
    U = random_links(N, c["link_sigma"], c["seed"])
    E = random_efield(N, c["e_sigma"], c["seed"] + 1)
    R.ovlref_set_links(ptr(U))
    R.ovlref_set_efield(ptr(E))
    out = np.zeros(2)
    R.ovlref_gauss_restore(ptr(out))
    E1 = np.zeros_like(E)
    R.ovlref_get_efield(ptr(E1))
    return dict(N=np.array(N), links=U, efield=E, efield_restored=E1, max_violation=out[0], avg_violation=out[1])


# Gradient-flow cooling and the Chern-Simons calibration (GRADIENTFLOW/Cooling.cpp,
# TOPOLOGY/CoolingMethod.cpp) with blocking in both phases: block_frequency 2 blocks
# the standard phase at step 2 and the calibration phase at step 16.
COOL_CASES = {"cooling_n8": dict(N=(8, 8, 8), link_sigma=0.6, seed=41, standard_steps=3, standard_blocking=1,
                                 calibration_steps=20, calibration_blocking=2, block_frequency=2)}


def run_cool_case(name: str, c: dict) -> dict:
    import ctypes as C

    R = reference("wilson")
    N = c["N"]
    R.ovlref_init(*N, 1, 0, 0.1, 1.0, 0.0, 6.0, 0.05, 1.0, 1)
    U = random_links(N, c["link_sigma"], c["seed"])
    R.ovlref_set_links(ptr(U))
    log = np.zeros((c["calibration_steps"] + 1, 5))
    rows, out, cooled, cn = C.c_int(0), np.zeros(3), np.zeros_like(U), (C.c_int * 3)()
    R.ovlref_cool(c["standard_steps"], c["standard_blocking"], c["calibration_steps"], c["calibration_blocking"],
                  c["block_frequency"], ptr(log), C.byref(rows), ptr(out), ptr(cooled), cn)
    Nc = tuple(cn)
    return dict(N=np.array(N), links=U, schedule=np.array([c[k] for k in ("standard_steps", "standard_blocking",
                                                                           "calibration_steps", "calibration_blocking",
                                                                           "block_frequency")]),
                log=log[:rows.value], out=out, cooled_N=np.array(Nc),
                cooled=cooled.reshape(-1)[:4 * 3 * Nc[0] * Nc[1] * Nc[2]].reshape(-1, 3, 4))


RUNNERS = [(CASES, run_case), (RITZ_CASES, run_ritz_case), (GAUSS_CASES, run_gauss_case), (COOL_CASES, run_cool_case)]

if __name__ == "__main__":
    only = set(sys.argv[1:])  # case names to (re)generate; all when none are given
    for cases, run in RUNNERS:
        for name, c in cases.items():
            if only and name not in only:
                continue
            out = HERE / f"{name}.npz"
            np.savez_compressed(out, **run(name, c))
            print(out, out.stat().st_size, "bytes")
