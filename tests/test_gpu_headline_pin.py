"""The benchmark's headline workload pinned to the CPU checkers.

Workload: SU(2), N = 16^3, Wilson r = 1, m = 0.05, MDWHeight = 0, dt = 0.05,
quasi-particle links and E (occupancy 1/g^2 = 4 below Qs = 1, Gauss's law
restored), a U(1) background of n_B = 4 flux quanta in the hopping term, links
moving every half step.  A 64-mode slice of the plane-wave basis (global modes
4096-4159, the slice one MPI rank of 512 holds, MPI/ModePartition.cpp:12-24) is
advanced 200 leapfrog steps by

  * the oracle (the plain-C restatement, with the same U(1) phases) against the
    FP64 fused and plain forms and the FP32 form with hop variant 3, the
    packed-pair kernel the benchmark's headline runs
    (wilson_packed_kernel<1,true,false>);
  * the reference's own code (FERMIONS/WILSON/Update.cpp:48-79, compiled from
    source) with n_B = 0 -- its hopping term has no U(1) phase -- against the
    same GPU forms without the background.

Tolerances: FP64 fields and links 1e-12 of their largest element; FP32 fields
2e-5 of the largest element (storage and hop arithmetic in FP32, links FP64,
200 steps); the slice's charges 1e-12 (FP64) and 1e-6 (FP32) of the sum of the
modes' contributions to a charge."""
from __future__ import annotations

import ctypes as C
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from _helpers import oracle_currents, oracle_params, rel_err
from _oracle import have_reference, oracle, ptr, reference
from overlap_b200 import Context
from overlap_b200.inputs import quasi_particles, u1_flux, volume

pytestmark = pytest.mark.gpu

N = (16, 16, 16)
V = volume(N)
FIRST, NM, STEPS = 4096, 64, 200
M_F, DT = 0.05, 0.05
THREADS = 4  # the oracle's slice split over host threads (it keeps no shared scratch)

TOL = {"fp64": 1e-12, "fp32": 2e-5}
CHARGE_TOL = {"fp64": 1e-12, "fp32": 1e-6}


def oracle_run(p, U, E, psi, mid, steps):
    """orc_wilson_leapfrog on `psi`, `mid` (copies), modes split over THREADS
    threads, each with its own copy of the links (they move identically)."""
    psi = np.ascontiguousarray(psi.copy())
    mid = np.ascontiguousarray(mid.copy())
    parts = np.array_split(np.arange(psi.shape[0]), THREADS)
    links = [np.ascontiguousarray(U.copy()) for _ in parts]

    def run(k):
        a, b = parts[k][0], parts[k][-1] + 1
        pa, pb = np.ascontiguousarray(psi[a:b]), np.ascontiguousarray(mid[a:b])
        t = C.c_int(0)
        oracle().orc_wilson_leapfrog(C.byref(p), ptr(links[k]), ptr(np.ascontiguousarray(E)), ptr(pa.view(np.float64)),
                                     ptr(pb.view(np.float64)), b - a, C.byref(t), steps)
        psi[a:b], mid[a:b] = pa, pb

    with ThreadPoolExecutor(THREADS) as ex:
        list(ex.map(run, range(len(parts))))
    return psi, mid, links[0]


def reference_run(U, E, steps):
    """The reference's own leapfrog on rank 64 of 512 (global modes 4096-4159)."""
    R = reference("wilson")
    nm = R.ovlref_init(*N, 512, FIRST // NM, M_F, 1.0, 0.0, 1e300, DT, 1.0, 1)
    assert nm == NM and R.ovlref_first_mode() == FIRST
    R.ovlref_set_links(ptr(np.ascontiguousarray(U)))
    R.ovlref_set_efield(ptr(np.ascontiguousarray(E)))
    R.ovlref_set_free_fermions()
    R.ovlref_step(steps)
    psi = np.zeros((NM, V, 2, 4), np.complex128)
    mid = np.zeros_like(psi)
    R.ovlref_get_modes(ptr(psi.view(np.float64)), ptr(mid.view(np.float64)))
    Uo = np.zeros((V, 3, 4))
    R.ovlref_get_links(ptr(Uo))
    return psi, mid, Uo


@pytest.fixture(scope="module")
def pinned():
    # the workload's gauge fields: quasi-particles, Gauss's law restored on the
    # device as the benchmark does, then handed to every side unchanged
    U0, E0 = quasi_particles(N, 4.0, 1.0, 20261203)
    with Context(N=N, n_modes=32, precision="fp64", form="fused", m_fermion=M_F, m_dw=0.0, dt=DT) as ctx:
        ctx.set_links(U0)
        ctx.set_efield(E0)
        ctx.gauss_restore()
        U, E = ctx.get_links(), ctx.get_efield()
    u1 = u1_flux(N, 4)
    p = oracle_params(N, m=M_F, mdw=0.0, dt=DT)
    psi0 = np.zeros((NM, V, 2, 4), np.complex128)
    mid0 = np.zeros_like(psi0)
    assert oracle().orc_free_fermions(C.byref(p), FIRST, NM, ptr(psi0.view(np.float64)),
                                      ptr(mid0.view(np.float64))) == 0
    u1f = np.ascontiguousarray(u1).view(np.float64).ravel()
    oracle().orc_set_u1(ptr(u1f))
    try:
        with ThreadPoolExecutor(2) as ex:
            ref = ex.submit(reference_run, U, E, STEPS) if have_reference("wilson") else None
            opsi, omid, oU = oracle_run(p, U, E, psi0, mid0, STEPS)
            ocur = oracle_currents(p, oU, opsi, FIRST)
            ref = ref.result() if ref is not None else None
    finally:
        oracle().orc_set_u1(None)
    scale = 1.0 / (2.0 * V) * float(np.max(np.sum(np.abs(opsi) ** 2, axis=(1, 2, 3))))
    return dict(U=U, E=E, u1=u1, psi0=psi0, mid0=mid0, opsi=opsi, omid=omid, oU=oU, ocur=ocur, ref=ref, scale=scale)


def gpu_run(d, precision, form, variant, with_u1):
    with Context(N=N, n_modes=NM, first_mode=FIRST, precision=precision, form=form, m_fermion=M_F, m_dw=0.0, dt=DT,
                 t_sphaleron=1e300, hop_variant=variant) as ctx:
        ctx.set_links(d["U"])
        ctx.set_efield(d["E"])
        if with_u1:
            ctx.set_u1(d["u1"])
        assert ctx.set_free_fermions() == 0
        a, b = ctx.get_modes()
        tol0 = 1e-14 if precision == "fp64" else 1e-7
        assert rel_err(a, d["psi0"]) < tol0 and rel_err(b, d["mid0"]) < tol0  # the same plane waves
        ctx.step(STEPS)
        assert ctx.tuning()[0] == variant or variant < 0
        psi, mid = ctx.get_modes()
        return psi, mid, ctx.get_links(), ctx.charges()


@pytest.mark.parametrize("precision,form,variant", [("fp64", "fused", -1), ("fp64", "plain", -1), ("fp32", "fused", 3)])
def test_headline_slice_with_u1_matches_the_oracle(pinned, precision, form, variant):
    d = pinned
    psi, mid, U, ch = gpu_run(d, precision, form, variant, with_u1=True)
    e_psi, e_mid = rel_err(psi, d["opsi"]), rel_err(mid, d["omid"])
    assert e_psi < TOL[precision] and e_mid < TOL[precision], (e_psi, e_mid)
    assert rel_err(U, d["oU"]) < 1e-12
    # the slice's charges: sum_x jV^0, N_5 = sum_x jA^0, sum_x PS
    want = {"NV": d["ocur"]["jV"][:, 0].sum(), "N5": d["ocur"]["jA"][:, 0].sum(), "PS": d["ocur"]["PS"].sum()}
    for k, w in want.items():
        assert abs(ch[k] - w) <= CHARGE_TOL[precision] * NM * d["scale"], (k, ch[k], w)


@pytest.mark.skipif(not have_reference("wilson"), reason="reference library not built")
@pytest.mark.parametrize("precision,form,variant", [("fp64", "fused", -1), ("fp64", "plain", -1), ("fp32", "fused", 3)])
def test_headline_slice_without_u1_matches_the_reference(pinned, precision, form, variant):
    d = pinned
    rpsi, rmid, rU = d["ref"]
    psi, mid, U, _ = gpu_run(d, precision, form, variant, with_u1=False)
    e_psi, e_mid = rel_err(psi, rpsi), rel_err(mid, rmid)
    assert e_psi < TOL[precision] and e_mid < TOL[precision], (e_psi, e_mid)
    assert rel_err(U, rU) < 1e-12
