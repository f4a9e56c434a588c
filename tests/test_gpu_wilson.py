"""GPU parity of the fermion leapfrog, plane-wave init and currents.

Every test drives the CUDA library through the C ABI (overlap_b200.Context) and
compares with the oracle, the golden vectors the reference produced, or the
reference compiled from source.  Tolerances: FP64 forms 1e-12 relative (the
bar stated for the plain form); FP32 modes 2e-5 relative per step count used
here.  Current densities are compared after normalising by the size of one
mode's contribution (the vacuum-weighted mode sum cancels)."""
import numpy as np
import pytest

from _helpers import current_scale, oracle_currents, oracle_leapfrog, oracle_params, random_modes, rel_err
from _oracle import have_reference, oracle, ptr, reference
from overlap_b200 import Context, OvlError
from overlap_b200.inputs import random_efield, random_links, unit_links, volume

pytestmark = pytest.mark.gpu

CASES = ["wilson_n4", "wilson_n465"]
FORMS = [("fp64", "plain"), ("fp64", "fused"), ("fp32", "fused"), ("fp32", "plain")]


def load(golden_dir, name):
    g = dict(np.load(golden_dir / f"{name}.npz"))
    g["N"] = tuple(int(n) for n in g["N"])
    return g


def ctx_for(g, precision, form, **kw):
    return Context(N=g["N"], n_modes=int(g["n_modes"]), first_mode=int(g["first_mode"]), precision=precision,
                   form=form, r_wilson=float(g["r_wilson"]), m_fermion=float(g["m_fermion"]), m_dw=float(g["m_dw"]),
                   dt=float(g["dt"]), qs=1.0, t_sphaleron=float(g["t_sphaleron"]), **kw)


def tol(precision):
    return 1e-12 if precision == "fp64" else 2e-5


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("precision,form", FORMS)
def test_leapfrog_matches_reference_golden(golden_dir, name, precision, form):
    g = load(golden_dir, name)
    with ctx_for(g, precision, form) as ctx:
        ctx.set_links(g["links"])
        ctx.set_efield(g["efield"])
        ctx.set_modes(g["psi0"], g["psimid0"])
        ctx.step(int(g["steps"]))
        assert ctx.step_count == int(g["steps"])
        psi, mid = ctx.get_modes()
        assert rel_err(psi, g["psi"]) < tol(precision)
        assert rel_err(mid, g["psimid"]) < tol(precision)
        assert rel_err(ctx.get_links(), g["links_after"]) < 1e-13
        cur = ctx.currents()
        scale = current_scale(g["psi"])
        ctol = 1e-12 if precision == "fp64" else 1e-5
        for k in ("jV", "jA", "jVw", "jAw", "PS", "WA"):
            assert np.max(np.abs(cur[k].ravel() - g[k])) <= ctol * scale, k


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_free_fermions_match_reference_golden(golden_dir, name, precision):
    g = load(golden_dir, name)
    with ctx_for(g, precision, "fused") as ctx:
        assert ctx.set_free_fermions() == 0
        psi, mid = ctx.get_modes()
        t = 1e-13 if precision == "fp64" else 1e-6
        assert np.max(np.abs(psi - g["psi0"])) < t
        assert np.max(np.abs(mid - g["psimid0"])) < t


@pytest.mark.parametrize("precision,form", FORMS)
def test_ragged_modes_odd_offset_asymmetric_lattice(precision, form):
    """45 modes (one partial mode block), odd first mode, N = (5, 4, 6), random
    modes and links, links frozen after the second step."""
    N = (5, 4, 6)
    n, first = 45, 7
    U = random_links(N, 0.9, 31)
    E = random_efield(N, 0.4, 32)
    psi0 = random_modes(n, N, 33)
    mid0 = random_modes(n, N, 34)
    p = oracle_params(N, m=0.07, r=1.0, mdw=0.2, dt=0.03, t_sph=0.05)
    opsi, omid, oU, _ = oracle_leapfrog(p, U, E, psi0, mid0, 6)
    with Context(N=N, n_modes=n, first_mode=first, precision=precision, form=form, m_fermion=0.07, r_wilson=1.0,
                 m_dw=0.2, dt=0.03, t_sphaleron=0.05, plain_chunk_modes=40) as ctx:
        ctx.set_links(U)
        ctx.set_efield(E)
        ctx.set_modes(psi0, mid0)
        ctx.step(6)
        psi, mid = ctx.get_modes()
        assert rel_err(psi, opsi) < tol(precision)
        assert rel_err(mid, omid) < tol(precision)
        assert rel_err(ctx.get_links(), oU) < 1e-13
        ocur = oracle_currents(p, oU, opsi, first)
        cur = ctx.currents()
        scale = current_scale(opsi)
        for k in ocur:
            assert np.max(np.abs(cur[k] - ocur[k])) <= (1e-12 if precision == "fp64" else 1e-5) * scale, k
        # lattice sums straight from the modes (the WA sum uses forward hops only)
        ch = ctx.charges()
        qtol = (1e-12 if precision == "fp64" else 1e-6) * scale * volume(N)
        assert abs(ch["N5"] - ocur["jA"][:, 0].sum()) <= qtol
        assert abs(ch["NV"] - ocur["jV"][:, 0].sum()) <= qtol
        assert abs(ch["PS"] - ocur["PS"].sum()) <= qtol
        assert abs(ch["WA"] - ocur["WA"].sum()) <= qtol


def test_partial_mode_transfers_roundtrip():
    N = (4, 4, 4)
    with Context(N=N, n_modes=70, precision="fp32", form="fused") as ctx:
        a = random_modes(70, N, 41)
        ctx.set_modes(a, a)
        b = random_modes(9, N, 42)
        ctx.set_modes(b, None, first=33)
        psi, mid = ctx.get_modes()
        expect = a.copy()
        expect[33:42] = b
        assert np.max(np.abs(psi - expect)) < 1e-6
        assert np.max(np.abs(mid - a)) < 1e-6
        part, _ = ctx.get_modes(first=60, count=10)
        assert np.max(np.abs(part - a[60:70])) < 1e-6


def test_free_plane_waves_evolve_by_their_frequency():
    """U = 1: each free Wilson mode is an eigenmode; over many steps the leapfrog
    keeps |psi| per site constant and the plain and fused forms agree."""
    N = (6, 6, 6)
    out = {}
    for form in ("plain", "fused"):
        with Context(N=N, precision="fp64", form=form, m_fermion=0.1, m_dw=0.0, dt=0.05) as ctx:
            ctx.set_links(unit_links(N))
            assert ctx.set_free_fermions() == 0
            ctx.step(40)
            out[form] = ctx.get_modes()[0]
    assert rel_err(out["fused"], out["plain"]) < 1e-12
    dens = np.sum(np.abs(out["fused"]) ** 2, axis=(2, 3))
    assert np.max(np.abs(dens - dens[:, :1])) < 1e-10


@pytest.mark.skipif(not have_reference("wilson"), reason="reference library not built")
def test_config1_against_reference_mode_slice():
    """SU(2), N = 8, m = 0.1, r = 1, MDWHeight = 0, dt = 0.05, all 4096 plane-wave
    modes on the GPU, links exp(i A.sigma/2) with A ~ N(0, 0.3^2), E = 0, 200
    steps.  The reference (compiled from source) evolves the 64-mode slice of MPI
    rank 37 of 64; the GPU's copy of that slice must agree to 1e-12."""
    N = (8, 8, 8)
    V = volume(N)
    U = random_links(N, 0.3, 20261203)
    E = np.zeros((V, 3, 3))
    R = reference("wilson")
    m = R.ovlref_init(*N, 64, 37, 0.1, 1.0, 0.0, 6.0, 0.05, 1.0, 1)
    first = R.ovlref_first_mode()
    R.ovlref_set_links(ptr(U))
    R.ovlref_set_efield(ptr(E))
    R.ovlref_set_free_fermions()
    R.ovlref_step(200)
    rpsi = np.zeros((m, V, 2, 4), np.complex128)
    rmid = np.zeros_like(rpsi)
    R.ovlref_get_modes(ptr(rpsi.view(np.float64)), ptr(rmid.view(np.float64)))
    for form in ("plain", "fused"):
        with Context(N=N, precision="fp64", form=form, m_fermion=0.1, r_wilson=1.0, m_dw=0.0, dt=0.05,
                     t_sphaleron=6.0) as ctx:
            ctx.set_links(U)
            ctx.set_efield(E)
            assert ctx.set_free_fermions() == 0
            ctx.step(200)
            psi, mid = ctx.get_modes(first=first, count=m)
            assert rel_err(psi, rpsi) < 1e-12, form
            assert rel_err(mid, rmid) < 1e-12, form


def test_fp32_tracks_fp64_axial_charge():
    """FP32 modes against FP64 on the same inputs: after 50..200 steps N_5 agrees
    to 1e-6 of the scale of its terms (sum over modes and sites of
    |psi|^2 / 2V = n_modes / 2 for plane waves)."""
    N = (8, 8, 8)
    U = random_links(N, 0.3, 5)
    E = random_efield(N, 0.05, 6)
    res = {}
    for prec in ("fp64", "fp32"):
        with Context(N=N, precision=prec, form="fused", m_fermion=0.1, m_dw=0.0, dt=0.05, t_sphaleron=1e9) as ctx:
            ctx.set_links(U)
            ctx.set_efield(E)
            ctx.set_free_fermions()
            n5 = []
            for _ in range(4):
                ctx.step(50)
                n5.append(ctx.charges()["N5"])
            res[prec] = np.array(n5)
    scale = 8 * volume(N) / 2.0
    assert np.max(np.abs(res["fp32"] - res["fp64"])) <= 1e-6 * scale


def test_errors_leave_the_context_usable():
    N = (4, 4, 4)
    with Context(N=N, n_modes=32, precision="fp64", form="fused") as ctx:
        bad = unit_links(N)
        bad[3, 1, 2] = np.nan
        with pytest.raises(OvlError, match="NONFINITE"):
            ctx.set_links(bad)
        with pytest.raises(OvlError, match="OVL_E_ARG"):
            ctx.get_modes(first=30, count=5)
        with pytest.raises(OvlError, match="OVL_E_ARG"):
            ctx.step(-1)
        ctx.set_links(unit_links(N))
        ctx.set_free_fermions()
        before = ctx.launch_count
        ctx.step(2)
        assert ctx.launch_count > before
        assert np.isfinite(ctx.charges()["NV"])


@pytest.mark.parametrize("variant,precision,form",
                         [(v, p, f) for v in (0, 1, 2) for p, f in (("fp64", "fused"), ("fp32", "fused"), ("fp64", "plain"))]
                         + [(3, "fp32", "fused"), (3, "fp32", "plain")])
def test_every_hop_variant_matches_the_oracle(variant, precision, form):
    """The autotuner picks among kernel variants; each must give the same
    evolution (N = (4, 6, 5): an odd z extent exercises the partial z chunk of
    the z-marching variant, and V = 120 a partial last CTA of 16 sites in the
    packed FP32 variant 3; 33 modes a ragged last lane pair)."""
    N = (4, 6, 5)
    n = 33
    U = random_links(N, 0.7, 51)
    E = random_efield(N, 0.3, 52)
    psi0 = random_modes(n, N, 53)
    mid0 = random_modes(n, N, 54)
    p = oracle_params(N, m=0.1, mdw=0.0, dt=0.05, t_sph=1e9)
    opsi, omid, _, _ = oracle_leapfrog(p, U, E, psi0, mid0, 3)
    with Context(N=N, n_modes=n, precision=precision, form=form, m_fermion=0.1, m_dw=0.0, dt=0.05, t_sphaleron=1e9,
                 hop_variant=variant) as ctx:
        ctx.set_links(U)
        ctx.set_efield(E)
        ctx.set_modes(psi0, mid0)
        ctx.step(3)
        psi, mid = ctx.get_modes()
        assert rel_err(psi, opsi) < tol(precision)
        assert rel_err(mid, omid) < tol(precision)


def test_autotune_keeps_state_and_reports_each_variant():
    N = (6, 6, 6)
    U = random_links(N, 0.5, 61)
    with Context(N=N, precision="fp32", form="fused", m_fermion=0.1, m_dw=0.0, dt=0.05) as ctx:
        ctx.set_links(U)
        ctx.set_free_fermions()
        before = ctx.get_modes()
        v, ms = ctx.autotune()
        after = ctx.get_modes()
        assert v in (0, 1, 2, 3) and len(ms) == 4 and all(t > 0 for t in ms)
        assert np.array_equal(before[0], after[0]) and np.array_equal(before[1], after[1])


@pytest.mark.parametrize("precision,variant", [("fp64", 0), ("fp32", 0), ("fp40", 0), ("fp32", 3)])
@pytest.mark.parametrize("group", [1, 3])
def test_grouped_step_equals_the_ungrouped_step(precision, variant, group):
    """The grouped fused step (both half steps per group of mode blocks, with the
    half-step links built out of place) does the same arithmetic per element as
    the ungrouped fused step: equal fields and links bit for bit, with moving
    links, a ragged last group and the tSphaleron gate crossed mid-run.  With
    hop variant 3 the grouped step is the pipelined persistent launch (second
    half steps waiting on their group's first), V = 120 a partial last tile."""
    N = (4, 5, 6)
    n = 7 * 32 - 5
    U = random_links(N, 0.5, 71)
    E = random_efield(N, 0.3, 72)
    psi0 = random_modes(n, N, 73)
    mid0 = random_modes(n, N, 74)
    out = {}
    for g in (0, group):
        with Context(N=N, n_modes=n, first_mode=1, precision=precision, form="fused", m_fermion=0.1, m_dw=0.0,
                     dt=0.05, t_sphaleron=0.12, hop_variant=variant, mode_group=g) as ctx:
            ctx.set_links(U)
            ctx.set_efield(E)
            ctx.set_modes(psi0, mid0)
            ctx.step(4)
            assert ctx.tuning() == (variant, g)
            psi, mid = ctx.get_modes()
            out[g] = (psi, mid, ctx.get_links(), ctx.charges()["N5"])
    a, b = out[0], out[group]
    for k in range(3):
        assert np.array_equal(a[k], b[k])
    assert a[3] == b[3]


@pytest.mark.parametrize("group", [2, 5])
def test_pipelined_observing_step_equals_step_then_charges(group):
    """ovl_step_observe on the pipelined grouped step (FP32, hop variant 3) sums
    the charges in its second half steps: the same fields as the ungrouped
    packed step and the same charges as ovl_charges after it."""
    from overlap_b200.inputs import u1_flux

    N = (4, 6, 6)
    n = 6 * 32 + 7
    out = []
    for g, observe in ((0, False), (group, True)):
        with Context(N=N, n_modes=n, first_mode=1, precision="fp32", form="fused", m_fermion=0.05, m_dw=0.0,
                     dt=0.05, t_sphaleron=1e9, hop_variant=3, mode_group=g) as ctx:
            ctx.set_links(random_links(N, 0.5, 3))
            ctx.set_efield(random_efield(N, 0.3, 4))
            ctx.set_u1(u1_flux(N, 2))
            ctx.set_modes(random_modes(n, N, 5), random_modes(n, N, 6))
            if observe:
                ch = ctx.step_observe(3)
            else:
                ctx.step(3)
                ch = ctx.charges()
            out.append((ctx.get_modes()[0], ctx.get_links(), ch))
    (p0, u0, c0), (p1, u1, c1) = out
    assert np.array_equal(p0, p1) and np.array_equal(u0, u1)
    for k in ("NV", "N5", "PS"):
        assert abs(c0[k] - c1[k]) <= 1e-13 * max(1.0, abs(c0[k])), k


def test_pipelined_wait_times_out_on_a_counter_nobody_sets():
    """Failure detection without a GPU fault: the self-test withholds the first
    group's first-half tiles, so the second half steps waiting on them run out
    their bounded wait; the host reads OVL_E_TIMEOUT, the modes are untouched
    and the context keeps working."""
    N = (4, 4, 4)
    with Context(N=N, n_modes=96, precision="fp32", form="fused", m_fermion=0.1, m_dw=0.0, dt=0.05,
                 t_sphaleron=1e9, hop_variant=3, mode_group=1) as ctx:
        ctx.set_links(random_links(N, 0.5, 91))
        ctx.set_modes(random_modes(96, N, 92), random_modes(96, N, 93))
        before = ctx.get_modes()
        assert ctx.pipeline_selftest() == 4  # OVL_E_TIMEOUT
        after = ctx.get_modes()
        assert np.array_equal(before[0], after[0]) and np.array_equal(before[1], after[1])
        ctx.step(2)  # the pipelined step runs normally afterwards
        assert np.isfinite(ctx.charges()["N5"])


def test_fp40_storage_tracks_fp64_to_its_rounding():
    """40-bit storage (the top 40 bits of each FP64 real, FP64 hop arithmetic):
    the leapfrog follows the oracle to the storage rounding (2^-29 per write),
    and modes round-trip through ovl_set_modes / ovl_get_modes to 2^-29."""
    N = (4, 6, 5)
    n = 45
    U = random_links(N, 0.6, 81)
    E = random_efield(N, 0.3, 82)
    psi0 = random_modes(n, N, 83)
    mid0 = random_modes(n, N, 84)
    p = oracle_params(N, m=0.1, mdw=0.0, dt=0.05, t_sph=1e9)
    opsi, omid, oU, _ = oracle_leapfrog(p, U, E, psi0, mid0, 6)
    ocur = oracle_currents(p, oU, opsi, 3)
    with Context(N=N, n_modes=n, first_mode=3, precision="fp40", form="fused", m_fermion=0.1, m_dw=0.0, dt=0.05,
                 t_sphaleron=1e9) as ctx:
        ctx.set_links(U)
        ctx.set_efield(E)
        ctx.set_modes(psi0, mid0)
        a, b = ctx.get_modes()
        assert rel_err(a, psi0) < 2.0 ** -28 and rel_err(b, mid0) < 2.0 ** -28
        ctx.step(6)
        psi, mid = ctx.get_modes()
        assert rel_err(psi, opsi) < 1e-7
        assert rel_err(mid, omid) < 1e-7
        assert rel_err(ctx.get_links(), oU) < 1e-13
        cur = ctx.currents()
        scale = current_scale(opsi)
        for k in ocur:
            assert np.max(np.abs(cur[k] - ocur[k])) <= 1e-7 * scale, k


def test_fp40_free_fermions_and_observables_match_fp64():
    N = (4, 4, 6)
    out = {}
    for prec in ("fp64", "fp40"):
        with Context(N=N, precision=prec, form="fused", m_fermion=0.05, m_dw=0.0, dt=0.05) as ctx:
            assert ctx.set_free_fermions() == 0
            ctx.set_links(random_links(N, 0.4, 91))
            out[prec] = (ctx.get_modes(), ctx.charges(), ctx.fermion_energy(), ctx.color_force())
    for k in range(2):
        assert rel_err(out["fp40"][0][k], out["fp64"][0][k]) < 2.0 ** -28
    for k in ("NV", "N5", "PS", "WA"):
        assert abs(out["fp40"][1][k] - out["fp64"][1][k]) < 1e-7
    assert abs(out["fp40"][2] - out["fp64"][2]) < 1e-9 * abs(out["fp64"][2])
    assert np.max(np.abs(out["fp40"][3] - out["fp64"][3])) < 1e-8


@pytest.mark.parametrize("form", ["fused", "plain"])
def test_packed_variant_on_a_ragged_lattice(form):
    """Hop variant 3 where neither the sites nor the modes fill its tiles:
    V = 75 (a CTA of 8 sites runs past the lattice), 45 modes (the last mode
    block 13 of 32 lanes, an odd lane pair half empty); the leapfrog against the
    oracle, and the observing step's charges against ovl_charges."""
    N = (5, 5, 3)
    n = 45
    U = random_links(N, 0.6, 61)
    E = random_efield(N, 0.3, 62)
    psi0 = random_modes(n, N, 63)
    mid0 = random_modes(n, N, 64)
    p = oracle_params(N, m=0.1, mdw=0.0, dt=0.05, t_sph=1e9)
    opsi, omid, _, _ = oracle_leapfrog(p, U, E, psi0, mid0, 3)
    with Context(N=N, n_modes=n, first_mode=1, precision="fp32", form=form, m_fermion=0.1, m_dw=0.0, dt=0.05,
                 t_sphaleron=1e9, hop_variant=3) as ctx:
        ctx.set_links(U)
        ctx.set_efield(E)
        ctx.set_modes(psi0, mid0)
        ctx.step(3)
        psi, mid = ctx.get_modes()
        assert rel_err(psi, opsi) < tol("fp32") and rel_err(mid, omid) < tol("fp32")
        if form == "fused":
            ch = ctx.step_observe(1)
            ref = ctx.charges()
            for k in ("NV", "N5", "PS"):
                assert abs(ch[k] - ref[k]) <= 1e-13 * max(1.0, abs(ref[k])), k


@pytest.mark.parametrize("form", ["fused", "plain"])
def test_packed_variant_beyond_one_cta_row_of_mode_blocks(form):
    """300 modes = 10 mode blocks, the last one 12 of 32 lanes: a CTA of the
    packed kernel runs 8 mode blocks, so the second row of CTAs (blockIdx.y = 1)
    holds blocks 8 and 9.  With a U(1) background, against the oracle with the
    same phases; in the fused form the observing step's charges (one row of
    partial sums per CTA, indexed by blockIdx.y) against ovl_charges."""
    from overlap_b200.inputs import u1_flux

    N = (4, 5, 6)
    n = 300
    U = random_links(N, 0.6, 31)
    E = random_efield(N, 0.3, 32)
    psi0 = random_modes(n, N, 33)
    mid0 = random_modes(n, N, 34)
    u1 = u1_flux(N, 3)
    p = oracle_params(N, m=0.1, mdw=0.0, dt=0.05, t_sph=1e9)
    oracle().orc_set_u1(ptr(np.ascontiguousarray(u1).view(np.float64).ravel()))
    try:
        opsi, omid, _, _ = oracle_leapfrog(p, U, E, psi0, mid0, 3)
    finally:
        oracle().orc_set_u1(None)
    with Context(N=N, n_modes=n, first_mode=1, precision="fp32", form=form, m_fermion=0.1, m_dw=0.0, dt=0.05,
                 t_sphaleron=1e9, hop_variant=3) as ctx:
        ctx.set_links(U)
        ctx.set_efield(E)
        ctx.set_u1(u1)
        ctx.set_modes(psi0, mid0)
        ctx.step(3)
        psi, mid = ctx.get_modes()
        assert rel_err(psi, opsi) < tol("fp32") and rel_err(mid, omid) < tol("fp32")
        if form == "fused":
            ch = ctx.step_observe(1)
            ref = ctx.charges()
            for k in ("NV", "N5", "PS"):
                assert abs(ch[k] - ref[k]) <= 1e-13 * max(1.0, abs(ref[k])), k


@pytest.mark.parametrize("precision,form,variant",
                         [("fp64", "fused", 0), ("fp64", "fused", 1), ("fp64", "plain", 0), ("fp64", "plain", 1),
                          ("fp40", "fused", 0), ("fp40", "fused", 1)])
def test_fp64_fp40_stencils_on_a_ragged_lattice_beyond_one_cta_row(precision, form, variant):
    """300 modes = 10 mode blocks (the last one 12 of 32 lanes) on N = (3, 5, 4),
    V = 60: variant 0's last CTA holds 4 of its 8 sites, and variant 1's 4 x 2
    tiles stop short in x (3 of 4) and in y.  With a U(1) background, against
    the oracle with the same phases."""
    from overlap_b200.inputs import u1_flux

    N = (3, 5, 4)
    n = 300
    U = random_links(N, 0.6, 61)
    E = random_efield(N, 0.3, 62)
    psi0 = random_modes(n, N, 63)
    mid0 = random_modes(n, N, 64)
    u1 = u1_flux(N, 2)
    p = oracle_params(N, m=0.1, mdw=0.0, dt=0.05, t_sph=1e9)
    oracle().orc_set_u1(ptr(np.ascontiguousarray(u1).view(np.float64).ravel()))
    try:
        opsi, omid, _, _ = oracle_leapfrog(p, U, E, psi0, mid0, 3)
    finally:
        oracle().orc_set_u1(None)
    bar = tol("fp64") if precision == "fp64" else 1e-7  # FP40: the storage rounding, 2^-29 per write
    with Context(N=N, n_modes=n, first_mode=1, precision=precision, form=form, m_fermion=0.1, m_dw=0.0, dt=0.05,
                 t_sphaleron=1e9, hop_variant=variant) as ctx:
        ctx.set_links(U)
        ctx.set_efield(E)
        ctx.set_u1(u1)
        ctx.set_modes(psi0, mid0)
        ctx.step(3)
        psi, mid = ctx.get_modes()
        assert rel_err(psi, opsi) < bar and rel_err(mid, omid) < bar


@pytest.mark.parametrize("n", [40, 960, 3400])
@pytest.mark.parametrize("precision,form", [("fp64", "fused"), ("fp64", "plain"), ("fp40", "fused")])
def test_link_table_mode_blocks_per_cta(precision, form, n):
    """FP64 variants 0 and 1 and the FP40 half steps run up to 8 mode blocks per
    CTA on links gathered once in shared memory, halving the count while the
    grid would hold fewer than 4 CTAs per SM, down to 1 (the stencil without
    the table).  On N = (7, 7, 7), V = 343 (the last CTA of 8 sites holds 7;
    variant 1's 4 x 2 tiles stop short in x and y), 40, 960 and 3400 modes
    (2, 30 and 107 mode blocks, the last ones partial) give 1, 2 and 8 mode
    blocks per CTA on a 148-SM B200.  With a U(1) background, against hop
    variant 2 (one mode block per CTA, no table, the same arithmetic in the same
    order): FP64 bit for bit, FP40 to its storage rounding."""
    from overlap_b200.inputs import u1_flux

    N = (7, 7, 7)
    U = random_links(N, 0.6, 71)
    E = random_efield(N, 0.3, 72)
    psi0 = random_modes(n, N, 73)
    mid0 = random_modes(n, N, 74)
    u1 = u1_flux(N, 2)

    def run(prec, variant):
        with Context(N=N, n_modes=n, first_mode=1, precision=prec, form=form, m_fermion=0.1, m_dw=0.0, dt=0.05,
                     t_sphaleron=1e9, hop_variant=variant) as ctx:
            ctx.set_links(U)
            ctx.set_efield(E)
            ctx.set_u1(u1)
            ctx.set_modes(psi0, mid0)
            ctx.step(3)
            return ctx.get_modes()

    ref = run("fp64", 2)
    for variant in (0, 1):
        psi, mid = run(precision, variant)
        if precision == "fp64":
            assert np.array_equal(psi, ref[0]) and np.array_equal(mid, ref[1]), variant
        else:
            assert rel_err(psi, ref[0]) < 1e-7 and rel_err(mid, ref[1]) < 1e-7, variant


@pytest.mark.parametrize("group", [4, 9])
def test_pipelined_step_beyond_one_cta_row_of_mode_blocks(group):
    """The pipelined grouped step (hop variant 3) on 10 mode blocks in groups
    of 4 (a ragged last group of 2) and of 9 (one group past a CTA row of the
    ungrouped kernel): bit for bit the ungrouped packed step."""
    N = (4, 5, 6)
    n = 300
    out = {}
    for g in (0, group):
        with Context(N=N, n_modes=n, first_mode=1, precision="fp32", form="fused", m_fermion=0.1, m_dw=0.0,
                     dt=0.05, t_sphaleron=1e9, hop_variant=3, mode_group=g) as ctx:
            ctx.set_links(random_links(N, 0.5, 41))
            ctx.set_efield(random_efield(N, 0.3, 42))
            ctx.set_modes(random_modes(n, N, 43), random_modes(n, N, 44))
            ctx.step(3)
            out[g] = (*ctx.get_modes(), ctx.get_links())
    for k in range(3):
        assert np.array_equal(out[0][k], out[group][k])


def test_packed_variant_is_fp32_only():
    with pytest.raises(OvlError):
        Context(N=(4, 4, 4), precision="fp64", form="fused", m_dw=0.0, dt=0.05, hop_variant=3)


@pytest.mark.parametrize("precision,variant", [("fp64", 0), ("fp32", 0), ("fp32", 3), ("fp40", 0)])
def test_step_observe_equals_step_then_charges(precision, variant):
    """ovl_step_observe sums N_V, N_5, PS inside the last half step: the same
    state as ovl_step and the same charges as ovl_charges (both form the
    bilinears in FP64 from the stored modes; only the summation order differs)."""
    from overlap_b200.inputs import u1_flux

    N = (4, 6, 6)
    out = []
    for observe in (False, True):
        with Context(N=N, n_modes=80, first_mode=1, precision=precision, form="fused", m_fermion=0.05, m_dw=0.0,
                     dt=0.05, t_sphaleron=1e9, hop_variant=variant) as ctx:
            ctx.set_links(random_links(N, 0.5, 3))
            ctx.set_efield(random_efield(N, 0.3, 4))
            ctx.set_u1(u1_flux(N, 2))
            ctx.set_modes(random_modes(80, N, 5), random_modes(80, N, 6))
            if observe:
                ch = ctx.step_observe(3)
            else:
                ctx.step(3)
                ch = ctx.charges()
            out.append((ctx.get_modes()[0], ctx.get_links(), ch))
    (p0, u0, c0), (p1, u1, c1) = out
    assert np.array_equal(p0, p1) and np.array_equal(u0, u1)
    for k in ("NV", "N5", "PS"):
        assert abs(c0[k] - c1[k]) <= 1e-13 * max(1.0, abs(c0[k])), k
