#!/usr/bin/env python
"""Benchmark: mode-site updates per second of the Wilson fermion leapfrog.

One "step" is one full leapfrog step (Dynamics::Fermions::Update,
FERMIONS/WILSON/Update.cpp:48-79) of every mode of the workload: two half steps
of psi += dt D psi' and two link half steps.  A mode-site update (MSU) is one
mode at one site advanced by one step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload n16|n8]

Default workload (n16): SU(2), N = 16^3, Wilson r = 1, m = 0.05, MDWHeight = 0,
dt = 0.05, all 32768 modes (free plane waves), FP32-class modes with FP64 links;
quasi-particle gauge fields (occupancy 1/g^2 = 4 below Qs = 1, Gauss's law
restored on the device) and a U(1) background with n_B = 4 flux quanta in the
hopping term; links move every half step.  The
modes (8.6 GB per field in FP32) exceed the 126 MB L2, so no L2 flush is
needed between steps.  The line reports the FP32 fused form as `value`, the
FP64 plain (two-phase, as the reference) and FP64 fused forms beside it, the
roofline of the dominant kernel, the end-to-end rate through the C ABI with
host buffers, and the reference's own CPU code on this host's cores.

Under torchrun (N > 1) every rank runs an independent replica on its own GPU
(the workload does not shard across GPUs); value = all ranks' MSU / max time.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import shutil
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    "n16": dict(N=(16, 16, 16), m=0.05, r=1.0, mdw=0.0, dt=0.05, init="quasi", n0=4.0, qs=1.0, nb=4,
                seed=20261203, ref_ranks=512),
    "n8": dict(N=(8, 8, 8), m=0.1, r=1.0, mdw=0.0, dt=0.05, link_sigma=0.3, e_sigma=0.0, seed=20261203,
               ref_ranks=64),
}
METRIC = "mode-site updates/s"


# ----------------------------------------------------------------- helpers --
def gauge_fields(wl):
    """(links, E) of a workload before Gauss's law is restored: quasi-particles
    (occupancy n0 = 1/g^2 below Qs) or seeded random links and E."""
    from overlap_b200.inputs import quasi_particles, random_efield, random_links

    if wl.get("init") == "quasi":
        return quasi_particles(wl["N"], wl["n0"], wl["qs"], wl["seed"])
    return random_links(wl["N"], wl["link_sigma"], wl["seed"]), random_efield(wl["N"], wl["e_sigma"], wl["seed"] + 1)


def setup_gauge(ctx, wl):
    """Links, E (Gauss's law restored for the quasi-particle start, as
    SetQuasiParticles does) and the U(1) background of the workload."""
    from overlap_b200.inputs import u1_flux

    U, E = gauge_fields(wl)
    ctx.set_links(U)
    ctx.set_efield(E)
    if wl.get("init") == "quasi":
        ctx.gauss_restore()
    if wl.get("nb"):
        ctx.set_u1(u1_flux(wl["N"], wl["nb"]))



def volume(N):
    return N[0] * N[1] * N[2]


def n_modes(N):
    return 8 * volume(N)


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# What each FP32-class form stores and computes in.
DTYPES = {"fp32": "f32 modes and hop arithmetic, f64 links",
          "fp40": "modes in 40 bits (top bits of f64), f64 hop arithmetic, observables and links"}

# The FP32 fused half-step kernel of each hop variant (ovl_wilson.cu).
HOP_KERNELS = {0: "wilson_tuned_kernel<float,1,0,LinksF32<{u1}>>",
               1: "wilson_tuned_kernel<float,1,1,LinksF32<{u1}>>",
               2: "wilson_zmarch_kernel<float,1,LinksF32<{u1}>>",
               3: "wilson_packed_kernel<1,{u1},false>"}


def committed_traffic(kernel: str):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text())
    v = d.get(kernel)
    return None if v is None else float(v["bytes_per_launch"])


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"ovl_clocks_{os.getpid()}.csv"

    def __enter__(self):
        exe = shutil.which("nvidia-smi")
        if exe:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen([exe, f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                         "-i", str(self.gpu), "-lms", "200"], stdout=self.fh,
                                        stderr=subprocess.DEVNULL)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if not self.proc or not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        self.path.unlink(missing_ok=True)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------ reference CPU arm --
def _ref_worker(args):
    """One emulated MPI rank of the reference's own code (compiled from source):
    its mode slice advanced by `steps` Dynamics::Fermions::Update calls."""
    wl, rank, steps, warmup = args
    sys.path.insert(0, str(ROOT / "tests"))
    import numpy as np

    from _oracle import ptr, reference

    R = reference("wilson")
    N = wl["N"]
    m = R.ovlref_init(*N, wl["ref_ranks"], rank, wl["m"], wl["r"], wl["mdw"], 1e300, wl["dt"], 1.0, 1)
    U, E = gauge_fields(wl)
    R.ovlref_set_links(ptr(np.ascontiguousarray(U)))
    R.ovlref_set_efield(ptr(np.ascontiguousarray(E)))
    if wl.get("init") == "quasi":
        R.ovlref_gauss_restore(ptr(np.zeros(2)))  # the reference's own GaussLawRestoration::Restore
    R.ovlref_set_free_fermions()
    if warmup:
        R.ovlref_step(warmup)
    secs = R.ovlref_step(steps)
    return m, secs


def reference_cpu(wl, steps: int, warmup: int, max_procs: int | None = None):
    """Aggregate MSU/s of the reference hot path on this host: one process per
    core, each an emulated MPI rank (MPI/ModePartition.cpp:12-24) holding
    4*Nc*V/ref_ranks modes."""
    cores = os.cpu_count() or 1
    procs = min(cores, wl["ref_ranks"], max_procs or cores)
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        res = pool.map(_ref_worker, [(wl, r, steps, warmup) for r in range(procs)])
    wall = time.perf_counter() - t0
    V = volume(wl["N"])
    msu = sum(m * V * steps for m, _ in res)
    slowest = max(s for _, s in res)
    modes = res[0][0]
    return {"value": msu / slowest, "unit": METRIC, "cores": procs, "kind": "reference",
            "sample": f"{steps} leapfrog steps of a {modes}-mode slice (MPI rank emulation, {wl['ref_ranks']} ranks) "
                      f"per process, {procs} processes, reference C++ built -O3 -march=x86-64-v3",
            "seconds": slowest, "wall_seconds": wall}


# --------------------------------------------------------- oracle slice --
# The checker for the accuracy leg: a 64-mode slice of the workload (global
# modes 4096-4159, one MPI rank of 512) advanced by the oracle (the plain-C
# restatement, tests' checker) on host cores while the GPU legs run, started in
# spawned processes before any CUDA call.  Each process restores Gauss's law
# (the reference's algorithm, restated) on the workload's fields itself.
SLICE_FIRST, SLICE_MODES, SLICE_PROCS = 4096, 64, 4


def _oracle_slice_worker(args):
    wl, first, count, steps = args
    sys.path.insert(0, str(ROOT / "tests"))
    import ctypes as C

    import numpy as np

    from _oracle import oracle, orc_params, ptr
    from overlap_b200.inputs import u1_flux

    N = wl["N"]
    V = volume(N)
    p = orc_params(tuple(N), r=wl["r"], m=wl["m"], mdw=wl["mdw"], dt=wl["dt"])
    U, E = gauge_fields(wl)
    U, E = np.ascontiguousarray(U), np.ascontiguousarray(E)
    if wl.get("init") == "quasi":
        oracle().orc_gauss_restore(C.byref(p), ptr(U), ptr(E), 10000, 1e-14, ptr(np.zeros(2)))
    U0, E0 = U.copy(), E.copy()
    psi = np.zeros((count, V, 2, 4), np.complex128)
    mid = np.zeros_like(psi)
    oracle().orc_free_fermions(C.byref(p), first, count, ptr(psi.view(np.float64)), ptr(mid.view(np.float64)))
    u1 = np.ascontiguousarray(u1_flux(N, wl["nb"])).view(np.float64).ravel() if wl.get("nb") else None
    oracle().orc_set_u1(ptr(u1) if u1 is not None else None)
    t = C.c_int(0)
    t0 = time.perf_counter()
    oracle().orc_wilson_leapfrog(C.byref(p), ptr(U), ptr(E), ptr(psi.view(np.float64)), ptr(mid.view(np.float64)),
                                 count, C.byref(t), steps)
    secs = time.perf_counter() - t0
    cur = [np.zeros(4 * V) for _ in range(4)] + [np.zeros(V), np.zeros(V)]
    oracle().orc_wilson_currents(C.byref(p), ptr(U), ptr(psi.view(np.float64)), count, first, *[ptr(a) for a in cur])
    oracle().orc_set_u1(None)
    charges = np.array([cur[0].reshape(V, 4)[:, 0].sum(), cur[1].reshape(V, 4)[:, 0].sum(), cur[4].sum()])
    return psi, mid, U, charges, U0, E0, secs


def oracle_slice_start(wl, steps):
    """Starts the oracle slice (SLICE_PROCS spawned processes); returns the pool
    and its pending result."""
    ctx = mp.get_context("spawn")
    pool = ctx.Pool(SLICE_PROCS)
    per = SLICE_MODES // SLICE_PROCS
    jobs = [(wl, SLICE_FIRST + k * per, per, steps) for k in range(SLICE_PROCS)]
    return pool, pool.map_async(_oracle_slice_worker, jobs), steps


def oracle_slice_compare(handle, wl, device, hop_variant):
    """The GPU forms on the oracle's slice, same fields and steps: FP64 fused
    and FP32 fused (hop variant `hop_variant`).  Errors: fields max |a - b| /
    max |b|, links the same, charges N_V, N_5, PS of the slice absolute and over
    the sum of the modes' contributions (64 x 1/2 for plane waves)."""
    import numpy as np

    from overlap_b200 import Context
    from overlap_b200.inputs import u1_flux

    pool, pending, steps = handle
    res = pending.get()
    pool.close()
    pool.join()
    psi = np.concatenate([r[0] for r in res])
    mid = np.concatenate([r[1] for r in res])
    oU = res[0][2]
    och = sum(r[3] for r in res)
    U0, E0 = res[0][4], res[0][5]
    N = wl["N"]
    scale = SLICE_MODES * 0.5
    out = {"slice": f"global modes {SLICE_FIRST}-{SLICE_FIRST + SLICE_MODES - 1} (one MPI rank of 512)",
           "steps": steps, "oracle_seconds": max(r[6] for r in res), "oracle_processes": SLICE_PROCS,
           "oracle_charges": {"NV": och[0], "N5": och[1], "PS": och[2]}}
    for prec, hv in (("fp64", -1), ("fp32", hop_variant)):
        with Context(N=N, n_modes=SLICE_MODES, first_mode=SLICE_FIRST, precision=prec, form="fused",
                     m_fermion=wl["m"], r_wilson=wl["r"], m_dw=wl["mdw"], dt=wl["dt"], t_sphaleron=1e300,
                     device=device, hop_variant=hv) as ctx:
            ctx.set_links(U0)
            ctx.set_efield(E0)
            if wl.get("nb"):
                ctx.set_u1(u1_flux(N, wl["nb"]))
            ctx.set_free_fermions()
            ctx.step(steps)
            gp, gm = ctx.get_modes()
            ch = ctx.charges()
            o = {"hop_variant": ctx.tuning()[0],
                 "field_rel_err": max(float(np.max(np.abs(gp - psi)) / np.max(np.abs(psi))),
                                      float(np.max(np.abs(gm - mid)) / np.max(np.abs(mid)))),
                 "links_rel_err": float(np.max(np.abs(ctx.get_links() - oU)) / np.max(np.abs(oU)))}
            for k, name in enumerate(("NV", "N5", "PS")):
                err = abs(ch[name] - och[k])
                o[f"{name}_abs_err"] = err
                o[f"{name}_err_of_mode_sum"] = err / scale
            out[prec] = o
    return out


# ---------------------------------------------------------------- GPU arm --
def time_form(wl, precision, form, steps, warmup, device, profile, hop_variant=-1, mode_group=0):
    if hop_variant == 3 and precision != "fp32":
        hop_variant = -1  # the packed-pair kernel is FP32's only: the others autotune
    import numpy as np
    import torch

    from overlap_b200 import Context

    N = wl["N"]
    stream = torch.cuda.Stream(device)  # a real stream: the library and the events share it
    ctx = Context(N=N, n_modes=wl.get("modes"), precision=precision, form=form, m_fermion=wl["m"], r_wilson=wl["r"], m_dw=wl["mdw"],
                  dt=wl["dt"], t_sphaleron=1e300, device=device, stream=stream.cuda_stream, hop_variant=hop_variant,
                  mode_group=mode_group)
    ctx.torch_stream = stream  # keeps the stream alive as long as the context
    setup_gauge(ctx, wl)
    assert ctx.set_free_fermions() == 0
    if hop_variant < 0:
        variant, variant_ms = ctx.autotune()
    else:
        variant, variant_ms = hop_variant, None
    ctx.step(warmup)
    ctx.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if profile:
        ctx.profile(True)
    l0 = ctx.launch_count
    barrier()
    torch.cuda.synchronize(device)
    start.record(stream)
    ctx.step(steps)
    stop.record(stream)
    torch.cuda.synchronize(device)
    barrier()
    ms = start.elapsed_time(stop)
    out = {"ms": ms, "launches": ctx.launch_count - l0, "charges": ctx.charges(),
           "hop_variant": variant, "hop_variant_ms": variant_ms, "mode_group": ctx.tuning()[1]}
    if profile:
        out["prof"] = ctx.profile_read()
        ctx.profile(False)
    return ctx, out


def time_e2e(ctx, wl, steps, device):
    """Same metric through the C ABI with host buffers: each step uploads the
    gauge fields from pinned host memory, advances one leapfrog step and reads
    the step's charges (N_V, N_5, PS, summed inside the step by
    ovl_step_observe) back to pinned host memory.  The calls are the
    asynchronous forms (ovl_upload_gauge_async, ovl_step_observe_async): step
    k+1 is queued, uploads included, before the host waits for step k's
    charges, so the GPU does not idle between steps; every step's charges are
    read on the host inside the timed region."""
    import numpy as np
    import torch

    N = wl["N"]
    U = torch.empty((volume(N), 3, 4), dtype=torch.float64, pin_memory=True).numpy()
    E = torch.empty((volume(N), 3, 3), dtype=torch.float64, pin_memory=True).numpy()
    outs = [torch.empty(3, dtype=torch.float64, pin_memory=True).numpy() for _ in range(2)]
    U[...] = ctx.get_links()
    E[...] = ctx.get_efield()
    stream = ctx.torch_stream
    done = [torch.cuda.Event(), torch.cuda.Event()]
    ctx.synchronize()
    barrier()
    t0 = time.perf_counter()
    ch = None
    for k in range(steps):
        ctx.upload_gauge_async(U, E)
        ctx.step_observe_async(1, outs[k % 2])  # N_V, N_5, PS summed inside the step's second half step
        done[k % 2].record(stream)
        if k > 0:
            done[(k - 1) % 2].synchronize()
            ch = dict(zip(("NV", "N5", "PS"), outs[(k - 1) % 2].tolist()))  # step k-1's charges on the host
    done[(steps - 1) % 2].synchronize()
    ch = dict(zip(("NV", "N5", "PS"), outs[(steps - 1) % 2].tolist()))
    ctx.synchronize()
    secs = time.perf_counter() - t0
    secs = max_over_ranks(secs)
    h2d = U.nbytes + E.nbytes
    d2h = 3 * 8
    return secs, h2d, d2h, ch


def accuracy(wl, steps, every, device, hop_variant=-1, field_modes=256):
    """FP32 and FP40 modes against FP64 on the same inputs over `steps` leapfrog
    steps, sampled every `every` steps.  For each observable o (N_5, N_CS, the
    vector charge N_V = sum jV^0, the fermion energy H_F, the gauge energy T00,
    the Gauss-law maximum): the error max_t |o(t) - o_64(t)| absolute, relative
    to the FP64 span max_t |o_64(t) - o_64(0)| and relative to max_t |o_64(t)|.
    N_CS is accumulated by the cooling-path rule (CoolingMethod::GetDeltaNCs,
    cooling off).  Fields: ||psi - psi_64|| / ||psi_64|| over the first
    `field_modes` modes at the end.  FP32 runs hop variant `hop_variant` (the
    timed FP32 context's choice; -1 tunes), FP40 and FP64 tune their own."""
    import numpy as np
    import torch

    from overlap_b200 import Context

    N = wl["N"]
    names = ("N5", "NCS", "NV", "HF", "T00", "gauss_max")
    series, fields = {}, {}
    for prec in ("fp64", "fp32", "fp40"):
        hv = hop_variant if prec == "fp32" else -1  # the FP32 form runs the timed variant; the others tune
        ctx = Context(N=N, n_modes=wl.get("modes"), precision=prec, form="fused", m_fermion=wl["m"], r_wilson=wl["r"],
                      m_dw=wl["mdw"], dt=wl["dt"], t_sphaleron=1e300, device=device, hop_variant=hv)
        setup_gauge(ctx, wl)
        ctx.set_free_fermions()
        ctx.ncs_update()

        def sample(ncs):
            ch, b = ctx.charges(), ctx.bulk()
            return (ch["N5"], ncs, ch["NV"], ctx.fermion_energy(), b["T00"], b["gauss_max"])

        rows = [sample(0.0)]
        for _ in range(steps // every):
            ctx.step(every)
            rows.append(sample(ctx.ncs_update()[1]))
        nf = min(field_modes, ctx.n_modes)
        fields[prec] = ctx.get_modes(0, nf)[0]
        ctx.close()
        series[prec] = np.array(rows)
        torch.cuda.synchronize(device)
    out = {"steps": (steps // every) * every, "every": every, "fp32_hop_variant": hop_variant}
    b = series["fp64"]
    for k, name in enumerate(names):
        span = float(np.max(np.abs(b[:, k] - b[0, k])))
        out[f"{name}_fp64_final"] = float(b[-1, k])
        out[f"{name}_fp64_span"] = span
    for prec in ("fp32", "fp40"):
        o = {}
        for k, name in enumerate(names):
            err = float(np.max(np.abs(series[prec][:, k] - b[:, k])))
            span = out[f"{name}_fp64_span"]
            scale = float(np.max(np.abs(b[:, k])))
            o[f"{name}_rel_err"] = err / span if span > 0 else (0.0 if err == 0 else None)
            o[f"{name}_abs_err"] = err
            o[f"{name}_err_of_value"] = err / scale if scale > 0 else 0.0
        f64 = fields["fp64"]
        o["field_rel_err"] = float(np.linalg.norm(fields[prec] - f64) / np.linalg.norm(f64))
        out[prec] = o
    out["field_modes"] = int(fields["fp64"].shape[0])
    return out


def ensemble_leg(steps, warmup, device, tile=0):
    """The batched-ensemble configuration: 64 independent SU(2) trajectories,
    16 each at N = 8, 10, 12, 16, 4096 Z2 stochastic vacuum modes each, U(1)
    flux n_B in {0, 2, 4, 8}, dt = 0.05, FP32 modes, seeded random links
    (sigma 0.3) and E (sigma 0.1).  Times `steps` leapfrog steps of the
    ensemble (one CUDA graph per step) against the same members stepped one
    context at a time with the packed kernel (hop variant 3).  tile 0: the
    ensemble tunes its tiles; 16: packed-pair tiles."""
    import numpy as np
    import torch

    from overlap_b200 import Ensemble, Params
    from overlap_b200.inputs import random_efield, random_links, u1_flux

    sizes = [8] * 16 + [10] * 16 + [12] * 16 + [16] * 16
    params = [Params(N=(n, n, n), n_modes=4096, precision="fp32", form="fused", m_fermion=0.05, r_wilson=1.0,
                     m_dw=0.0, dt=0.05, t_sphaleron=1e300, device=device, hop_variant=3)
              for n in sizes]
    work = sum(p.n_modes * n ** 3 for p, n in zip(params, sizes))  # mode-sites per step
    ens = Ensemble(params)
    try:
        if tile:
            ens.set_tile(tile)
        for i, n in enumerate(sizes):
            N = (n, n, n)
            ens[i].set_links(random_links(N, 0.3, 1000 + i))
            ens[i].set_efield(random_efield(N, 0.1, 2000 + i))
            nb = (0, 2, 4, 8)[i % 4]
            if nb:
                ens[i].set_u1(u1_flux(N, nb))
            ens[i].set_stochastic_modes(seed=3000 + i)
        stream = torch.cuda.ExternalStream(ens.stream, device=device)
        ens.step(warmup)
        ens.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = ens.info()["launches"]
        a.record(stream)
        ens.step(steps)
        b.record(stream)
        b.synchronize()
        t_ens = a.elapsed_time(b) / 1e3
        launches_per_step = (ens.info()["launches"] - l0) / steps
        # the same members, one context at a time (same stream, same kernels)
        a.record(stream)
        for _ in range(steps):
            for i in range(len(sizes)):
                ens[i].step(1)
        b.record(stream)
        b.synchronize()
        t_seq = a.elapsed_time(b) / 1e3
        info = ens.info()
        n5 = ens.charges()[:, 1]
    finally:
        ens.close()
    return {"config": "64 trajectories (16 each at N=8,10,12,16), 4096 Z2 stochastic modes each, "
                      "n_B in {0,2,4,8}, dt=0.05, FP32 modes",
            "value": work * steps / t_ens, "unit": METRIC, "ms_per_step": 1e3 * t_ens / steps,
            "one_context_at_a_time": work * steps / t_seq, "tile_sites": info["sites"],
            "tile_ms": info["tile_ms"], "launches_per_step": launches_per_step,
            "N5_finite": bool(np.all(np.isfinite(n5)))}


def serving_leg(count, device, tile=0, time_box=60.0):
    """The serving configuration: `count` Poisson arrivals (mean 20/s) of
    trajectory requests, N uniform over {8, 12, 16, 24}, 4096-8192 modes,
    200-2000 steps, U(1) flux n_B in {0, 2, 4, 8}, FP32 modes; a quarter
    SU(3), an eighth overlap fermions (Chebyshev degree 64, plane waves), the
    Wilson requests on Z2 stochastic modes.  Admitted by device memory: Wilson
    requests (SU(2) and SU(3)) into one continuously batched ensemble on the
    stream of highest priority, overlap requests as contexts of their own
    beside it; N_5, N_CS and energy streamed every 50 steps.  The offered load
    is far above the GPU's capacity (one overlap step on 24^3 with 8192 modes
    is about a second of GPU time), so the leg is time-boxed: it serves for
    `time_box` seconds and reports the offered and the sustained load, the
    requests completed, still running, queued and not yet arrived, and
    latency over the completed ones.  Queued requests are admitted smallest
    total work first, every one that fits (in arrival order two or three
    overlap requests on 24^3 fill the memory and nothing finishes inside the
    box).  tile: the ensemble's tile shape (16: packed-pair tiles; 0: tuned)."""
    from overlap_b200.serve import Server, poisson_requests, request_cost

    reqs = poisson_requests(count, 20.0, seed=7, su3_fraction=0.25, overlap_fraction=0.125)
    window = max(reqs[-1].arrival, 1e-9)
    offered = sum(r.mode_sites() * r.steps for r in reqs) / window
    offered_cost = sum(request_cost(r) * r.steps for r in reqs) / window
    srv = Server(precision="fp32", device=device, tick_steps=50, tile=tile, admission="shortest")
    try:
        m = srv.serve(reqs, time_box=time_box)
        streamed = sum(len(r.observables) for r in reqs)
        done_kinds = {}
        for r in srv.done:
            k = f"SU({r.n_colours}) {r.fermion}"
            done_kinds[k] = done_kinds.get(k, 0) + 1
    finally:
        srv.close()
    kinds = {}
    for r in reqs:
        k = f"SU({r.n_colours}) {r.fermion}"
        kinds[k] = kinds.get(k, 0) + 1
    m.update({"config": f"{count} requests, Poisson 20/s (arrival window {window:.1f} s), N in {{8,12,16,24}}, "
                        "4096-8192 modes, 200-2000 steps, Wilson or overlap (Chebyshev degree 64), SU(2)/SU(3), "
                        "n_B in {0,2,4,8}, FP32, observables every 50 steps; admission by device memory, smallest "
                        f"work first; time-boxed at {time_box:g} s, latency over the requests completed in the box",
              "request_kinds": kinds, "completed_kinds": done_kinds,
              "offered_mode_site_updates_per_s": offered, "offered_wilson_equivalent_per_s": offered_cost,
              "sustained_over_offered": m["throughput_wilson_equivalent"] / offered_cost,
              "observations_streamed": streamed})
    return m


def su3_overlap_leg(steps, warmup, device, modes=0):
    """The SU(3) overlap configuration: N = 12^3, overlap fermions
    D_ov = 1 + gamma_5 sign(H_W) with Wilson kernel mass -1 (MDWHeight 1, m = 0),
    sign(H_W) through the Chebyshev series of degree 96 of (H_W^2)^(-1/2) on the
    spectrum rescaled to [0.01, 1] (lambda_max the bound (|6r - 2M|/2 + 3)^2 on
    H_W^2), all 20736 plane-wave modes in FP32, FP64 links with
    reunitarisation; seeded random links exp(i A^a t^a), A ~ N(0, 0.5^2), and E
    ~ N(0, 0.1^2) (links move every half step).  Times `steps` leapfrog steps;
    N_5 (one more overlap application, OverlapCurrents.cpp) and N_CS (geodesic
    Delta N_CS) are timed once after them as the per-step observables."""
    import torch

    from overlap_b200 import Context
    from overlap_b200.inputs import random_efield_su3, random_links_su3

    N = (12, 12, 12)
    V = volume(N)
    M = modes or 12 * V
    K, eps = 96, 0.01
    stream = torch.cuda.Stream(device)
    ctx = Context(N=N, n_colours=3, n_modes=M, fermion="overlap", sign_method="chebyshev", cheb_degree=K,
                  cheb_eps=eps, precision="fp32", m_fermion=0.0, m_dw=1.0, r_wilson=1.0, dt=0.05, t_sphaleron=1e300,
                  reunitarize=True, device=device, stream=stream.cuda_stream)
    try:
        ctx.set_links(random_links_su3(N, 0.5, 20261203))
        ctx.set_efield(random_efield_su3(N, 0.1, 20261204))
        assert ctx.set_free_fermions() == 0
        ctx.step(warmup)
        ctx.ncs_update()
        ctx.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = ctx.launch_count
        torch.cuda.synchronize(device)
        a.record(stream)
        ctx.step(steps)
        b.record(stream)
        b.synchronize()
        ms = a.elapsed_time(b)
        launches = ctx.launch_count - l0
        variant = ctx.tuning()[0]
        t0 = time.perf_counter()
        ch = ctx.charges()
        t1 = time.perf_counter()
        d, total = ctx.ncs_update()
        t2 = time.perf_counter()
    finally:
        ctx.close()
    field = M * V * 12 * 8  # one FP32 mode field
    # algorithmic bytes of one overlap application (the minimum: each Clenshaw
    # term reads b_{k+1} and b_{k+2} and writes b_k once, 3 K elements per
    # mode-site, plus 6 for phi, D chi and the combination into the destination)
    alg = field * (3 * K + 6)
    # the field passes the kernels make as built: 7 per term (w = D b: read b,
    # write w; term: read w, b_1, b_2, phi, write b_0), K + 1 terms, then D chi
    # (2) and the combination into the destination (4); two memsets (2)
    built = field * (7 * (K + 1) + 8)
    half_ms = ms / (2 * steps)
    peak, peak_kind = measured_peaks()
    return {"config": f"SU(3), N=12^3, overlap (Chebyshev degree {K}, [eps, 1] = [{eps}, 1]), Wilson kernel mass -1, "
                      f"{M} plane-wave modes FP32, FP64 links reunitarised, random links sigma 0.5, E sigma 0.1",
            "value": M * V * steps / (ms / 1e3), "unit": METRIC, "steps": steps, "ms_per_step": ms / steps,
            "launches_per_step": launches / steps,
            "hop_variant": variant,
            "overlap_application": {"ms": half_ms, "algorithmic_bytes": alg, "achieved_GBs": alg / (half_ms / 1e3) / 1e9,
                                    "frac_of_peak": alg / (half_ms / 1e3) / 1e9 / peak, "peak_source": peak_kind,
                                    "bytes_as_built": built,
                                    "built_GBs": built / (half_ms / 1e3) / 1e9},
            "observables_per_step_ms": {"N5": 1e3 * (t1 - t0), "N_CS": 1e3 * (t2 - t1)},
            "N5": ch["N5"], "delta_NCS": d}


# ------------------------------------------------------------ distributed --
_dist = None


def init_dist():
    global _dist
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        _dist = dist
    return int(os.environ.get("RANK", "0")), ws, int(os.environ.get("LOCAL_RANK", "0"))


def barrier():
    if _dist is not None:
        _dist.barrier()


def max_over_ranks(x: float) -> float:
    if _dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    _dist.all_reduce(t, op=_dist.ReduceOp.MAX)
    return float(t.item())


# ------------------------------------------------------------------- main --
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", choices=tuple(WORKLOADS), default="n16")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the batched-ensemble leg")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving leg")
    ap.add_argument("--no-su3", action="store_true", help="skip the SU(3) overlap leg")
    ap.add_argument("--su3-steps", type=int, default=3, help="timed leapfrog steps of the SU(3) overlap leg")
    ap.add_argument("--serving-requests", type=int, default=256, help="requests of the serving leg")
    ap.add_argument("--serving-time-box", type=float, default=60.0, help="seconds the serving leg serves")
    ap.add_argument("--headline", choices=("fp40", "fp32"), default="fp32",
                    help="the FP32-class form of the headline value (the other is reported beside it)")
    ap.add_argument("--mode-group", type=int, default=0,
                    help="fused form: mode blocks per group (0: whole batch, -1: autotune with the variant)")
    # -1: the library's autotuner picks the hop kernel (and the ensemble its
    # tiles).  Where a launch takes a millisecond or more it times each
    # candidate over sustained windows, under the power cap that sets the clock
    # of a long run, so it sees the packed kernel's lower power per mode-site.
    ap.add_argument("--hop-variant", type=int, default=-1, choices=(-1, 0, 1, 2, 3),
                    help="-1: autotune the hop kernel before warm-up; 0-3: fixed variant (3: FP32 forms, the "
                         "other forms autotune)")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 forms")
    ap.add_argument("--modes", type=int, default=0, help="run a smaller case with this many modes (profiling)")
    ap.add_argument("--accuracy-steps", type=int, default=1000,
                    help="FP32-vs-FP64 accuracy leg length in leapfrog steps (0 = skip)")
    ap.add_argument("--no-oracle-slice", action="store_true",
                    help="skip the oracle's 64-mode slice beside the accuracy leg")
    args = ap.parse_args()
    wl = dict(WORKLOADS[args.workload])
    N = wl["N"]
    V, M = volume(N), n_modes(N)
    if args.modes:
        M = wl["modes"] = min(args.modes, M)
    rank, world, local = init_dist()
    if wl.get("init") == "quasi":
        init = (f"quasi-particles (occupancy n0=1/g^2={wl['n0']} below Qs={wl['qs']}, seed {wl['seed']}), Gauss law "
                f"restored; links updated every half step")
    else:
        init = (f"seeded random links (sigma={wl['link_sigma']}) and E (sigma={wl['e_sigma']}), links updated every "
                f"half step")
    if wl.get("nb"):
        init += (f"; U(1) background B along z, n_B={wl['nb']} flux quanta, in the hopping term (the reference arm's "
                 f"hop has no U(1) term; its cost does not depend on the background)")
    config = {"workload": f"SU(2) Wilson fermions, N={N[0]}x{N[1]}x{N[2]}, {M} modes (plane-wave basis), "
                          f"r={wl['r']}, m={wl['m']}, MDWHeight={wl['mdw']}, dt={wl['dt']}",
              "lattice": list(N), "modes": M, "gauge_init": init,
              "l2": "inputs larger than L2 (no flush)", "parallelism": f"replicas x{world}"}

    if args.impl == "reference":
        if rank == 0:
            # the GPU arm's step and warm-up counts; a step is one leapfrog step of
            # every process's 64-mode slice (about 0.15 s per process at N=16)
            steps, warmup = max(1, args.steps), max(3, args.warmup)
            cpu = reference_cpu(wl, steps=steps, warmup=warmup)
            line = {"metric": METRIC, "value": cpu["value"], "unit": METRIC, "n_gpus": args.gpus, "steps": steps,
                    "warmup": warmup, "ms_per_step": 1e3 * cpu["seconds"] / steps,
                    "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                    "data": "synthetic", "config": config, "impl": "reference",
                    "cpu_baseline": {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")},
                    "e2e": {"value": cpu["value"], "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
            print(json.dumps(line), flush=True)
        return

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        # before any CUDA call (spawned workers)
        # about 2.5 s per process: 12 steps of a 64-mode slice at N=16, 60 at N=8
        cpu = reference_cpu(wl, steps=12 if args.workload == "n16" else 60, warmup=0, max_procs=64)
    orc_slice = None
    if rank == 0 and args.accuracy_steps > 0 and not args.no_oracle_slice:
        # the checker of the accuracy leg, on host cores while the GPU legs run
        orc_slice = oracle_slice_start(wl, args.accuracy_steps)

    import torch

    device = local if torch.cuda.device_count() > local else 0
    torch.cuda.set_device(device)
    K, W = args.steps, max(3, args.warmup)

    # batched form of FP32 storage class (headline: --headline, FP32 by default)
    head = args.headline
    with ClockSampler(device) as clocks:
        ctx, fp32 = time_form(wl, head, "fused", K, W, device, profile=True, hop_variant=args.hop_variant,
                                 mode_group=args.mode_group)
    clk = clocks.summary()
    e2e_steps = max(3, min(K, 60))
    e2e_secs, h2d, d2h, _ = time_e2e(ctx, wl, e2e_steps, device)
    ctx.close()
    del ctx
    ms = max_over_ranks(fp32["ms"])
    value = world * M * V * K / (ms / 1e3)

    forms = {}
    other = "fp32" if head == "fp40" else "fp40"
    c, r = time_form(wl, other, "fused", K, W, device, profile=True, hop_variant=args.hop_variant,
                     mode_group=args.mode_group)
    c.close()
    del c
    r_ms = max_over_ranks(r["ms"])
    other_form = {"value": world * M * V * K / (r_ms / 1e3), "ms_per_step": r_ms / K,
                  "hop_ms_per_launch": r["prof"]["hop"][0] / max(1, r["prof"]["hop"][1]), "N5": r["charges"]["N5"],
                  "hop_variant": r["hop_variant"], "mode_group": r["mode_group"], "hop_variant_ms": r["hop_variant_ms"]}
    if not args.no_fp64:
        for form in ("plain", "fused"):
            c, r = time_form(wl, "fp64", form, max(2, K // 2), W, device, profile=True, hop_variant=args.hop_variant,
                                 mode_group=args.mode_group)
            c.close()
            del c
            r_ms = max_over_ranks(r["ms"])
            forms[form] = {"value": world * M * V * max(2, K // 2) / (r_ms / 1e3), "ms_per_step": r_ms / max(2, K // 2),
                           "hop_ms_per_launch": r["prof"]["hop"][0] / max(1, r["prof"]["hop"][1]),
                           "N5": r["charges"]["N5"], "hop_variant": r["hop_variant"], "mode_group": r["mode_group"],
                           "hop_variant_ms": r["hop_variant_ms"]}

    ens = None
    if not args.no_ensemble:
        ens = ensemble_leg(max(3, min(K, 20)), 2, device, tile=16 if args.hop_variant == 3 else 0)

    srv = None
    if not args.no_serving:
        srv = serving_leg(args.serving_requests, device, tile=16 if args.hop_variant == 3 else 0,
                          time_box=args.serving_time_box)

    su3 = None
    if not args.no_su3:
        su3 = su3_overlap_leg(args.su3_steps, 1, device, modes=args.modes)

    acc = None
    if args.accuracy_steps > 0 and rank == 0:
        # the FP32 forms run the variant the timed FP32 context chose (its own
        # tuning at the full mode count), so the checks face the timed kernel
        fp32_variant = fp32["hop_variant"] if head == "fp32" else other_form["hop_variant"]
        acc = accuracy(wl, args.accuracy_steps, 50, device, fp32_variant)
        if orc_slice is not None:
            acc["vs_oracle_slice"] = oracle_slice_compare(orc_slice, wl, device, fp32_variant)

    # roofline of the dominant kernel (Wilson fused half step, FP32).  Ungrouped:
    # one event pair per half-step launch, 3 elements per mode-site (read the
    # source, read and write the destination).  Grouped (mode_group > 0): one
    # event pair around a step's launches, whose minimal traffic is 4 elements
    # per mode-site (read psi and psimid, write both: the second half step
    # re-reads the first one's output from L2).
    hop_ms, hop_n = fp32["prof"]["hop"]
    per_launch_ms = hop_ms / max(1, hop_n)
    elem = 8 * 8 if head == "fp32" else 8 * 10  # 2 colours x 4 spins x (8 B [+ 2 extension bytes]) per complex
    n_mb = (M + 31) // 32
    grouped = 0 < fp32["mode_group"] < n_mb
    if grouped:
        alg_bytes = 4 * M * V * elem + 2 * 3 * V * 32
        unit = f"one leapfrog step: both half steps in groups of {fp32['mode_group']} mode blocks"
    else:
        alg_bytes = 3 * M * V * elem + 3 * V * 32
        unit = "one half step (one launch)"
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (per_launch_ms / 1e3) / 1e9
    u1 = "true" if wl.get("nb") else "false"
    kernel = (HOP_KERNELS[fp32["hop_variant"]] if head == "fp32" else "wilson_fp40_kernel<1,LinksF64<{u1}>>").format(u1=u1)
    traffic = committed_traffic(kernel + (" grouped" if grouped else ""))

    if rank == 0:
        total_ms = {k: v[0] for k, v in fp32["prof"].items()}
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": DTYPES[head], "data": "synthetic", "config": config,
            "e2e": {"value": world * M * V * e2e_steps / e2e_secs, "unit": METRIC, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "path": "C ABI, pinned host buffers: ovl_upload_gauge_async (links + E) + ovl_step_observe_async(1) (N_V, N_5, PS read back every step; step k+1 queued before step k's charges are read)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic,
                         "traffic_source": "profiles/traffic.json: ncu DRAM bytes of a 2048-mode capture of this "
                                           "kernel, scaled by the mode count (committed, not measured in this run)",
                         "kernel": kernel + f" ({head} fused half step)",
                         "algorithmic_bytes_per_launch": alg_bytes, "ms_per_launch": per_launch_ms,
                         "unit_of_work": unit,
                         "peak_source": peak_kind},
            "gpu_launches": fp32["launches"],
            "kernel_ms": total_ms,
            "forms": {f"{head}_fused": {"value": value, "ms_per_step": ms / K, "N5": fp32["charges"]["N5"],
                                     "hop_variant": fp32["hop_variant"], "hop_variant_ms": fp32["hop_variant_ms"],
                                     "mode_group": fp32["mode_group"]},
                      f"{other}_fused": other_form,
                      **{f"fp64_{k}": v for k, v in forms.items()}},
            "clocks": clk,
        }
        if "plain" in forms:
            line["headline_vs_fp64_plain"] = value / forms["plain"]["value"]
        if acc is not None:
            line["accuracy_vs_fp64"] = acc
        if ens is not None:
            line["ensemble"] = ens
        if srv is not None:
            line["serving"] = srv
        if su3 is not None:
            line["su3_overlap"] = su3
        if cpu is not None:
            line["cpu_baseline"] = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
        print(json.dumps(line), flush=True)
    if _dist is not None:
        _dist.destroy_process_group()


if __name__ == "__main__":
    main()
