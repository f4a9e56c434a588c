"""Serving: trajectory requests arrive over time, are admitted as device
memory frees up, and advance together (continuous batching: a request that
arrives while others run joins as soon as memory allows, and a finished one
leaves).  Wilson requests (SU(2) and SU(3)) share one batched ensemble (one
CUDA graph per step for all of them); overlap requests, which the batched
kernels do not cover, run as contexts of their own.  The GPU's time is shared
equally between the running requests: chunks of steps of the ensemble and of
each overlap request are queued back to back, the next chunk going to the
group that has had the least measured GPU time per request.  Each request's
observables -- N_5, N_CS along the cooling-free path (ovl_ncs_update) and the
gauge energy -- are streamed back every `observe_every` steps.

No counterpart in the reference, whose driver runs one trajectory per job
(Simulation.cpp).  All requests of a server share its precision (FP32 or FP64;
overlap requests use the Chebyshev sign function).
"""
from __future__ import annotations

import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from .api import Context, Ensemble, OvlError, Params
from .inputs import random_efield, random_efield_su3, random_links, random_links_su3, u1_flux, volume


@dataclass
class Request:
    """One trajectory: lattice N, modes, physics, steps, inputs by seed."""
    N: tuple
    n_modes: int
    steps: int
    m_fermion: float = 0.05
    dt: float = 0.05
    n_b: int = 0                 # U(1) flux quanta (QED.cpp:62-84); 0: none
    link_sigma: float = 0.3      # seeded random links, exp(i A.sigma/2), A ~ N(0, sigma^2)
    e_sigma: float = 0.1         # seeded random E
    stochastic: bool = True      # Z2 stochastic vacuum modes; False: plane waves (n_modes = 4 Nc V)
    n_colours: int = 2           # 2: SU(2); 3: SU(3)
    fermion: str = "wilson"      # or "overlap" (Chebyshev sign function)
    cheb_degree: int = 64
    m_dw: float = 1.0            # overlap: Wilson kernel mass -m_dw
    seed: int = 0
    observe_every: int = 50
    arrival: float = 0.0         # seconds after the server's start
    # filled by the server
    rid: int = -1
    admitted: float = float("nan")
    finished: float = float("nan")
    gpu_s: float = 0.0           # GPU time of its chunks, a chunk's shared by the requests in it
    observables: list = field(default_factory=list)  # (step, N5, N_CS, energy)
    error: str = ""              # why its set-up failed, if it did

    def mode_sites(self) -> int:
        return self.n_modes * volume(self.N)

    def batchable(self) -> bool:
        """Wilson requests (two or three colours) join the batched ensemble."""
        return self.fermion == "wilson"


def request_cost(req: Request) -> float:
    """GPU work of one step of a request in two-colour Wilson mode-site updates:
    an overlap step is two applications of the Chebyshev series, K + 1 terms of
    seven field passes against the Wilson step's six; three colours carry 1.5x
    the bytes per mode-site."""
    c = float(req.mode_sites())
    if req.fermion == "overlap":
        c *= 2 * (req.cheb_degree + 1) * 7 / 6.0
    return c * (1.5 if req.n_colours == 3 else 1.0)


def request_inputs(r: Request):
    """The request's seeded gauge fields on the host: links, E and the U(1)
    background (None without flux)."""
    if r.n_colours == 3:
        links, efield = random_links_su3(r.N, r.link_sigma, r.seed), random_efield_su3(r.N, r.e_sigma, r.seed + 1)
    else:
        links, efield = random_links(r.N, r.link_sigma, r.seed), random_efield(r.N, r.e_sigma, r.seed + 1)
    return links, efield, (u1_flux(r.N, r.n_b) if r.n_b else None)


def request_bytes(req: Request, precision: str) -> int:
    """Device memory of a request's context: four mode fields (psi, psimid,
    and the two operator buffers; four more for the Chebyshev recurrence of
    overlap requests), links, E and reduction scratch."""
    n_mb = (req.n_modes + 31) // 32
    V = volume(req.N)
    comp = 4 * req.n_colours
    per_complex = {"fp64": 16, "fp32": 8, "fp40": 10}[precision]
    fields = 8 if req.fermion == "overlap" else 4
    links = 3 * V * (144 + 80 + 64) if req.n_colours == 3 else V * (96 + 72 + 48)
    return fields * n_mb * V * comp * 32 * per_complex + links + 64 * V * 8 + (8 << 20)


class Server:
    """Continuous-batching server on one GPU.

    Groups -- the batched ensemble (all Wilson requests) and each overlap
    request -- advance in chunks of steps, one group's chunk after another on
    the GPU.  The next chunk goes to the group with the least GPU time per
    request it carries (fair queueing on the chunks' CUDA-event times, a
    queued chunk counted by its estimate; the ensemble counts its members, a
    group that starts takes the least time of the others).  Up to two chunks
    are queued, the second waiting on the first's end event so that the GPU
    does not wait for the host between them; a group has one chunk queued at
    most.  As a chunk ends the host streams the observables due, retires
    finished requests and admits queued ones.  Wilson requests join or leave
    the ensemble only between its chunks.
    tick_steps: steps of one chunk at most.  A chunk holds about tick_seconds
    of GPU work, estimated from request_cost at rate_wilson two-colour Wilson
    mode-site updates per second, and at least one step (an overlap step on
    24^3 with 8192 modes is about a second); it ends at the next observation
    point or last step of any request it carries.
    memory_bytes: device memory the requests may hold (default: 80 % of the
    free memory at start).
    admission: "fifo" admits queued requests in arrival order and stops at the
    first that does not fit; "shortest" admits, smallest total work
    (request_cost x steps) first, every queued request that fits.
    """

    def __init__(self, precision: str = "fp32", device: int = 0, tick_steps: int = 25,
                 memory_bytes: int | None = None, tile: int = 0, tick_seconds: float = 0.5,
                 rate_wilson: float = 1.2e10, admission: str = "fifo"):
        import torch

        if admission not in ("fifo", "shortest"):
            raise ValueError(f"admission: {admission!r}")
        self.precision = precision
        self.tile = int(tile)  # the ensemble's tile shape (ovl_ensemble_set_tile; 0 = tuned)
        self.device = device
        self.tick_steps = int(tick_steps)
        self.tick_seconds = float(tick_seconds)
        self.rate_wilson = float(rate_wilson)
        self.admission = admission
        if memory_bytes is None:
            free, _ = torch.cuda.mem_get_info(device)
            memory_bytes = int(0.8 * free)
        self.memory_bytes = int(memory_bytes)
        self.ensemble: Ensemble | None = None
        self._ens_stream = None  # the ensemble's torch stream (kept alive with it)
        self.active: list[Request] = []  # in ensemble member order
        self.solo: list[tuple[Request, object]] = []  # requests with contexts of their own
        self.done: list[Request] = []
        self.used_bytes = 0
        self._next_id = 0
        self._phases = {}  # host seconds of the parts of admissions

    # ------------------------------------------------------------ members
    def _params(self, r: Request) -> Params:
        if r.fermion == "overlap":
            return Params(N=tuple(r.N), n_colours=r.n_colours, n_modes=r.n_modes, first_mode=0,
                          precision=self.precision, fermion="overlap", sign_method="chebyshev",
                          cheb_degree=r.cheb_degree, m_fermion=r.m_fermion, r_wilson=1.0, m_dw=r.m_dw, dt=r.dt,
                          t_sphaleron=1e300, device=self.device)
        return Params(N=tuple(r.N), n_colours=r.n_colours, n_modes=r.n_modes, first_mode=0, precision=self.precision,
                      form="fused", m_fermion=r.m_fermion, r_wilson=1.0, m_dw=0.0, dt=r.dt, t_sphaleron=1e300,
                      device=self.device)

    def _admit(self, r: Request, now: float):
        t = [time.perf_counter()]

        def phase(name):  # host time of the admission's parts
            t.append(time.perf_counter())
            self._phases[name] = self._phases.get(name, 0.0) + t[-1] - t[-2]

        p = self._params(r)
        ctx, member = None, None  # the request's context; its index in the ensemble
        try:
            if not r.batchable():
                import torch

                stream = torch.cuda.Stream(self.device)
                p.stream = stream.cuda_stream
                ctx = Context(p)
                ctx.torch_stream = stream  # keeps the stream alive with the context
            elif self.ensemble is None:
                import torch

                self._ens_stream = torch.cuda.Stream(self.device)
                p.stream = self._ens_stream.cuda_stream  # the ensemble runs on the first member's stream
                ensemble = Ensemble([p])
                self.ensemble, member = ensemble, 0
                if self.tile:
                    self.ensemble.set_tile(self.tile)
                ctx = self.ensemble[0]
            else:
                ctx = self.ensemble.add(p)
                member = len(self.ensemble) - 1
            self._setup(r, ctx, now, phase)
        except OvlError:
            # the request leaves no trace: its context (or ensemble member) is released
            if member is not None:
                self.ensemble.remove(member)
            elif ctx is not None:
                ctx.close()
            raise
        if r.batchable():
            self.active.append(r)
        else:
            self.solo.append((r, ctx))
        self.used_bytes += request_bytes(r, self.precision)

    def _setup(self, r: Request, ctx, now: float, phase):
        """The request's fields and first observation on its new context."""
        phase("create_s")
        fut = getattr(r, "_inputs", None)
        links, efield, u1 = fut.result() if fut is not None else request_inputs(r)
        r._inputs = None
        phase("inputs_s")
        ctx.set_links(links)
        ctx.set_efield(efield)
        if u1 is not None:
            ctx.set_u1(u1)
        if r.stochastic and r.fermion == "wilson":  # the Z2 modes are projected with the Wilson h(p)
            ctx.set_stochastic_modes(seed=r.seed + 2)
        else:
            ctx.set_free_fermions()
        phase("fields_s")
        ctx.ncs_update()
        r.admitted = now
        r._step = 0
        r._ncs = 0.0
        self._observe(r, ctx)
        phase("first_observation_s")

    def _observe(self, r: Request, ctx):
        n5 = ctx.charges()["N5"]
        _, ncs = ctx.ncs_update()
        energy = ctx.bulk()["T00"]
        r.observables.append((r._step, n5, ncs, energy))

    def _retire(self, i: int, now: float):
        r = self.active.pop(i)
        self.ensemble.remove(i)
        self._finish(r, now)

    def _retire_solo(self, i: int, now: float):
        r, ctx = self.solo.pop(i)
        ctx.close()
        self._finish(r, now)

    def _finish(self, r: Request, now: float):
        r.finished = now
        self.used_bytes -= request_bytes(r, self.precision)
        self.done.append(r)

    def _chunk_steps(self, group: list) -> int:
        """Steps of the next chunk of a group of requests stepped together."""
        cost = sum(request_cost(r) for r in group)
        k = max(1, min(self.tick_steps, int(self.tick_seconds * self.rate_wilson / max(cost, 1.0))))
        for r in group:
            k = min(k, r.steps - r._step, r.observe_every - r._step % r.observe_every)
        return k

    # ---------------------------------------------------------------- loop
    def serve(self, requests: list[Request], time_box: float | None = None) -> dict:
        """Runs `requests` (arrival times relative to now) to completion, or
        until `time_box` seconds have passed, and returns latency and
        throughput figures.  A request larger than the whole memory budget is
        rejected (finished = NaN, in `rejected`); one whose set-up on the device
        raises (OvlError: out of device memory, say) fails alone (`failed`, the
        message in request.error) and the others go on.  With a time box the figures
        count what finished inside it (and the work of the chunks queued at its
        end); the requests still running, queued or not yet arrived at its end
        are reported as such."""
        import torch

        self.done = []  # figures of this call only
        pending = sorted(requests, key=lambda r: r.arrival)
        for r in pending:  # a request object may be served again: start it afresh
            r.rid = self._next_id
            self._next_id += 1
            r.observables = []
            r.admitted = r.finished = float("nan")
            r.gpu_s = 0.0
            r.error = ""
        queue: list[Request] = []
        rejected = []
        failed = []  # set-up raised: error text in request.error
        inflight = {}  # group key ("ensemble" or a solo rid) -> (start, end, steps, requests)
        vtime = {}  # group key -> GPU seconds per request it carried
        last_end = [None]  # end event of the chunk queued last
        acc = {"work": 0, "cost": 0.0, "gpu_s": 0.0}  # mode-site updates; request_cost units; chunk time
        host = {"admit_s": 0.0, "observe_s": 0.0, "chunks": 0, "idle_polls": 0}  # host time by activity
        self._phases = {}
        t0 = time.perf_counter()

        def clock():
            return time.perf_counter() - t0

        def account(key, start, end, steps, group):
            dt = start.elapsed_time(end) / 1e3
            acc["gpu_s"] += dt
            vtime[key] = vtime.get(key, 0.0) + dt / len(group)
            for r in group:
                r._step += steps
                r.gpu_s += dt / len(group)
                acc["work"] += steps * r.mode_sites()
                acc["cost"] += steps * request_cost(r)

        def fits(q):
            return self.used_bytes + request_bytes(q, self.precision) <= self.memory_bytes

        def start_group(key):  # a group that (re)starts takes the least time of the others
            others = [v for k, v in vtime.items() if k != key]
            vtime[key] = min(others) if others else 0.0

        def queue_chunk(key, stream, run, steps, group):
            if last_end[0] is not None:
                stream.wait_event(last_end[0])  # back to back with the chunk queued before
            start = torch.cuda.Event(enable_timing=True)
            end = torch.cuda.Event(enable_timing=True)
            start.record(stream)
            run(steps)
            end.record(stream)
            last_end[0] = end
            inflight[key] = (start, end, steps, group)
            host["chunks"] += 1

        prep = ThreadPoolExecutor(max_workers=1)
        boxed = False
        try:
            while pending or queue or self.active or self.solo:
                now = clock()
                if time_box is not None and now >= time_box:
                    boxed = True
                    break
                while pending and pending[0].arrival <= now:
                    r = pending.pop(0)
                    if request_bytes(r, self.precision) > self.memory_bytes:
                        rejected.append(r)
                    else:
                        r._inputs = prep.submit(request_inputs, r)  # generated while the GPU works
                        queue.append(r)
                busy = False
                # chunks that ended: account, stream the observables due, retire
                h0 = time.perf_counter()
                if "ensemble" in inflight and inflight["ensemble"][1].query():
                    account("ensemble", *inflight.pop("ensemble"))
                    for i in range(len(self.active) - 1, -1, -1):
                        r = self.active[i]
                        if r._step % r.observe_every == 0 or r._step == r.steps:
                            self._observe(r, self.ensemble[i])
                    for i in range(len(self.active) - 1, -1, -1):
                        if self.active[i]._step >= self.active[i].steps:
                            self._retire(i, clock())
                    if not self.active:
                        vtime.pop("ensemble", None)
                    busy = True
                for i in range(len(self.solo) - 1, -1, -1):
                    r, ctx = self.solo[i]
                    if r.rid in inflight and inflight[r.rid][1].query():
                        account(r.rid, *inflight.pop(r.rid))
                        if r._step % r.observe_every == 0 or r._step == r.steps:
                            self._observe(r, ctx)
                        if r._step >= r.steps:
                            self._retire_solo(i, clock())
                            vtime.pop(r.rid, None)
                        busy = True
                host["observe_s"] += time.perf_counter() - h0
                # admission (into the ensemble only while it has no chunk queued)
                h0 = time.perf_counter()
                admitted = []

                def admit(q):
                    try:
                        self._admit(q, clock())
                        admitted.append(q)
                    except OvlError as e:  # set-up failed (device memory, say): the request fails alone
                        q.error = str(e)
                        failed.append(q)

                if self.admission == "shortest":
                    queue.sort(key=lambda q: request_cost(q) * q.steps)
                    for q in list(queue):
                        if fits(q) and ("ensemble" not in inflight or not q.batchable()):
                            queue.remove(q)
                            admit(q)
                else:
                    while queue and fits(queue[0]) and ("ensemble" not in inflight or not queue[0].batchable()):
                        admit(queue.pop(0))
                for q in admitted:
                    key = "ensemble" if q.batchable() else q.rid
                    if key not in vtime:
                        start_group(key)
                    busy = True
                host["admit_s"] += time.perf_counter() - h0
                # the next chunks: up to two on the GPU, each for the group with the
                # least GPU time per request, counting the estimate of a chunk it
                # has queued; if that group has one queued already, none is added
                while len(inflight) < 2:
                    groups = [("ensemble", None, self.active)] if self.active else []
                    groups += [(r.rid, ctx, [r]) for r, ctx in self.solo]
                    if not groups:
                        break

                    def projected(g):
                        v = vtime.get(g[0], 0.0)
                        if g[0] in inflight:
                            _, _, k, grp = inflight[g[0]]
                            v += k * sum(request_cost(r) for r in grp) / (self.rate_wilson * len(grp))
                        return v

                    key, ctx, grp = min(groups, key=projected)
                    if key in inflight:
                        break
                    if key == "ensemble":
                        queue_chunk(key, self._ens_stream, self.ensemble.step, self._chunk_steps(grp), list(grp))
                    else:
                        queue_chunk(key, ctx.torch_stream, ctx.step, self._chunk_steps(grp), list(grp))
                    busy = True
                if not busy:
                    host["idle_polls"] += 1
                    if self.active or self.solo:
                        time.sleep(0.0005)
                    elif pending:
                        time.sleep(max(0.0, min(0.05, pending[0].arrival - clock())))
        finally:
            prep.shutdown(wait=False, cancel_futures=True)  # also when a step raises
        for r in queue:
            r._inputs = None
        in_flight = len(self.active) + len(self.solo)
        for key, (start, end, k, group) in list(inflight.items()):  # chunks queued at the end of the box still run
            end.synchronize()
            account(key, start, end, k, group)
        wall = clock()
        lat = np.array([r.finished - r.arrival for r in self.done]) if self.done else np.zeros(1)
        wait = np.array([r.admitted - r.arrival for r in self.done]) if self.done else np.zeros(1)
        admitted = [r for r in requests if r.admitted == r.admitted]  # not NaN
        all_wait = np.array([r.admitted - r.arrival for r in admitted]) if admitted else np.zeros(1)
        work, work_cost = acc["work"], acc["cost"]
        return {"requests": len(self.done), "rejected": len(rejected), "failed": len(failed), "wall_s": wall,
                "throughput": work / wall if wall > 0 else 0.0, "unit": "mode-site updates/s",
                "throughput_wilson_equivalent": work_cost / wall if wall > 0 else 0.0,
                "gpu_busy_fraction": acc["gpu_s"] / wall if wall > 0 else 0.0,
                "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
                "queue_wait_p50_s": float(np.percentile(wait, 50)), "queue_wait_p99_s": float(np.percentile(wait, 99)),
                "time_box_s": time_box, "time_boxed": boxed, "in_flight_at_end": in_flight if boxed else 0,
                "queued_at_end": len(queue) if boxed else 0, "not_arrived_at_end": len(pending) if boxed else 0,
                "admitted": len(admitted), "queue_wait_admitted_p50_s": float(np.percentile(all_wait, 50)),
                "queue_wait_admitted_p99_s": float(np.percentile(all_wait, 99)),
                "host": {k: (round(v, 3) if isinstance(v, float) else v) for k, v in host.items()},
                "admission_parts_s": {k: round(v, 3) for k, v in self._phases.items()}}

    def close(self):
        for _, ctx in self.solo:
            ctx.close()
        self.solo = []
        if self.ensemble is not None:
            self.ensemble.close()
            self.ensemble = None
            self._ens_stream = None


def poisson_requests(count: int, rate: float, seed: int, sizes=(8, 12, 16, 24), modes=(4096, 8192),
                     steps=(200, 2000), observe_every: int = 50, su3_fraction: float = 0.0,
                     overlap_fraction: float = 0.0, overlap_sizes=None, overlap_steps=None) -> list[Request]:
    """`count` requests with exponential inter-arrival times (mean 1/rate s),
    N uniform over `sizes`, modes uniform over [modes[0], modes[1]] in pairs,
    steps uniform over [steps[0], steps[1]] in multiples of observe_every,
    U(1) flux n_b uniform over {0, 2, 4, 8}.  A fraction `su3_fraction` are
    SU(3), and a fraction `overlap_fraction` overlap fermions (Chebyshev degree
    64) with N from `overlap_sizes` and steps from `overlap_steps` (by default
    the Wilson requests' distributions; an overlap step costs ~150 Wilson
    steps, request_cost)."""
    overlap_sizes = sizes if overlap_sizes is None else overlap_sizes
    overlap_steps = steps if overlap_steps is None else overlap_steps
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += rng.exponential(1.0 / rate)
        overlap = bool(rng.random() < overlap_fraction)
        nc = 3 if rng.random() < su3_fraction else 2
        n = int(rng.choice(overlap_sizes if overlap else sizes))
        m = int(rng.integers(modes[0] // 64, modes[1] // 64 + 1)) * 64
        lo, hi = overlap_steps if overlap else steps
        s = int(rng.integers(max(1, lo // observe_every), hi // observe_every + 1)) * observe_every
        out.append(Request(N=(n, n, n), n_modes=m, steps=s, n_b=int(rng.choice((0, 2, 4, 8))), n_colours=nc,
                           fermion="overlap" if overlap else "wilson", seed=1000 * i + 17,
                           observe_every=observe_every, arrival=t))
    return out
