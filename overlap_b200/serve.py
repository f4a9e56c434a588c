"""Serving: trajectory requests arrive over time, are admitted as device
memory frees up, and advance together (continuous batching: a request that
arrives while others run joins at the next tick, and a finished one leaves).
Wilson requests (SU(2) and SU(3)) share one batched ensemble (one CUDA graph
per step for all of them); overlap requests, which the batched kernels do not
cover, run as contexts of their own on their own streams, stepped in the same
ticks so their kernels overlap the ensemble's on the GPU.  Each request's
observables -- N_5, N_CS along the cooling-free path (ovl_ncs_update) and the
gauge energy -- are streamed back every `observe_every` steps.

No counterpart in the reference, whose driver runs one trajectory per job
(Simulation.cpp).  All requests of a server share its precision (FP32 or FP64;
overlap requests use the Chebyshev sign function).
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from .api import Context, Ensemble, Params
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
    observables: list = field(default_factory=list)  # (step, N5, N_CS, energy)

    def mode_sites(self) -> int:
        return self.n_modes * volume(self.N)

    def batchable(self) -> bool:
        """Wilson requests (two or three colours) join the batched ensemble."""
        return self.fermion == "wilson"


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

    tick_steps: steps between admission rounds (shortened so that no request
    passes an observation point or its last step inside a tick).
    memory_bytes: device memory the requests may hold (default: 80 % of the
    free memory at start).
    """

    def __init__(self, precision: str = "fp32", device: int = 0, tick_steps: int = 25,
                 memory_bytes: int | None = None, tile: int = 0):
        import torch

        self.precision = precision
        self.tile = int(tile)  # the ensemble's tile shape (ovl_ensemble_set_tile; 0 = tuned)
        self.device = device
        self.tick_steps = int(tick_steps)
        if memory_bytes is None:
            free, _ = torch.cuda.mem_get_info(device)
            memory_bytes = int(0.8 * free)
        self.memory_bytes = int(memory_bytes)
        self.ensemble: Ensemble | None = None
        self.active: list[Request] = []  # in ensemble member order
        self.solo: list[tuple[Request, object]] = []  # requests with contexts of their own
        self.done: list[Request] = []
        self.used_bytes = 0
        self._next_id = 0

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
        p = self._params(r)
        if not r.batchable():
            import torch

            stream = torch.cuda.Stream(self.device)
            p.stream = stream.cuda_stream
            ctx = Context(p)
            ctx.torch_stream = stream  # keeps the stream alive with the context
        elif self.ensemble is None:
            self.ensemble = Ensemble([p])
            if self.tile:
                self.ensemble.set_tile(self.tile)
            ctx = self.ensemble[0]
        else:
            ctx = self.ensemble.add(p)
        if r.n_colours == 3:
            ctx.set_links(random_links_su3(r.N, r.link_sigma, r.seed))
            ctx.set_efield(random_efield_su3(r.N, r.e_sigma, r.seed + 1))
        else:
            ctx.set_links(random_links(r.N, r.link_sigma, r.seed))
            ctx.set_efield(random_efield(r.N, r.e_sigma, r.seed + 1))
        if r.n_b:
            ctx.set_u1(u1_flux(r.N, r.n_b))
        if r.stochastic and r.fermion == "wilson":  # the Z2 modes are projected with the Wilson h(p)
            ctx.set_stochastic_modes(seed=r.seed + 2)
        else:
            ctx.set_free_fermions()
        ctx.ncs_update()
        r.admitted = now
        r._step = 0
        r._ncs = 0.0
        self._observe(r, ctx)
        if r.batchable():
            self.active.append(r)
        else:
            self.solo.append((r, ctx))
        self.used_bytes += request_bytes(r, self.precision)

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

    # ---------------------------------------------------------------- loop
    def serve(self, requests: list[Request]) -> dict:
        """Runs `requests` (arrival times relative to now) to completion and
        returns latency and throughput figures.  A request larger than the
        whole memory budget is rejected (finished = NaN, in `rejected`)."""
        self.done = []  # figures of this call only
        pending = sorted(requests, key=lambda r: r.arrival)
        for r in pending:  # a request object may be served again: start it afresh
            r.rid = self._next_id
            self._next_id += 1
            r.observables = []
            r.admitted = r.finished = float("nan")
        queue: list[Request] = []
        rejected = []
        t0 = time.perf_counter()
        work = 0
        while pending or queue or self.active or self.solo:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now:
                r = pending.pop(0)
                if request_bytes(r, self.precision) > self.memory_bytes:
                    rejected.append(r)
                else:
                    queue.append(r)
            while queue and self.used_bytes + request_bytes(queue[0], self.precision) <= self.memory_bytes:
                self._admit(queue.pop(0), time.perf_counter() - t0)
            if not self.active and not self.solo:
                if pending:
                    time.sleep(max(0.0, min(0.05, pending[0].arrival - (time.perf_counter() - t0))))
                continue
            # a tick: as many steps as no active request passes an observation or its end
            running = self.active + [r for r, _ in self.solo]
            k = self.tick_steps
            for r in running:
                k = min(k, r.steps - r._step, r.observe_every - r._step % r.observe_every)
            if self.active:
                self.ensemble.step(k)
            for _, ctx in self.solo:  # queued on their own streams, beside the ensemble's graph
                ctx.step(k)
            for r in running:
                r._step += k
                work += k * r.mode_sites()
            for i in range(len(self.active) - 1, -1, -1):
                r = self.active[i]
                if r._step % r.observe_every == 0 or r._step == r.steps:
                    self._observe(r, self.ensemble[i])
            for r, ctx in self.solo:
                if r._step % r.observe_every == 0 or r._step == r.steps:
                    self._observe(r, ctx)
            now = time.perf_counter() - t0
            for i in range(len(self.active) - 1, -1, -1):
                if self.active[i]._step >= self.active[i].steps:
                    self._retire(i, now)
            for i in range(len(self.solo) - 1, -1, -1):
                if self.solo[i][0]._step >= self.solo[i][0].steps:
                    self._retire_solo(i, now)
        wall = time.perf_counter() - t0
        lat = np.array([r.finished - r.arrival for r in self.done]) if self.done else np.zeros(1)
        wait = np.array([r.admitted - r.arrival for r in self.done]) if self.done else np.zeros(1)
        return {"requests": len(self.done), "rejected": len(rejected), "wall_s": wall,
                "throughput": work / wall if wall > 0 else 0.0, "unit": "mode-site updates/s",
                "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
                "queue_wait_p50_s": float(np.percentile(wait, 50)), "queue_wait_p99_s": float(np.percentile(wait, 99))}

    def close(self):
        for _, ctx in self.solo:
            ctx.close()
        self.solo = []
        if self.ensemble is not None:
            self.ensemble.close()
            self.ensemble = None


def poisson_requests(count: int, rate: float, seed: int, sizes=(8, 12, 16, 24), modes=(4096, 8192),
                     steps=(200, 2000), observe_every: int = 50, su3_fraction: float = 0.0,
                     overlap_fraction: float = 0.0, overlap_sizes=(8,), overlap_steps=(100, 200)) -> list[Request]:
    """`count` requests with exponential inter-arrival times (mean 1/rate s),
    N uniform over `sizes`, modes uniform over [modes[0], modes[1]] in pairs,
    steps uniform over [steps[0], steps[1]] in multiples of observe_every,
    U(1) flux n_b uniform over {0, 2, 4, 8}.  A fraction `su3_fraction` are
    SU(3), and a fraction `overlap_fraction` overlap fermions (Chebyshev degree
    64) with N from `overlap_sizes` and steps from `overlap_steps` (an overlap
    step costs ~130 Wilson steps)."""
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
