"""The serving scheduler's host logic (overlap_b200.serve.Server) on the CPU,
with the contexts, the ensemble, the CUDA streams and events replaced by a
simulated serial device: a chunk of k steps of a group occupies it for k
times the group's step time (its requests' request_cost at a fixed rate), in
the order the chunks are queued.  Checks what the scheduler promises: equal
GPU time per running request, chunks that end at observation points and last
steps, the time box's accounting, admission in arrival order or smallest
first, and a request whose set-up fails failing alone."""
import time

import numpy as np
import pytest

import overlap_b200.serve as serve
from overlap_b200.api import OvlError
from overlap_b200.serve import Request, Server, request_bytes, request_cost

RATE = 2e9  # simulated mode-site updates per second


class SimDevice:
    def __init__(self):
        self.t0 = time.perf_counter()
        self.busy_until = 0.0

    def now(self):
        return time.perf_counter() - self.t0

    def run(self, seconds):
        self.busy_until = max(self.now(), self.busy_until) + seconds


DEV = {}


class SimEvent:
    def __init__(self, enable_timing=False):
        self.t = None

    def record(self, stream=None):
        self.t = max(DEV["gpu"].now(), DEV["gpu"].busy_until)

    def query(self):
        return DEV["gpu"].now() >= self.t

    def synchronize(self):
        while not self.query():
            time.sleep(0.0005)

    def elapsed_time(self, end):
        return 1e3 * (end.t - self.t)


class SimStream:
    def __init__(self, device=None, priority=0):
        self.cuda_stream = id(self)

    def wait_event(self, ev):
        pass  # one serial device


class SimContext:
    def __init__(self, p):
        if min(p.N) < 3:
            raise OvlError(1, f"ovl_create: N[0]={p.N[0]} outside [3, 1024]")
        self.p = p
        self.closed = False

    def step_seconds(self):
        r = Request(N=self.p.N, n_modes=self.p.n_modes, steps=1, n_colours=self.p.n_colours, fermion=self.p.fermion,
                    cheb_degree=self.p.cheb_degree)
        return request_cost(r) / RATE

    def step(self, k):
        DEV["gpu"].run(k * self.step_seconds())

    def set_links(self, U): pass
    def set_efield(self, E): pass
    def set_u1(self, u): pass
    def set_stochastic_modes(self, seed=0): pass
    def set_free_fermions(self): return 0
    def ncs_update(self): return 0.0, 0.0
    def charges(self): return {"N5": 0.0}
    def bulk(self): return {"T00": 0.0}

    def close(self):
        self.closed = True


class SimEnsemble:
    def __init__(self, params):
        self.members = [SimContext(p) for p in params]

    def __len__(self):
        return len(self.members)

    def __getitem__(self, i):
        return self.members[i]

    def add(self, p):
        c = SimContext(p)
        self.members.append(c)
        return c

    def remove(self, i):
        del self.members[i]

    def set_tile(self, t): pass

    def step(self, k):
        DEV["gpu"].run(k * sum(m.step_seconds() for m in self.members))

    def close(self): pass


@pytest.fixture
def sim(monkeypatch):
    import torch

    DEV["gpu"] = SimDevice()
    monkeypatch.setattr(serve, "Context", SimContext)
    monkeypatch.setattr(serve, "Ensemble", SimEnsemble)
    monkeypatch.setattr(torch.cuda, "Stream", SimStream)
    monkeypatch.setattr(torch.cuda, "Event", SimEvent)
    monkeypatch.setattr(serve, "request_inputs", lambda r: (None, None, None))
    return DEV["gpu"]


def req(i, N, modes, steps, arrival=0.0, **kw):
    return Request(N=N, n_modes=modes, steps=steps, seed=i, observe_every=10, arrival=arrival, **kw)


def server(**kw):
    kw.setdefault("memory_bytes", 1 << 40)
    return Server(precision="fp32", rate_wilson=RATE, tick_seconds=0.01, tick_steps=10, **kw)


def test_running_requests_get_equal_gpu_time(sim):
    reqs = [req(0, (16, 16, 16), 256, 10 ** 6), req(1, (8, 8, 8), 128, 10 ** 6),
            req(2, (8, 8, 8), 64, 10 ** 6, fermion="overlap", cheb_degree=16)]
    m = server().serve(reqs, time_box=1.0)
    g = np.array([r.gpu_s for r in reqs])
    assert m["in_flight_at_end"] == 3 and g.min() > 0
    assert g.max() < 1.3 * g.min(), g
    assert abs(g[0] - g[1]) < 1e-9  # the ensemble's chunk time is split between its members
    # each chunk ends at an observation point: every streamed step is a multiple of observe_every
    for r in reqs:
        assert all(s % 10 == 0 for s, *_ in r.observables) and len(r.observables) >= 2


def test_time_box_and_admission_policies(sim):
    big = lambda i, t: req(i, (16, 16, 16), 512, 10 ** 6, t)
    small = lambda i, t: req(i, (4, 4, 4), 32, 30, t)
    budget = request_bytes(big(0, 0), "fp32") + request_bytes(small(0, 0), "fp32")
    out = {}
    for adm in ("fifo", "shortest"):
        reqs = [big(0, 0.0), big(1, 0.0), small(2, 0.01), small(3, 3600.0)]
        out[adm] = (server(memory_bytes=budget, admission=adm).serve(reqs, time_box=0.5), reqs)
    m, reqs = out["fifo"]
    assert m["time_boxed"] and m["requests"] == 0 and m["in_flight_at_end"] == 1
    assert m["queued_at_end"] == 2 and m["not_arrived_at_end"] == 1 and m["admitted"] == 1
    m, reqs = out["shortest"]
    assert m["requests"] == 1 and m["queued_at_end"] == 1 and m["admitted"] == 2
    assert reqs[2].observables[-1][0] == 30  # the last step observed
    assert m["latency_p50_s"] < 0.5 and m["queue_wait_p50_s"] < 0.1


def test_failed_setup_fails_alone(sim):
    reqs = [req(0, (4, 4, 4), 32, 20), req(1, (2, 2, 2), 32, 20, 0.01),
            req(2, (2, 2, 2), 32, 20, 0.01, fermion="overlap", cheb_degree=8), req(3, (4, 4, 6), 32, 20, 0.02)]
    m = server().serve(reqs)
    assert m["requests"] == 2 and m["failed"] == 2
    assert "N[0]=2" in reqs[1].error and "N[0]=2" in reqs[2].error
    assert [len(r.observables) for r in (reqs[0], reqs[3])] == [3, 3]  # steps 0, 10, 20
