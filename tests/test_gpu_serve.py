"""Continuous-batching server (overlap_b200.serve): a request's streamed
observables are the same whether it runs alone or joins a running batch of
others, also when the memory budget serialises the requests.  The batched
kernels do per member the arithmetic of a batch of one; the autotuned tile
shape selects one of two compiled kernels, which may contract multiply-adds
differently, so results agree to rounding: 1e-12 (FP64) and 1e-5 (FP32) of
each observable's scale."""
import numpy as np
import pytest

from overlap_b200.serve import Request, Server, request_bytes

pytestmark = pytest.mark.gpu


def req(i, N, modes, steps, arrival, n_b=0, **kw):
    return Request(N=N, n_modes=modes, steps=steps, n_b=n_b, seed=100 + 7 * i, observe_every=10, arrival=arrival, **kw)


def same(a, b, precision):
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert a.shape == b.shape
    scale = np.maximum(np.max(np.abs(b), axis=0), 1e-30)
    return bool(np.all(np.abs(a - b) <= tol * scale))


def serve(reqs, **kw):
    s = Server(**kw)
    try:
        metrics = s.serve(reqs)
        return {r.seed: np.array(r.observables) for r in s.done}, metrics
    finally:
        s.close()


@pytest.mark.parametrize("precision,tile", [("fp32", 0), ("fp64", 0), ("fp32", 16)])
def test_request_results_are_the_same_alone_and_in_the_mix(precision, tile):
    a = lambda arrival: req(0, (4, 5, 6), 64, 60, arrival, n_b=2)
    alone, _ = serve([a(0.0)], precision=precision, tick_steps=7, tile=tile)
    mix = [req(1, (6, 6, 6), 96, 80, 0.0), a(0.05), req(2, (5, 4, 4), 32, 40, 0.08, n_b=4)]
    mixed, m = serve(mix, precision=precision, tick_steps=7, tile=tile)
    assert m["requests"] == 3 and m["rejected"] == 0
    assert m["latency_p50_s"] <= m["latency_p99_s"] and m["throughput"] > 0
    ref = alone[a(0).seed]
    assert ref.shape == (7, 4)  # steps 0, 10, ..., 60
    assert same(mixed[a(0).seed], ref, precision)
    # one request at a time: the budget admits the next only after the previous leaves
    budget = max(request_bytes(r, precision) for r in mix)
    serial, m2 = serve(mix, precision=precision, tick_steps=7, memory_bytes=budget, tile=tile)
    for seed, obs in mixed.items():
        assert same(serial[seed], obs, precision)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_su3_and_overlap_requests_alongside_the_batch(precision):
    """SU(3) Wilson requests join the batched ensemble beside SU(2) ones, and
    overlap requests run as contexts of their own next to it: each result is
    the same alone and in the mix."""
    mk = [lambda t: req(3, (4, 4, 6), 64, 30, t, n_colours=3),
          lambda t: req(4, (4, 4, 4), 64, 20, t, fermion="overlap", cheb_degree=16, n_b=2),
          lambda t: req(5, (4, 4, 4), 64, 20, t, fermion="overlap", cheb_degree=16, n_colours=3)]
    alone = {}
    for f in mk:
        out, m = serve([f(0.0)], precision=precision, tick_steps=7)
        assert m["requests"] == 1
        alone.update(out)
    mix = [req(1, (6, 6, 6), 96, 40, 0.0)] + [f(0.02 * (i + 1)) for i, f in enumerate(mk)]
    mixed, m = serve(mix, precision=precision, tick_steps=7)
    assert m["requests"] == 4 and m["rejected"] == 0
    for f in mk:
        seed = f(0).seed
        assert mixed[seed].shape == alone[seed].shape
        assert same(mixed[seed], alone[seed], precision), seed


def test_time_box_accounts_for_every_request():
    """A time-boxed serve stops at the box: requests that finished inside it
    are counted with their latency, the ones still running, queued or not yet
    arrived are reported as such, and the server closes cleanly with work in
    flight."""
    import time

    reqs = [req(0, (4, 4, 4), 32, 20, 0.0),                  # finishes early
            req(1, (8, 8, 8), 256, 10 ** 6, 0.0),            # runs past the box
            req(2, (8, 8, 8), 256, 10 ** 6, 0.0),            # waits for memory: queued
            req(3, (4, 4, 4), 32, 20, 3600.0)]               # arrives after the box
    budget = request_bytes(reqs[0], "fp32") + request_bytes(reqs[1], "fp32")
    s = Server(precision="fp32", tick_steps=10, memory_bytes=budget)
    try:
        t0 = time.perf_counter()
        m = s.serve(reqs, time_box=2.0)
        wall = time.perf_counter() - t0
        assert m["time_boxed"] and 2.0 <= m["wall_s"] <= wall < 30.0
        assert m["requests"] == 1 and [r.seed for r in s.done] == [reqs[0].seed]
        assert m["in_flight_at_end"] == 1 and m["queued_at_end"] == 1 and m["not_arrived_at_end"] == 1
        assert m["admitted"] == 2 and m["rejected"] == 0
        assert m["throughput"] > 0 and m["throughput_wilson_equivalent"] == m["throughput"]
        assert len(reqs[1].observables) >= 2  # streamed while it ran
    finally:
        s.close()


def test_shortest_first_admission_backfills_past_a_large_request():
    """In arrival order a small request waits behind a large one that does not
    fit; admitted smallest first it runs beside the request already on the
    GPU and finishes inside the box."""
    reqs = lambda: [req(1, (8, 8, 8), 256, 10 ** 6, 0.0),   # runs past the box
                    req(2, (8, 8, 8), 256, 10 ** 6, 0.0),   # does not fit beside it
                    req(0, (4, 4, 4), 32, 20, 0.01)]        # fits beside it
    budget = request_bytes(reqs()[0], "fp32") + request_bytes(reqs()[2], "fp32")
    out = {}
    for admission in ("fifo", "shortest"):
        s = Server(precision="fp32", tick_steps=10, memory_bytes=budget, admission=admission)
        try:
            out[admission] = s.serve(reqs(), time_box=2.0)
        finally:
            s.close()
    assert out["fifo"]["requests"] == 0 and out["fifo"]["queued_at_end"] == 2
    assert out["shortest"]["requests"] == 1 and out["shortest"]["queued_at_end"] == 1
    assert out["shortest"]["admitted"] == 2


def test_running_requests_share_the_gpu_time_equally():
    """The GPU's time goes to the running requests in equal shares: two Wilson
    requests in the batched ensemble and an overlap request of its own, all
    running through the box, each get about a third of the chunks' time (the
    ensemble's chunk time split between its members)."""
    reqs = [req(0, (8, 8, 8), 256, 10 ** 6, 0.0), req(1, (6, 6, 6), 128, 10 ** 6, 0.0),
            req(2, (4, 4, 4), 64, 10 ** 6, 0.0, fermion="overlap", cheb_degree=16)]
    s = Server(precision="fp32", tick_steps=10, tick_seconds=0.05)
    try:
        m = s.serve(reqs, time_box=4.0)
    finally:
        s.close()
    assert m["in_flight_at_end"] == 3 and m["requests"] == 0
    g = np.array([r.gpu_s for r in reqs])
    assert g.min() > 0 and g.max() < 2.0 * g.min(), g
    assert abs(g[0] - g[1]) < 1e-9 * g[0]  # one chunk time, split between the members
    assert 0.0 < m["gpu_busy_fraction"] <= 1.05


@pytest.mark.parametrize("fermion", ["wilson", "overlap"])
def test_a_request_whose_setup_fails_fails_alone(fermion):
    """A request the library refuses at set-up (here a 2^3 lattice, below the
    contexts' minimum extent) is reported as failed with the library's message;
    the ensemble or the server goes on, and the other requests' results are
    those they have alone."""
    kw = dict(fermion="overlap", cheb_degree=16) if fermion == "overlap" else {}
    good = lambda t: req(8, (4, 4, 4), 64, 20, t, **kw)
    bad = req(9, (2, 2, 2), 64, 20, 0.01, **kw)
    alone, _ = serve([good(0.0)], precision="fp64", tick_steps=7)
    mixed, m = serve([good(0.0), bad, req(10, (4, 4, 6), 32, 20, 0.02)], precision="fp64", tick_steps=7)
    assert m["requests"] == 2 and m["failed"] == 1 and "N[0]=2" in bad.error
    assert same(mixed[good(0).seed], alone[good(0).seed], "fp64")
