"""ovl_ncsdot_noalloc, the allocation-free NCsDot, against the context entry
point and against the oracle.

The allocation-free entry point serves callers that cannot allocate device
memory (a step loop that must not block on an allocation, or memory owned by
another allocator): they pass device inputs and a device output, and the
library's fixed scratch array holds the partial sums.  This file is collected
last so that a failure here comes after every other test has run."""
import numpy as np
import pytest

from _helpers import oracle_params
from _oracle import oracle, ptr
from overlap_b200 import Context, _lib
from overlap_b200.inputs import random_efield, random_links

pytestmark = pytest.mark.gpu


def noalloc_ncsdot(U, E, N, torch):
    dU = torch.from_numpy(np.ascontiguousarray(U)).to("cuda")
    dE = torch.from_numpy(np.ascontiguousarray(E)).to("cuda")
    out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    rc = _lib.lib().ovl_ncsdot_noalloc(dU.data_ptr(), dE.data_ptr(), N[0], N[1], N[2], out.data_ptr(),
                                       stream.cuda_stream)
    assert rc == 0
    torch.cuda.synchronize()
    return float(out.item())


def context_ncsdot(U, E, N):
    with Context(N=N, n_modes=32, precision="fp64", form="fused") as ctx:
        ctx.set_links(U)
        ctx.set_efield(E)
        return ctx.ncsdot()


def oracle_ncsdot(U, E, N):
    import ctypes as C

    p = oracle_params(N)
    return oracle().orc_ncsdot(C.byref(p), ptr(np.ascontiguousarray(U)), ptr(np.ascontiguousarray(E)))


def test_noalloc_ncsdot_matches_context_entry_and_oracle_on_consecutive_calls():
    torch = pytest.importorskip("torch")
    # the second call has a smaller lattice, so stale partial sums of the first
    # call would be read if the entry point did not overwrite what it reads
    for N, seed in (((8, 8, 6), 3), ((5, 4, 6), 4)):
        U = random_links(N, 0.9, seed)
        E = random_efield(N, 0.5, seed + 100)
        got = noalloc_ncsdot(U, E, N, torch)
        want = context_ncsdot(U, E, N)
        orc = oracle_ncsdot(U, E, N)
        assert abs(got - want) <= 1e-13 * max(1.0, abs(want)), (N, got, want)
        assert abs(got - orc) <= 1e-12 * max(1.0, abs(orc)), (N, got, orc)


def test_noalloc_ncsdot_at_its_size_limit():
    # 64^3 sites use all 1024 partial sums of the scratch array
    torch = pytest.importorskip("torch")
    N = (64, 64, 64)
    U = random_links(N, 0.7, 11)
    E = random_efield(N, 0.4, 12)
    got = noalloc_ncsdot(U, E, N, torch)
    want = context_ncsdot(U, E, N)
    assert abs(got - want) <= 1e-12 * max(1.0, abs(want)), (got, want)
    # and a small lattice right after, on the same array
    n2 = (4, 5, 6)
    U2 = random_links(n2, 0.8, 13)
    E2 = random_efield(n2, 0.3, 14)
    got2 = noalloc_ncsdot(U2, E2, n2, torch)
    orc2 = oracle_ncsdot(U2, E2, n2)
    assert abs(got2 - orc2) <= 1e-12 * max(1.0, abs(orc2)), (got2, orc2)


def test_noalloc_rejects_lattices_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    assert _lib.lib().ovl_ncsdot_noalloc(p, p, 65, 64, 64, p, 0) == 1  # OVL_E_ARG
