"""Asynchronous step loop (ovl_upload_gauge_async, ovl_step_observe_async):
the same kernels in the same order as the synchronous calls, so a loop that
queues step k+1 before reading step k's charges gives bit for bit the charges
of the synchronous loop; buffers that are not page-locked are refused."""
import numpy as np
import pytest
import torch

from overlap_b200 import Context, OvlError
from overlap_b200.inputs import random_efield, random_links, u1_flux, volume

pytestmark = pytest.mark.gpu

N = (6, 4, 5)


def pinned(shape):
    return torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()


def make(hop_variant, U, E):
    s = torch.cuda.Stream()
    ctx = Context(N=N, n_modes=96, precision="fp32", form="fused", m_fermion=0.1, dt=0.05, hop_variant=hop_variant,
                  stream=s.cuda_stream)
    ctx.torch_stream = s
    ctx.set_links(U)
    ctx.set_efield(E)
    ctx.set_u1(u1_flux(N, 2))
    ctx.set_free_fermions()
    return ctx


@pytest.mark.parametrize("hop_variant", [0, 3])
def test_async_loop_gives_the_synchronous_charges(hop_variant):
    V = volume(N)
    Us = [random_links(N, 0.4, 10 + k) for k in range(6)]  # a new upload every step
    E = random_efield(N, 0.2, 3)
    with make(hop_variant, Us[0], E) as a:
        want = []
        for U in Us:
            a.set_links(U)
            a.set_efield(E)
            ch = a.step_observe(1)
            want.append([ch["NV"], ch["N5"], ch["PS"]])
        links_a = a.get_links()
    bufs = [pinned((V, 3, 4)) for _ in range(2)]
    Ep = pinned((V, 3, 3))
    Ep[...] = E
    outs = [pinned(3) for _ in range(2)]
    done = [torch.cuda.Event(), torch.cuda.Event()]
    got = []
    with make(hop_variant, Us[0], E) as b:
        for k, U in enumerate(Us):
            if k >= 2:
                done[k % 2].synchronize()  # the step that read bufs[k % 2] is done
            bufs[k % 2][...] = U
            b.upload_gauge_async(bufs[k % 2], Ep)
            b.step_observe_async(1, outs[k % 2])
            done[k % 2].record(b.torch_stream)
            if k > 0:
                done[(k - 1) % 2].synchronize()
                got.append(outs[(k - 1) % 2].tolist())
        b.synchronize()
        got.append(outs[(len(Us) - 1) % 2].tolist())
        assert np.array_equal(b.get_links(), links_a)
    assert np.array_equal(np.array(got), np.array(want))


def test_async_calls_need_page_locked_buffers():
    V = volume(N)
    U, E = random_links(N, 0.4, 1), random_efield(N, 0.2, 2)
    with make(0, U, E) as ctx:
        with pytest.raises(OvlError, match="page-locked"):
            ctx.upload_gauge_async(np.ascontiguousarray(U), None)
        with pytest.raises(OvlError, match="page-locked"):
            ctx.step_observe_async(1, np.zeros(3))
        with pytest.raises(ValueError):
            ctx.upload_gauge_async(pinned((V, 3, 4))[:, :2], None)  # not contiguous: would need a copy
        out = pinned(3)
        ctx.step_observe_async(1, out)
        ctx.synchronize()
        assert np.all(np.isfinite(out))
