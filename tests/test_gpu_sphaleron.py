"""The handmade sphaleron start on the device (ovl_set_handmade_sphaleron)
against the oracle's restatement and the reference's own Setup
(INITIALCONDITIONS/HandmadeSphaleron.cpp:114-170), and the leapfrog from it:
the links reach the final pure gauge when Time() reaches tSphaleron and stay
there.  Tolerances: unit links exact, final links 1e-14, E 1e-13 relative
(the device's arctangent and tangent against the host's, a few ulp)."""
import ctypes as C

import numpy as np
import pytest

from _helpers import oracle_params, rel_err
from _oracle import have_reference, oracle, ptr, reference
from overlap_b200 import Context
from overlap_b200.inputs import volume

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,r,t", [((8, 8, 8), 2.0, 6.0), ((10, 8, 12), 3.0, 4.5), ((7, 9, 6), 1.5, 2.0)])
def test_device_sphaleron_matches_oracle_and_reference(N, r, t):
    V = volume(N)
    p = oracle_params(N)
    oU, oE, oUf, _ = np.zeros(12 * V), np.zeros(9 * V), np.zeros(12 * V), np.zeros(4 * V)
    oracle().orc_handmade_sphaleron(C.byref(p), r, t, ptr(oU), ptr(oE), ptr(oUf), ptr(_))
    with Context(N=N, n_modes=32, precision="fp64", form="fused", m_dw=0.0, dt=0.05, t_sphaleron=t) as ctx:
        Uf = ctx.set_handmade_sphaleron(r, t, final_links=True)
        U, E = ctx.get_links(), ctx.get_efield()
    assert np.array_equal(U.ravel(), oU)
    assert np.max(np.abs(Uf.ravel() - oUf)) < 1e-14
    assert rel_err(E.ravel(), oE) < 1e-13
    if have_reference("wilson"):
        R = reference("wilson")
        R.ovlref_init(*N, 1, 0, 0.1, 1.0, 0.0, t, 0.05, 1.0, 1)
        rUf = np.zeros(12 * V)
        R.ovlref_handmade_sphaleron(r, t, ptr(rUf), None, None)
        rE = np.zeros(9 * V)
        R.ovlref_get_efield(ptr(rE))
        assert np.max(np.abs(Uf.ravel() - rUf)) < 1e-14
        assert rel_err(E.ravel(), rE) < 1e-13


def test_leapfrog_from_the_sphaleron_start_reaches_the_final_links():
    """dt = 0.05, tSphaleron = 2: the links move for 40 steps (Update.cpp:57-60)
    along exp(-i t E) and arrive at G(x) G(x+mu)^+; later steps leave them."""
    N, r, t = (6, 6, 8), 2.0, 2.0
    with Context(N=N, n_modes=32, precision="fp64", form="fused", m_fermion=0.1, m_dw=0.0, dt=0.05,
                 t_sphaleron=t) as ctx:
        Uf = ctx.set_handmade_sphaleron(r, t, final_links=True)
        ctx.set_free_fermions()
        ctx.step(40)
        assert rel_err(ctx.get_links(), Uf) < 1e-12
        ctx.step(5)
        assert rel_err(ctx.get_links(), Uf) < 1e-12
