"""Z2 stochastic vacuum modes (ovl_set_stochastic_modes): the vacuum energy of
the free Wilson Hamiltonian, (1/2V) sum_m w_m <psi_m, h psi_m> = (1/2) Tr|h|,
is reproduced exactly by every noise sample (|eta|^2 = 1 per component), so it
must equal the complete plane-wave basis's (FermionField.cpp:145-328) to
rounding; the storage forms agree with FP64 to their rounding; psimid is the
half-step-later state, so the free leapfrog keeps the energy as the plane
waves do."""
import numpy as np
import pytest

from _helpers import rel_err
from overlap_b200 import Context, OvlError
from overlap_b200.inputs import unit_links, volume

pytestmark = pytest.mark.gpu

N = (4, 6, 6)  # even: plane waves of odd N take the reference's axis branch at k = (N-1)/2
KW = dict(N=N, form="fused", m_fermion=0.1, m_dw=0.0, dt=0.05, t_sphaleron=1e9)


def energy(ctx, steps=0):
    ctx.set_links(unit_links(N))
    if steps:
        ctx.step(steps)
    return ctx.fermion_energy()


def test_stochastic_vacuum_energy_is_exact():
    with Context(precision="fp64", **KW) as ctx:  # all 8V plane waves
        assert ctx.set_free_fermions() == 0
        e_pw = energy(ctx)
    for pairs in (1, 7):
        with Context(precision="fp64", n_modes=2 * pairs, **KW) as ctx:
            ctx.set_links(unit_links(N))
            ctx.set_stochastic_modes(seed=11)
            assert abs(ctx.fermion_energy() - e_pw) <= 1e-12 * abs(e_pw)


def test_stochastic_modes_in_every_storage_and_free_evolution():
    out = {}
    for prec in ("fp64", "fp40", "fp32"):
        with Context(precision=prec, n_modes=40, **KW) as ctx:
            ctx.set_links(unit_links(N))
            ctx.set_stochastic_modes(seed=3)
            out[prec] = ctx.get_modes()
            e0 = ctx.fermion_energy()
            ctx.step(20)
            assert abs(ctx.fermion_energy() - e0) <= 1e-3 * abs(e0), prec
    for prec, tol in (("fp40", 2.0 ** -28), ("fp32", 2.0 ** -23)):
        for k in range(2):
            assert rel_err(out[prec][k], out["fp64"][k]) < tol, prec
    psi, mid = out["fp64"]
    # pairs are orthogonal (P+ eta _|_ P- eta) and psimid has the norms of psi
    for r in range(20):
        assert abs(np.vdot(psi[2 * r], psi[2 * r + 1])) < 1e-12
    assert np.allclose(np.sum(np.abs(psi) ** 2, axis=(1, 2, 3)), np.sum(np.abs(mid) ** 2, axis=(1, 2, 3)))


def test_stochastic_modes_need_pairs():
    with Context(precision="fp64", n_modes=7, **KW) as ctx:
        with pytest.raises(OvlError):
            ctx.set_stochastic_modes(seed=1)
        ctx.set_stochastic_modes(seed=1, total_pairs=4)  # a slice of a larger estimate
