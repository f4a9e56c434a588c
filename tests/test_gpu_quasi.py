"""Quasi-particle gauge fields on the device (ovl_set_quasi_particles,
InitialConditions::SetQuasiParticles of INITIALCONDITIONS/SetQuasiParticles.cpp)
against the host restatement with the same counter-based amplitudes
(overlap_b200.inputs.quasi_particles, generator "counter"), two and three
colours: links and E to 1e-12 of their largest element (the device's
transcendental functions and the transform's summation order against numpy's);
then Gauss's law restored on the device as the reference does."""
import numpy as np
import pytest

from _helpers import rel_err
from overlap_b200 import Context
from overlap_b200.inputs import quasi_particles, su3_unpack

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nc", [2, 3])
@pytest.mark.parametrize("N", [(6, 8, 5), (8, 8, 8)])
def test_device_quasi_particles_equal_the_host_restatement(nc, N):
    n0, qs, seed = 4.0, 1.0, 20261203
    hU, hE = quasi_particles(N, n0, qs, seed, n_colours=nc, generator="counter")
    with Context(N=N, n_colours=nc, n_modes=32, precision="fp64", form="fused", m_dw=0.0, dt=0.05) as ctx:
        assert ctx.set_quasi_particles(n0, qs, seed, gauss_max_iter=0) == 0
        U, E = ctx.get_links(), ctx.get_efield()
    if nc == 3:
        U, hU = su3_unpack(U), su3_unpack(hU)
    assert rel_err(U, hU) < 1e-12
    assert rel_err(E, hE) < 1e-12


@pytest.mark.parametrize("nc", [2, 3])
def test_device_quasi_particles_with_gauss_law_restored(nc):
    N = (8, 6, 10)
    with Context(N=N, n_colours=nc, n_modes=32, precision="fp64", form="fused", m_dw=0.0, dt=0.05) as ctx:
        it = ctx.set_quasi_particles(4.0, 1.0, 7)
        b = ctx.bulk()
        assert it > 0 and abs(b["gauss_max"]) < 1e-13
        assert b["unitarity_max"] < 1e-13
        assert b["electric"] > 0.0
