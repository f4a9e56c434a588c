"""The handmade sphaleron initial condition (INITIALCONDITIONS/HandmadeSphaleron.cpp,
the production driver's gauge start, Simulation.cpp:580): the oracle's
restatement against the reference's own Setup run in the reference build.

The reference's gauge transformation of the links uses a macro of the missing
CALC/GaugeTransformation.cpp, restated in oracle/ref/ovl_calc_macros.h as
U' = G(x) U G(x+mu)^+.  That convention is checked by the reference's own
topology estimators: the vacuum N_CS of the final links
(ChernSimonsNumber::VacuumEstimator::NCS) equals the integral winding estimate
of G (WindingNumber::IntegralEstimate::Measure), which reads G alone."""
import ctypes as C

import numpy as np
import pytest

from _helpers import oracle_params
from _oracle import have_reference, oracle, ptr, reference
from overlap_b200.inputs import volume

CASES = [((8, 8, 8), 2.0, 6.0), ((10, 8, 12), 3.0, 4.5), ((7, 9, 6), 1.5, 2.0)]


def oracle_sphaleron(N, r, t):
    V = volume(N)
    p = oracle_params(N)
    U, E, Uf, G = np.zeros(12 * V), np.zeros(9 * V), np.zeros(12 * V), np.zeros(4 * V)
    oracle().orc_handmade_sphaleron(C.byref(p), r, t, ptr(U), ptr(E), ptr(Uf), ptr(G))
    return U, E, Uf, G


@pytest.mark.skipif(not have_reference("wilson"), reason="reference library not built")
@pytest.mark.parametrize("N,r,t", CASES)
def test_oracle_sphaleron_equals_the_reference_setup(N, r, t):
    V = volume(N)
    R = reference("wilson")
    R.ovlref_init(*N, 1, 0, 0.1, 1.0, 0.0, t, 0.05, 1.0, 1)
    rUf, rG, out4 = np.zeros(12 * V), np.zeros(4 * V), np.zeros(4)
    R.ovlref_handmade_sphaleron(r, t, ptr(rUf), ptr(rG), ptr(out4))
    rU, rE = np.zeros(12 * V), np.zeros(9 * V)
    R.ovlref_get_links(ptr(rU))
    R.ovlref_get_efield(ptr(rE))
    U, E, Uf, G = oracle_sphaleron(N, r, t)
    assert np.array_equal(U, rU)  # unit links
    assert np.max(np.abs(G - rG)) < 1e-14
    assert np.max(np.abs(Uf - rUf)) < 1e-14
    assert np.max(np.abs(E - rE)) < 1e-13 * max(1.0, np.max(np.abs(rE)))
    assert np.max(np.abs(E)) > 0.05  # a non-trivial field
    # the restated link transformation against the reference's topology estimators
    assert abs(out4[3] - out4[1]) < 1e-12, out4
    assert abs(out4[2]) < 1e-14


def test_sphaleron_field_carries_the_links_to_the_final_links():
    """exp(-i t E) applied to the unit links for the transition time gives the
    final links (Update.cpp's link update run for tSphaleron in one step)."""
    N, r, t = (6, 6, 8), 2.0, 3.0
    U, E, Uf, _ = oracle_sphaleron(N, r, t)
    p = oracle_params(N)
    oracle().orc_update_links(C.byref(p), ptr(U), ptr(E), t)
    assert np.max(np.abs(U - Uf)) < 1e-13
