"""The reference's own build with include/ovl_dropin.hpp in place of its
fermion hot path and include/ovl_dropin_gauge.hpp in place of its gauge
routines (tests/dropin/dropin_main.cpp) produces the reference's results:
modes, links and current arrays agree with the reference compiled from source,
and NCsDot, UpdateElectricFields and UpdateGaugeLinks agree with the
reference's own definitions run in the same process on the same fields.

Wilson build: 1e-12 (the plain form's bar).  Overlap build: the drop-in takes
its spectral bounds from the GPU's Ritz solver started from its own generator,
the reference from its RNG; the bounds agree to round-off and the evolution to
1e-10."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from _helpers import current_scale, rel_err
from _oracle import have_reference, ptr, reference
from overlap_b200.inputs import random_efield, random_links, volume

pytestmark = pytest.mark.gpu

BUILD = Path(__file__).resolve().parent / "dropin" / "_build"


def run_program(tmp_path, binary, N, nranks, rank, m, r, mdw, tsph, dt, steps, U, E, n_currents):
    V = volume(N)
    inp = tmp_path / "in.bin"
    out = tmp_path / "out.bin"
    np.concatenate([U.ravel(), E.ravel()]).tofile(inp)
    res = subprocess.run([str(binary), *map(str, N), str(nranks), str(rank), str(m), str(r), str(mdw), str(tsph),
                          str(dt), str(steps), str(inp), str(out)], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr
    first, nm = map(int, res.stdout.split()[-2:])
    data = np.fromfile(out, dtype=np.float64)
    k = nm * V * 16
    o = {"first": first, "nm": nm}
    o["psi"] = data[:k].view(np.complex128).reshape(nm, V, 2, 4)
    o["mid"] = data[k:2 * k].view(np.complex128).reshape(nm, V, 2, 4)
    pos = 2 * k
    o["links"] = data[pos:pos + 12 * V]
    pos += 12 * V
    o["cur"] = data[pos:pos + n_currents]
    pos += n_currents
    o["ncs"] = data[pos:pos + 2]
    pos += 2
    o["E_gpu"], o["E_ref"] = data[pos:pos + 9 * V], data[pos + 9 * V:pos + 18 * V]
    pos += 18 * V
    o["U_gpu"], o["U_ref"] = data[pos:pos + 12 * V], data[pos + 12 * V:pos + 24 * V]
    assert pos + 24 * V == data.size
    return o


def check_gauge_routines(o):
    ncs_gpu, ncs_ref = o["ncs"]
    assert abs(ncs_gpu - ncs_ref) <= 1e-13 * max(1.0, abs(ncs_ref))
    assert rel_err(o["E_gpu"], o["E_ref"]) < 1e-13
    assert rel_err(o["U_gpu"], o["U_ref"]) < 1e-13


@pytest.mark.skipif(not (BUILD / "ovl_dropin_test").exists() or not have_reference("wilson"),
                    reason="drop-in program or reference not built")
def test_dropin_build_matches_reference(tmp_path):
    N = (4, 6, 4)
    V = volume(N)
    nranks, rank, m, r, mdw, tsph, dt, steps = 12, 7, 0.1, 1.0, 0.0, 0.12, 0.05, 5
    U = random_links(N, 0.6, 71)
    E = random_efield(N, 0.3, 72)
    o = run_program(tmp_path, BUILD / "ovl_dropin_test", N, nranks, rank, m, r, mdw, tsph, dt, steps, U, E,
                    4 * 4 * V + 2 * V)
    check_gauge_routines(o)

    R = reference("wilson")
    assert R.ovlref_init(*N, nranks, rank, m, r, mdw, tsph, dt, 1.0, 1) == o["nm"]
    R.ovlref_set_links(ptr(U))
    R.ovlref_set_efield(ptr(E))
    R.ovlref_set_free_fermions()
    R.ovlref_step(steps)
    rpsi = np.zeros_like(o["psi"])
    rmid = np.zeros_like(o["psi"])
    R.ovlref_get_modes(ptr(rpsi.view(np.float64)), ptr(rmid.view(np.float64)))
    rU = np.zeros(12 * V)
    R.ovlref_get_links(ptr(rU))
    rcur = [np.zeros(4 * V) for _ in range(4)] + [np.zeros(V), np.zeros(V)]
    R.ovlref_currents(*[ptr(a) for a in rcur])
    assert o["first"] == R.ovlref_first_mode()
    assert rel_err(o["psi"], rpsi) < 1e-12
    assert rel_err(o["mid"], rmid) < 1e-12
    assert rel_err(o["links"], rU) < 1e-13
    scale = current_scale(rpsi)
    assert np.max(np.abs(o["cur"] - np.concatenate(rcur))) <= 1e-12 * scale


@pytest.mark.skipif(not (BUILD / "ovl_dropin_overlap_test").exists() or not have_reference("overlap"),
                    reason="overlap drop-in program or reference not built")
def test_overlap_dropin_build_matches_reference(tmp_path):
    """The overlap build: Update (OverlapUpdate.cpp:99-135, Ritz bounds before
    each half step) and ComputeCurrents (OverlapCurrents.cpp) on the GPU
    against the reference's overlap code compiled from source, from the same
    free overlap spinors, with links moving every half step."""
    N = (4, 4, 4)
    V = volume(N)
    nranks, rank, m, r, mdw, tsph, dt, steps = 16, 5, 0.1, 1.0, 1.4, 1e9, 0.05, 2
    U = random_links(N, 0.4, 121)
    E = random_efield(N, 0.2, 122)
    o = run_program(tmp_path, BUILD / "ovl_dropin_overlap_test", N, nranks, rank, m, r, mdw, tsph, dt, steps, U, E,
                    2 * 4 * V)
    check_gauge_routines(o)

    R = reference("overlap")
    assert R.ovlref_init(*N, nranks, rank, m, r, mdw, tsph, dt, 1.0, 7) == o["nm"]
    R.ovlref_set_links(ptr(U))
    R.ovlref_set_efield(ptr(E))
    R.ovlref_set_free_fermions()
    R.ovlref_step(steps)
    rpsi = np.zeros_like(o["psi"])
    rmid = np.zeros_like(o["psi"])
    R.ovlref_get_modes(ptr(rpsi.view(np.float64)), ptr(rmid.view(np.float64)))
    rU = np.zeros(12 * V)
    R.ovlref_get_links(ptr(rU))
    rcur = [np.zeros(4 * V) for _ in range(2)]
    assert R.ovlref_currents(ptr(rcur[0]), ptr(rcur[1]), None, None, None, None) == 2
    assert o["first"] == R.ovlref_first_mode()
    assert rel_err(o["psi"], rpsi) < 1e-10
    assert rel_err(o["mid"], rmid) < 1e-10
    assert rel_err(o["links"], rU) < 1e-13
    scale = current_scale(rpsi)
    assert np.max(np.abs(o["cur"] - np.concatenate(rcur))) <= 1e-10 * scale
