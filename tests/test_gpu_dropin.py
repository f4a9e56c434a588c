"""The reference's own build with include/ovl_dropin.hpp in place of its Wilson
hot path (tests/dropin/dropin_main.cpp) produces the reference's results: modes,
links and current arrays agree with the reference compiled from source."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from _helpers import current_scale, rel_err
from _oracle import have_reference, ptr, reference
from overlap_b200.inputs import random_efield, random_links, volume

pytestmark = pytest.mark.gpu

BIN = Path(__file__).resolve().parent / "dropin" / "_build" / "ovl_dropin_test"


@pytest.mark.skipif(not BIN.exists() or not have_reference("wilson"), reason="drop-in program or reference not built")
def test_dropin_build_matches_reference(tmp_path):
    N = (4, 6, 4)
    V = volume(N)
    nranks, rank, m, r, mdw, tsph, dt, steps = 12, 7, 0.1, 1.0, 0.0, 0.12, 0.05, 5
    U = random_links(N, 0.6, 71)
    E = random_efield(N, 0.3, 72)
    inp = tmp_path / "in.bin"
    out = tmp_path / "out.bin"
    np.concatenate([U.ravel(), E.ravel()]).tofile(inp)
    res = subprocess.run([str(BIN), *map(str, N), str(nranks), str(rank), str(m), str(r), str(mdw), str(tsph), str(dt),
                          str(steps), str(inp), str(out)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    first, nm = map(int, res.stdout.split())
    data = np.fromfile(out, dtype=np.float64)
    k = nm * V * 16
    psi = data[:k].view(np.complex128).reshape(nm, V, 2, 4)
    mid = data[k:2 * k].view(np.complex128).reshape(nm, V, 2, 4)
    links = data[2 * k:2 * k + 12 * V]
    cur = data[2 * k + 12 * V:]
    assert cur.size == 4 * 4 * V + 2 * V

    R = reference("wilson")
    assert R.ovlref_init(*N, nranks, rank, m, r, mdw, tsph, dt, 1.0, 1) == nm
    R.ovlref_set_links(ptr(U))
    R.ovlref_set_efield(ptr(E))
    R.ovlref_set_free_fermions()
    R.ovlref_step(steps)
    rpsi = np.zeros_like(psi)
    rmid = np.zeros_like(psi)
    R.ovlref_get_modes(ptr(rpsi.view(np.float64)), ptr(rmid.view(np.float64)))
    rU = np.zeros(12 * V)
    R.ovlref_get_links(ptr(rU))
    rcur = [np.zeros(4 * V) for _ in range(4)] + [np.zeros(V), np.zeros(V)]
    R.ovlref_currents(*[ptr(a) for a in rcur])
    assert first == R.ovlref_first_mode()
    assert rel_err(psi, rpsi) < 1e-12
    assert rel_err(mid, rmid) < 1e-12
    assert rel_err(links, rU) < 1e-13
    scale = current_scale(rpsi)
    assert np.max(np.abs(cur - np.concatenate(rcur))) <= 1e-12 * scale
