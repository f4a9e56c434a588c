"""Gradient-flow cooling and the Chern-Simons calibration on the device
(ovl_cool) against the oracle (orc_cool, pinned to the reference's
GRADIENTFLOW/Cooling.cpp and TOPOLOGY/CoolingMethod.cpp by
tests/test_oracle_cooling.py) and against the golden fixture the reference
produced: every log row (cooling time, magnetic and electric energy, Delta
N_CS along the calibration path, vacuum N_CS) to 1e-12 of its column's scale,
the cooled links to 1e-13, both colours, with blocking in both phases."""
import numpy as np
import pytest

from overlap_b200 import Context, OvlError
from overlap_b200.inputs import random_links, random_links_su3
from test_oracle_cooling import orc_cool, same_log

pytestmark = pytest.mark.gpu


def device_cool(N, U, schedule, nc=2):
    with Context(N=N, n_colours=nc, n_modes=32, precision="fp64") as ctx:
        ctx.set_links(U)
        s = list(schedule)
        r = ctx.cool(calibration_steps=s[2], standard_steps=s[0], standard_blocking=s[1], calibration_blocking=s[3],
                     block_frequency=s[4])
        assert np.array_equal(ctx.get_links(), U)  # the context's links are not touched
    return r


def test_cooling_matches_golden(golden_dir):
    g = dict(np.load(golden_dir / "cooling_n8.npz"))
    N = tuple(int(n) for n in g["N"])
    r = device_cool(N, g["links"], g["schedule"])
    assert r["cooled_N"] == tuple(int(n) for n in g["cooled_N"])
    assert same_log(r["log"], g["log"])
    assert abs(r["delta_ncs"] - g["out"][0]) < 1e-12 * abs(g["out"][0])
    assert r["cooling_time"] == g["out"][1] and r["blocking"] == g["out"][2]
    assert np.max(np.abs(r["cooled_links"] - g["cooled"])) < 1e-13


@pytest.mark.parametrize("nc,N,schedule", [(2, (16, 16, 8), (0, 0, 40, 2, 32)),   # the reference driver's schedule
                                           (2, (8, 8, 4), (5, 1, 12, 2, 2)),
                                           (2, (5, 6, 4), (4, 0, 6, 0, 32)),
                                           (3, (8, 4, 8), (3, 1, 10, 2, 2)),
                                           (3, (6, 6, 6), (0, 0, 8, 0, 32))])
def test_cooling_matches_the_oracle(nc, N, schedule):
    U = random_links_su3(N, 0.7, 3 + sum(N)) if nc == 3 else random_links(N, 0.8, 3 + sum(N))
    r = device_cool(N, U, schedule, nc)
    log, out, Nc, cooled = orc_cool(N, U, schedule, nc)
    assert r["cooled_N"] == Nc and r["log"].shape == log.shape
    assert same_log(r["log"], log)
    assert abs(r["delta_ncs"] - out[0]) <= 1e-12 * max(abs(out[0]), 1e-300)
    assert r["cooling_time"] == out[1] and r["blocking"] == out[2]
    got = r["cooled_links"].view(np.float64).reshape(-1) if nc == 3 else r["cooled_links"].reshape(-1)
    assert np.max(np.abs(got - cooled)) < 1e-13


def test_a_schedule_that_blocks_below_two_sites_is_refused():
    with Context(N=(3, 4, 4), n_modes=32, precision="fp64") as ctx:
        ctx.set_links(random_links((3, 4, 4), 0.5, 1))
        with pytest.raises(OvlError, match="blocking"):  # 3x4x4 -> 1x2x2 -> refused
            ctx.cool(calibration_steps=16, calibration_blocking=2, block_frequency=2)  # second one at step 16
        r = ctx.cool(calibration_steps=3, calibration_blocking=1, block_frequency=2)  # one blocking: 1x2x2
        assert r["blocking"] == 1 and r["cooled_N"] == (3, 4, 4) and r["log"].shape == (4, 5)
        log = orc_cool((3, 4, 4), ctx.get_links(), (0, 0, 3, 1, 2))[0]
        assert same_log(r["log"], log)
