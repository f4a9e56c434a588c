"""The C ABI library loads and exports every function include/ovl.h declares
(no GPU needed: nothing here launches work)."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def header_functions():
    text = (ROOT / "include" / "ovl.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(ovl_\w+)\s*\(", text, re.M)))


def test_header_declares_the_boundary():
    names = header_functions()
    for must in ("ovl_create", "ovl_destroy", "ovl_step", "ovl_currents", "ovl_ncsdot", "ovl_set_links", "ovl_set_modes"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from overlap_b200 import _lib
    L = _lib.lib()
    for name in header_functions():
        assert hasattr(L, name), name
    assert set(header_functions()) == set(_lib.SIGNATURES), "binding out of sync with include/ovl.h"


def test_params_init_matches_reference_defaults():
    from overlap_b200 import _lib
    p = _lib.ovl_params()
    assert _lib.lib().ovl_params_init(C.byref(p)) == 0
    # Simulation.cpp:74,168,194-200 and Dynamics.cpp:17
    assert (p.r_wilson, p.m_fermion, p.m_dw, p.dt, p.qs, p.t_sphaleron) == (1.0, 0.0, 1.4, 0.02, 1.0, 6.0)
    assert p.n_colours == 2


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    from overlap_b200 import _lib
    monkeypatch.setattr(_lib, "LIB_PATH", tmp_path / "absent.so")
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(ImportError, match="not built"):
        _lib.lib()


def test_create_rejects_bad_arguments_before_touching_a_gpu():
    from overlap_b200 import Context, OvlError
    with pytest.raises(OvlError, match="OVL_E_ARG"):
        Context(N=(2, 8, 8))
    with pytest.raises(OvlError, match="OVL_E_UNSUPPORTED"):
        Context(N=(4, 4, 4), fermion="overlap", precision="fp32")
    with pytest.raises(OvlError, match="OVL_E_ARG"):
        Context(N=(4, 4, 4), fermion="overlap", zolo_poles=0)
    with pytest.raises(OvlError, match="OVL_E_ARG"):
        Context(N=(4, 4, 4), dt=-1.0)


def test_zolotarev_rejects_bad_intervals():
    from overlap_b200 import OvlError, zolotarev
    with pytest.raises(OvlError, match="OVL_E_ARG"):
        zolotarev(1.0, 0.5)
    with pytest.raises(OvlError, match="OVL_E_ARG"):
        zolotarev(0.1, 2.0, npoles=0)


def test_abi_version_agrees_between_header_bindings_and_library():
    from overlap_b200 import _lib
    m = re.search(r"#define OVL_ABI_VERSION (\d+)", (ROOT / "include" / "ovl.h").read_text())
    assert int(m.group(1)) == _lib.ABI_VERSION == _lib.lib().ovl_abi_version()


def test_ctypes_params_layout_matches_the_c_compiler(tmp_path):
    """Offsets of every ovl_params field as gcc lays them out from include/ovl.h
    against the ctypes mirror: a mismatch would let ovl_params_init write past
    the caller's struct."""
    import shutil
    import subprocess
    from overlap_b200 import _lib
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    fields = [f[0] for f in _lib.ovl_params._fields_]
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "ovl.h"\nint main(void) {\n'
                   + "".join(f'  printf("%zu\\n", offsetof(ovl_params, {f}));\n' for f in fields)
                   + '  printf("%zu\\n", sizeof(ovl_params));\n  return 0;\n}\n')
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c11", "-I", str(ROOT / "include"), "-o", str(exe), str(src)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [getattr(_lib.ovl_params, f).offset for f in fields] + [C.sizeof(_lib.ovl_params)]
    assert got == want


def test_mode_group_is_validated():
    from overlap_b200 import Context, OvlError
    with pytest.raises(OvlError):
        Context(N=(4, 4, 4), n_modes=8, form="fused", mode_group=-2)


def test_fp40_is_rejected_outside_the_fused_wilson_form():
    from overlap_b200 import Context, OvlError
    for kw in (dict(form="plain"), dict(fermion="overlap", form="fused", sign_method="chebyshev")):
        with pytest.raises(OvlError, match="FP40"):
            Context(N=(4, 4, 4), n_modes=8, precision="fp40", **kw)


def test_poisson_requests_are_seeded_and_in_range():
    from overlap_b200.serve import poisson_requests, request_bytes
    a = poisson_requests(20, 20.0, seed=5)
    b = poisson_requests(20, 20.0, seed=5)
    assert [(r.N, r.n_modes, r.steps, r.arrival) for r in a] == [(r.N, r.n_modes, r.steps, r.arrival) for r in b]
    assert all(r.N[0] in (8, 12, 16, 24) and 4096 <= r.n_modes <= 8192 and 200 <= r.steps <= 2000 for r in a)
    assert all(x.arrival < y.arrival for x, y in zip(a, a[1:]))
    assert request_bytes(a[0], "fp32") < request_bytes(a[0], "fp64")


def test_serving_requests_follow_the_stated_mix():
    """Every kind of request (SU(2)/SU(3), Wilson/overlap) draws N from
    {8, 12, 16, 24} and 200-2000 steps; an overlap step costs two Chebyshev
    series of K + 1 terms in Wilson-step units."""
    from overlap_b200.serve import Request, poisson_requests, request_cost
    reqs = poisson_requests(256, 20.0, seed=7, su3_fraction=0.25, overlap_fraction=0.125)
    ov = [r for r in reqs if r.fermion == "overlap"]
    assert 16 <= len(ov) <= 48 and 40 <= sum(r.n_colours == 3 for r in reqs) <= 90
    assert {r.N[0] for r in ov} == {8, 12, 16, 24}
    assert min(r.steps for r in ov) >= 200 and max(r.steps for r in ov) <= 2000 and max(r.steps for r in ov) > 1000
    assert all(r.cheb_degree == 64 for r in ov)
    w = Request(N=(8, 8, 8), n_modes=4096, steps=1)
    o = Request(N=(8, 8, 8), n_modes=4096, steps=1, fermion="overlap", cheb_degree=64)
    assert request_cost(w) == 4096 * 512 and request_cost(o) / request_cost(w) == 2 * 65 * 7 / 6
    assert request_cost(Request(N=(8, 8, 8), n_modes=4096, steps=1, n_colours=3)) == 1.5 * request_cost(w)


def test_serving_chunks_end_at_observations_and_hold_a_bounded_gpu_time():
    """A chunk of a group holds about tick_seconds of GPU work and at least
    one step (an overlap request on 24^3 takes about a second per step), and
    ends at the next observation point or last step of any request in it."""
    from overlap_b200.serve import Request, Server
    s = Server.__new__(Server)
    s.rate_wilson, s.tick_seconds, s.tick_steps = 1.2e10, 0.5, 50
    w = [Request(N=(n, n, n), n_modes=6144, steps=1000) for n in (8, 12, 16, 24)]
    o = Request(N=(24, 24, 24), n_modes=8192, steps=1000, fermion="overlap")
    for r in w + [o]:
        r._step = 0
    assert s._chunk_steps(w) == 48 and s._chunk_steps([o]) == 1
    assert s._chunk_steps(w[:1]) == 50
    w[2]._step = 37  # next observation in 13 steps
    assert s._chunk_steps(w) == 13
    w[0]._step = 990  # ten steps left
    assert s._chunk_steps(w[:1]) == 10
