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
