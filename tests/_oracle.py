"""ctypes bindings for the CPU checkers (test infrastructure).

liboracle.so        plain-C restatement (oracle/ovl_oracle.c), always built.
libovlref_*.so      the reference's own C++ compiled from source by oracle/Makefile;
                    present only where the reference tree was available at build time.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
REF_DIR = ROOT / "oracle" / "_ref"

_dp = C.POINTER(C.c_double)


def ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


class OrcParams(C.Structure):
    _fields_ = [("N", C.c_int * 3), ("r_wilson", C.c_double), ("m_fermion", C.c_double),
                ("m_dw", C.c_double), ("dt", C.c_double), ("qs", C.c_double), ("t_sphaleron", C.c_double)]


def orc_params(N, r=1.0, m=0.1, mdw=0.0, dt=0.05, qs=1.0, t_sph=1e300) -> OrcParams:
    p = OrcParams()
    p.N[0], p.N[1], p.N[2] = N
    p.r_wilson, p.m_fermion, p.m_dw, p.dt, p.qs, p.t_sphaleron = r, m, mdw, dt, qs, t_sph
    return p


_oracle = None


def oracle():
    """The restated oracle; raises if it has not been built."""
    global _oracle
    if _oracle is None:
        path = REF_DIR / "liboracle.so"
        if not path.exists():
            raise RuntimeError(f"{path} missing: run `make -C oracle oracle`")
        L = C.CDLL(str(path))
        P = C.POINTER(OrcParams)
        L.orc_wilson_apply.argtypes = [P, _dp, _dp, _dp]
        L.orc_update_links.argtypes = [P, _dp, _dp, C.c_double]
        L.orc_update_efield.argtypes = [P, _dp, _dp, C.c_double]
        L.orc_wilson_leapfrog.argtypes = [P, _dp, _dp, _dp, _dp, C.c_int, C.POINTER(C.c_int), C.c_int]
        L.orc_free_fermions.argtypes = [P, C.c_int, C.c_int, _dp, _dp]
        L.orc_free_fermions.restype = C.c_int
        L.orc_wilson_currents.argtypes = [P, _dp, _dp, C.c_int, C.c_int] + [_dp] * 6
        L.orc_ncsdot.argtypes = [P, _dp, _dp]
        L.orc_ncsdot.restype = C.c_double
        L.orc_bulk.argtypes = [P, _dp, _dp, _dp]
        L.orc_u1_flux.argtypes = [P, C.c_int, _dp]
        L.orc_set_u1.argtypes = [_dp]
        L.orc_color_force.argtypes = [P, _dp, _dp, C.c_int, C.c_int, _dp]
        L.orc_fermion_energy.argtypes = [P, _dp, _dp, C.c_int, C.c_int]
        L.orc_fermion_energy.restype = C.c_double
        L.orc_gauss_restore.argtypes = [P, _dp, _dp, C.c_int, C.c_double, _dp]
        L.orc_gauss_restore.restype = C.c_int
        L.orc_ritz.argtypes = [P, _dp, _dp, C.c_double, C.c_int, C.c_int, C.c_double, C.POINTER(C.c_int)]
        L.orc_ritz.restype = C.c_double
        L.orc_coupled_leapfrog.argtypes = [P, _dp, _dp, _dp, _dp, C.c_int, C.c_int, C.POINTER(C.c_int), C.c_int,
                                           C.c_double, C.c_int]
        L.orc3_exp.argtypes = [C.c_double, _dp, _dp]
        L.orc_set_free_kind.argtypes = [C.c_int]
        L.orc3_wilson_apply.argtypes = [P, _dp, _dp, _dp]
        L.orc3_update_links.argtypes = [P, _dp, _dp, C.c_double]
        L.orc3_update_efield.argtypes = [P, _dp, _dp, C.c_double]
        L.orc3_wilson_leapfrog.argtypes = [P, _dp, _dp, _dp, _dp, C.c_int, C.POINTER(C.c_int), C.c_int]
        L.orc3_free_fermions.argtypes = [P, C.c_int, C.c_int, _dp, _dp]
        L.orc3_free_fermions.restype = C.c_int
        L.orc3_charges.argtypes = [P, _dp, _dp, C.c_int, C.c_int, _dp]
        L.orc3_ncsdot.argtypes = [P, _dp, _dp]
        L.orc3_ncsdot.restype = C.c_double
        L.orc3_delta_ncs.argtypes = [P, _dp, _dp]
        L.orc3_delta_ncs.restype = C.c_double
        L.orc3_bulk.argtypes = [P, _dp, _dp, _dp]
        L.orc3_gauss_restore.argtypes = [P, _dp, _dp, C.c_int, C.c_double, _dp]
        L.orc3_gauss_restore.restype = C.c_int
        L.orc3_color_force.argtypes = [P, _dp, _dp, C.c_int, C.c_int, _dp]
        L.orc3_fermion_energy.argtypes = [P, _dp, _dp, C.c_int, C.c_int]
        L.orc3_fermion_energy.restype = C.c_double
        L.orc3_coupled_leapfrog.argtypes = [P, _dp, _dp, _dp, _dp, C.c_int, C.c_int, C.POINTER(C.c_int), C.c_int,
                                            C.c_double, C.c_int]
        L.orc_chebyshev_coeffs.argtypes = [C.c_int, C.c_double, _dp]
        L.orc_handmade_sphaleron.argtypes = [P, C.c_double, C.c_double, _dp, _dp, _dp, _dp]
        L.orc_vacuum_ncs.argtypes = [P, C.c_int, _dp]
        L.orc_vacuum_ncs.restype = C.c_double
        L.orc_block_links.argtypes = [P, C.c_int, _dp, _dp]
        L.orc_cool.argtypes = [P, C.c_int, _dp] + [C.c_int] * 5 + [_dp, C.POINTER(C.c_int), _dp, _dp,
                                                                   C.POINTER(C.c_int)]
        L.orc_cool.restype = C.c_int
        L.orc3_overlap_apply.argtypes = [P, _dp, _dp, _dp, C.c_int, C.c_double, C.c_double]
        L.orc3_overlap_leapfrog.argtypes = [P, _dp, _dp, _dp, _dp, C.c_int, C.POINTER(C.c_int), C.c_int, C.c_int,
                                            C.c_double, C.c_double]
        _oracle = L
    return _oracle


def have_reference(kind: str = "wilson") -> bool:
    return (REF_DIR / f"libovlref_{kind}.so").exists()


_refs = {}


def reference(kind: str = "wilson"):
    """The reference compiled from source (one process-wide instance per kind)."""
    if kind not in _refs:
        path = REF_DIR / f"libovlref_{kind}.so"
        if not path.exists():
            raise RuntimeError(f"{path} missing")
        L = C.CDLL(str(path), mode=os.RTLD_LOCAL)
        L.ovlref_init.argtypes = [C.c_int] * 5 + [C.c_double] * 6 + [C.c_long]
        L.ovlref_init.restype = C.c_int
        for name in ("ovlref_set_links", "ovlref_get_links", "ovlref_set_efield", "ovlref_get_efield", "ovlref_bulk"):
            getattr(L, name).argtypes = [_dp]
        L.ovlref_set_modes.argtypes = [_dp, _dp]
        L.ovlref_get_modes.argtypes = [_dp, _dp]
        L.ovlref_step.argtypes = [C.c_int]
        L.ovlref_step.restype = C.c_double
        L.ovlref_currents.argtypes = [_dp] * 6
        L.ovlref_currents.restype = C.c_int
        L.ovlref_ncsdot.restype = C.c_double
        L.ovlref_delta_ncs.argtypes = [_dp, _dp]
        L.ovlref_delta_ncs.restype = C.c_double
        L.ovlref_update_links.argtypes = [C.c_double]
        L.ovlref_update_efield.argtypes = [C.c_double]
        L.ovlref_u1_flux.argtypes = [C.c_int, _dp]
        L.ovlref_apply.argtypes = [_dp, _dp, C.c_double, C.c_double]
        L.ovlref_set_step_count.argtypes = [C.c_int]
        L.ovlref_gauss_restore.argtypes = [_dp]
        L.ovlref_handmade_sphaleron.argtypes = [C.c_double, C.c_double, _dp, _dp, _dp]
        L.ovlref_save_configuration.argtypes = [C.c_char_p, C.c_long, C.c_char_p, C.c_char_p]
        L.ovlref_load_configuration.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p]
        L.ovlref_cool.argtypes = [C.c_int] * 5 + [_dp, C.POINTER(C.c_int), _dp, _dp, C.POINTER(C.c_int)]
        L.ovlref_cool_driver_log.argtypes = [C.c_char_p, C.c_long] + [C.c_int] * 5
        if kind == "overlap":
            L.ovlref_ritz_bounds.argtypes = [_dp]
            L.ovlref_ritz_solve.argtypes = [_dp, C.c_double]
            L.ovlref_ritz_solve.restype = C.c_double
            L.ovlref_zolotarev.argtypes = [C.c_double, C.c_double, _dp, _dp]
            L.ovlref_zolotarev.restype = C.c_double
            L.ovlref_take_bounds.argtypes = [_dp, C.c_int]
            L.ovlref_take_bounds.restype = C.c_int
            L.ovlref_last_bounds.argtypes = [_dp]
            L.ovlref_qed_hamiltonian.argtypes = [C.c_int, _dp, _dp]
        _refs[kind] = L
    return _refs[kind]
