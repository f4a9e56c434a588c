"""ctypes binding of the C ABI in include/ovl.h (libovl_b200.so).

The library is the only implementation: there is no CPU fallback.  Loading
fails with an ImportError naming the missing file when it has not been built
(`python -m overlap_b200.build`).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libovl_b200.so"

OVL_OK = 0
STATUS_NAMES = {
    0: "OVL_OK", 1: "OVL_E_ARG", 2: "OVL_E_OOM", 3: "OVL_E_NOT_CONVERGED", 4: "OVL_E_TIMEOUT",
    5: "OVL_E_NONFINITE", 6: "OVL_E_CUDA", 7: "OVL_E_STATE", 8: "OVL_E_UNSUPPORTED",
}


ABI_VERSION = 7  # OVL_ABI_VERSION of include/ovl.h
HOP_VARIANTS = 4  # OVL_HOP_VARIANTS
ENSEMBLE_TILES = 3  # OVL_ENSEMBLE_TILES: 8, 4 and 16 (packed) sites


class ovl_params(C.Structure):
    _fields_ = [
        ("N", C.c_int * 3), ("n_colours", C.c_int), ("n_modes", C.c_int), ("first_mode", C.c_int),
        ("fermion", C.c_int), ("precision", C.c_int), ("form", C.c_int),
        ("r_wilson", C.c_double), ("m_fermion", C.c_double), ("m_dw", C.c_double), ("dt", C.c_double),
        ("qs", C.c_double), ("t_sphaleron", C.c_double), ("device", C.c_int), ("plain_chunk_modes", C.c_int),
        ("stream", C.c_uint64), ("zolo_poles", C.c_int), ("zolo_tol", C.c_double), ("cg_max_iter", C.c_int),
        ("cg_tol", C.c_double), ("sign_method", C.c_int), ("cheb_degree", C.c_int), ("cheb_eps", C.c_double),
        ("hop_variant", C.c_int), ("reunitarize", C.c_int), ("gauge_force", C.c_int), ("backreaction", C.c_double),
        ("ritz_auto", C.c_int), ("ritz_seed", C.c_uint64), ("mode_group", C.c_int),
    ]


_dp = C.POINTER(C.c_double)
_vp = C.c_void_p
_ctx = C.c_void_p

# name -> (argtypes, restype); every function of include/ovl.h
SIGNATURES = {
    "ovl_params_init": ([C.POINTER(ovl_params)], C.c_int),
    "ovl_abi_version": ([], C.c_int),
    "ovl_create": ([C.POINTER(ovl_params), C.POINTER(_ctx)], C.c_int),
    "ovl_destroy": ([_ctx], C.c_int),
    "ovl_last_error": ([_ctx], C.c_char_p),
    "ovl_set_links": ([_ctx, _dp], C.c_int),
    "ovl_get_links": ([_ctx, _dp], C.c_int),
    "ovl_set_efield": ([_ctx, _dp], C.c_int),
    "ovl_get_efield": ([_ctx, _dp], C.c_int),
    "ovl_set_u1": ([_ctx, _dp], C.c_int),
    "ovl_set_modes": ([_ctx, C.c_int, C.c_int, _dp, _dp], C.c_int),
    "ovl_get_modes": ([_ctx, C.c_int, C.c_int, _dp, _dp], C.c_int),
    "ovl_set_free_fermions": ([_ctx, C.POINTER(C.c_int)], C.c_int),
    "ovl_step": ([_ctx, C.c_int], C.c_int),
    "ovl_step_observe": ([_ctx, C.c_int, _dp], C.c_int),
    "ovl_get_step_count": ([_ctx, C.POINTER(C.c_int)], C.c_int),
    "ovl_set_step_count": ([_ctx, C.c_int], C.c_int),
    "ovl_currents": ([_ctx, _dp, _dp, _dp, _dp, _dp, _dp], C.c_int),
    "ovl_charges": ([_ctx, _dp], C.c_int),
    "ovl_ncsdot": ([_ctx, _dp], C.c_int),
    "ovl_ncs_update": ([_ctx, _dp, _dp], C.c_int),
    "ovl_update_links": ([_ctx, C.c_double], C.c_int),
    "ovl_update_efield": ([_ctx, C.c_double], C.c_int),
    "ovl_ensemble_create": ([C.POINTER(ovl_params), C.c_int, C.POINTER(_ctx)], C.c_int),
    "ovl_ensemble_destroy": ([_ctx], C.c_int),
    "ovl_ensemble_last_error": ([_ctx], C.c_char_p),
    "ovl_ensemble_member": ([_ctx, C.c_int, C.POINTER(_ctx)], C.c_int),
    "ovl_ensemble_add": ([_ctx, C.POINTER(ovl_params), C.POINTER(C.c_int)], C.c_int),
    "ovl_ensemble_remove": ([_ctx, C.c_int], C.c_int),
    "ovl_ensemble_size": ([_ctx], C.c_int),
    "ovl_ensemble_step": ([_ctx, C.c_int], C.c_int),
    "ovl_ensemble_set_tile": ([_ctx, C.c_int], C.c_int),
    "ovl_ensemble_charges": ([_ctx, _dp], C.c_int),
    "ovl_ensemble_info": ([_ctx, C.POINTER(C.c_int), _dp, C.POINTER(C.c_uint64)], C.c_int),
    "ovl_ensemble_synchronize": ([_ctx], C.c_int),
    "ovl_ensemble_stream": ([_ctx], C.c_uint64),
    "ovl_set_stochastic_modes": ([_ctx, C.c_uint64, C.c_int], C.c_int),
    "ovl_tuning": ([_ctx, C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
    "ovl_ritz_bounds": ([_ctx, _dp, _dp, _dp, C.POINTER(C.c_int)], C.c_int),
    "ovl_color_force": ([_ctx, _dp], C.c_int),
    "ovl_fermion_energy": ([_ctx, _dp], C.c_int),
    "ovl_gauss_restore": ([_ctx, C.c_int, C.c_double, C.POINTER(C.c_int), _dp], C.c_int),
    "ovl_set_handmade_sphaleron": ([_ctx, C.c_double, C.c_double, _dp], C.c_int),
    "ovl_set_qed_eigenmodes": ([_ctx, _dp, _dp, C.POINTER(C.c_int)], C.c_int),
    "ovl_set_quasi_particles": ([_ctx, C.c_double, C.c_double, C.c_uint64, C.c_int, C.POINTER(C.c_int)], C.c_int),
    "ovl_bulk": ([_ctx, _dp], C.c_int),
    "ovl_save_configuration": ([_ctx, C.c_char_p, C.c_char_p], C.c_int),
    "ovl_upload_gauge_async": ([_ctx, _dp, _dp], C.c_int),
    "ovl_step_observe_async": ([_ctx, C.c_int, _dp], C.c_int),
    "ovl_cool": ([_ctx, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _dp, C.POINTER(C.c_int), _dp, _dp,
                  C.POINTER(C.c_int)], C.c_int),
    "ovl_load_configuration": ([_ctx, C.c_char_p, C.c_char_p], C.c_int),
    "ovl_synchronize": ([_ctx], C.c_int),
    "ovl_device_modes": ([_ctx, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(C.c_size_t)], C.c_int),
    "ovl_set_spectral_bounds": ([_ctx, _dp, C.c_int], C.c_int),
    "ovl_apply": ([_ctx, C.c_int, _dp, _dp], C.c_int),
    "ovl_autotune": ([_ctx, C.POINTER(C.c_int), _dp], C.c_int),
    "ovl_pipeline_selftest": ([_ctx, C.POINTER(C.c_int)], C.c_int),
    "ovl_zolotarev": ([C.c_double, C.c_double, C.c_double, C.c_int, _dp, _dp, _dp], C.c_int),
    "ovl_solver_stats": ([_ctx, C.POINTER(C.c_int)], C.c_int),
    "ovl_ncsdot_noalloc": ([_vp, _vp, C.c_int, C.c_int, C.c_int, _vp, C.c_uint64], C.c_int),
    "ovl_launch_count": ([_ctx, C.POINTER(C.c_uint64)], C.c_int),
    "ovl_profile_enable": ([_ctx, C.c_int], C.c_int),
    "ovl_profile_read": ([_ctx, _dp, C.POINTER(C.c_uint64)], C.c_int),
}

PROF_KINDS = ("hop", "axpy", "links", "obs")

_lib = None


def lib() -> C.CDLL:
    """The loaded library with typed signatures; ImportError if it is not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"overlap_b200 CUDA library not built: {LIB_PATH} is missing "
                              "(run `python -m overlap_b200.build`)")
        L = C.CDLL(str(LIB_PATH))
        L.ovl_abi_version.argtypes = []
        L.ovl_abi_version.restype = C.c_int
        if L.ovl_abi_version() != ABI_VERSION:
            raise ImportError(f"{LIB_PATH} has ABI {L.ovl_abi_version()}, the bindings expect {ABI_VERSION} "
                              "(run `python -m overlap_b200.build`)")
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib
