"""overlap_b200: the OVERLAP real-time fermion + SU(2) gauge evolution hot path
on one NVIDIA B200 (sm_100a), behind the C ABI of include/ovl.h.

    from overlap_b200 import Context
    with Context(N=(8, 8, 8), precision="fp64", form="plain", m_fermion=0.1, m_dw=0.0, dt=0.05) as ctx:
        ctx.set_links(U); ctx.set_free_fermions(); ctx.step(200); ctx.charges()
"""
from .api import Context, Ensemble, OvlError, Params, zolotarev  # noqa: F401
from . import inputs  # noqa: F401

__all__ = ["Context", "Ensemble", "OvlError", "Params", "inputs", "zolotarev"]
