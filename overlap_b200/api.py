"""Python host API over the C ABI.

`Context` owns one lattice, its SU(2) links and electric field, and a batch of
fermion modes resident on one GPU.  Its methods carry the names and meaning of
the reference routines they replace:

    step(n)            n x Dynamics::Fermions::Update (FERMIONS/WILSON/Update.cpp:48-79)
    currents()         Fermions::Observables::ComputeCurrents (FERMIONS/WILSON/Currents.cpp:7-394)
    ncsdot()           ChernSimonsNumber::NCsDot (TOPOLOGY/ChernSimonsDerivative.cpp:31-49)
    update_links(dt)   Dynamics::UpdateGaugeLinks (DYNAMICS/Dynamics.cpp:97-138)
    update_efield(dt)  Dynamics::UpdateElectricFields (DYNAMICS/Dynamics.cpp:145-197)
    bulk()             Observables::Bulk / GaussLaw / Unitarity (OBSERVABLES/*.cpp)
    set_free_fermions  InitialConditions::SetFreeFermions (INITIALCONDITIONS/FERMIONS/SetFreeFermions.cpp)

Arrays cross the boundary in the reference's layouts (see overlap_b200.inputs).
Errors raise OvlError carrying the C status code; the reference itself prints
and exits on errors (e.g. MPI/ModePartition.cpp:18-21).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from .inputs import volume

PRECISIONS = {"fp64": 0, "fp32": 1, "fp40": 2}  # fp40: modes in 40 bits (top bits of FP64), FP64 arithmetic
SIGN_METHODS = {"zolotarev": 0, "chebyshev": 1}
FORMS = {"plain": 0, "fused": 1}
FERMIONS = {"wilson": 0, "overlap": 1}


def zolotarev(lambda_min: float, lambda_max: float, tol: float = 1e-12, npoles: int = 25):
    """Zolotarev coefficients (b, d, eps) of (h_W^2)^(-1/2) on [lambda_min, lambda_max]."""
    b = np.zeros(npoles)
    d = np.zeros(npoles)
    eps = np.zeros(1)
    rc = _lib.lib().ovl_zolotarev(float(lambda_min), float(lambda_max), float(tol), int(npoles), _dp(b), _dp(d), _dp(eps))
    if rc != 0:
        raise OvlError(rc, _lib.lib().ovl_last_error(None).decode())
    return b, d, float(eps[0])


class OvlError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{_lib.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


@dataclass
class Params:
    N: tuple = (8, 8, 8)
    n_colours: int = 2               # 2: SU(2) links (u0, u1, u2, u3); 3: SU(3), 9 complex per link
    n_modes: int | None = None       # default: the full basis 4*Nc*V
    first_mode: int = 0
    fermion: str = "wilson"
    precision: str = "fp64"
    form: str = "plain"
    r_wilson: float = 1.0
    m_fermion: float = 0.0
    m_dw: float = 1.4
    dt: float = 0.02
    qs: float = 1.0
    t_sphaleron: float = 6.0
    device: int = 0
    plain_chunk_modes: int = 0
    stream: int = 0
    zolo_poles: int = 25         # OverlapOperator.cpp:13-18
    zolo_tol: float = 1e-12
    cg_max_iter: int = 1000
    cg_tol: float = 1e-16
    hop_variant: int = -1            # -1: autotune on the first step; 0..3 fixed (3: FP32 only)
    reunitarize: bool = False        # project links onto SU(2) after each update
    gauge_force: bool = False        # coupled evolution: staple force on E every step
    backreaction: float = 0.0        # coupled evolution: g^2 of the fermion force on E
    ritz_auto: bool = False          # overlap: GPU Ritz bounds before every application (no schedule set)
    ritz_seed: int = 0               # generator seed of the Ritz start vectors
    mode_group: int = 0              # fused form: mode blocks per group (0 whole batch, -1 autotune)
    sign_method: str = "zolotarev"  # or "chebyshev" (the FP32-capable polynomial form)
    cheb_degree: int = 96
    cheb_eps: float = 0.01

    def to_c(self) -> _lib.ovl_params:
        p = _lib.ovl_params()
        _lib.lib().ovl_params_init(C.byref(p))
        p.N[0], p.N[1], p.N[2] = (int(n) for n in self.N)
        p.n_colours = int(self.n_colours)
        p.n_modes = int(self.n_modes if self.n_modes is not None else 4 * int(self.n_colours) * volume(self.N))
        p.first_mode = int(self.first_mode)
        p.fermion = FERMIONS[self.fermion]
        p.precision = PRECISIONS[self.precision]
        p.form = FORMS[self.form]
        p.r_wilson, p.m_fermion, p.m_dw = self.r_wilson, self.m_fermion, self.m_dw
        p.dt, p.qs, p.t_sphaleron = self.dt, self.qs, self.t_sphaleron
        p.device = int(self.device)
        p.plain_chunk_modes = int(self.plain_chunk_modes)
        p.stream = int(self.stream)
        p.zolo_poles, p.zolo_tol = int(self.zolo_poles), float(self.zolo_tol)
        p.cg_max_iter, p.cg_tol = int(self.cg_max_iter), float(self.cg_tol)
        p.hop_variant = int(self.hop_variant)
        p.reunitarize = int(bool(self.reunitarize))
        p.gauge_force = int(bool(self.gauge_force))
        p.backreaction = float(self.backreaction)
        p.ritz_auto = int(bool(self.ritz_auto))
        p.ritz_seed = int(self.ritz_seed) & (2**64 - 1)
        p.mode_group = int(self.mode_group)
        p.sign_method = SIGN_METHODS[self.sign_method]
        p.cheb_degree, p.cheb_eps = int(self.cheb_degree), float(self.cheb_eps)
        return p


class Context:
    """One lattice + mode batch on one GPU (ovl_create ... ovl_destroy)."""

    def __init__(self, params: Params | None = None, **kw):
        self.params = params if params is not None else Params(**kw)
        self._L = _lib.lib()
        self._ctx = C.c_void_p()
        cp = self.params.to_c()
        rc = self._L.ovl_create(C.byref(cp), C.byref(self._ctx))
        if rc != 0:
            raise OvlError(rc, self._L.ovl_last_error(None).decode())
        self.N = tuple(int(n) for n in self.params.N)
        self.V = volume(self.N)
        self.n_modes = cp.n_modes
        self.nc = int(cp.n_colours)

    # -------------------------------------------------------------- plumbing
    def _check(self, rc: int):
        if rc != 0:
            raise OvlError(rc, self._L.ovl_last_error(self._ctx).decode())

    def close(self):
        if self._ctx and getattr(self, "_owned", True):
            self._L.ovl_destroy(self._ctx)
        self._ctx = C.c_void_p()

    @classmethod
    def _member(cls, handle: C.c_void_p, params: "Params", owner) -> "Context":
        """A view of a context owned by an Ensemble (not destroyed by close())."""
        self = cls.__new__(cls)
        self.params = params
        self._L = _lib.lib()
        self._ctx = handle
        self._owned = False
        self._owner = owner  # keeps the ensemble alive
        self.N = tuple(int(n) for n in params.N)
        self.V = volume(self.N)
        self.nc = int(params.n_colours)
        self.n_modes = int(params.n_modes if params.n_modes is not None else 4 * self.nc * self.V)
        return self

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _as_f64(a, shape) -> np.ndarray:
        a = np.ascontiguousarray(a, dtype=np.float64)
        if a.size != int(np.prod(shape)):
            raise ValueError(f"expected {int(np.prod(shape))} doubles, got {a.size}")
        return a

    # ---------------------------------------------------------------- fields
    # Two colours: links float64[V, 3, 4] (u0, u1, u2, u3), E float64[V, 3, 3];
    # three colours: links complex128[V, 3, 9] (U_ij at i + 3j), E float64[V, 3, 8].
    def set_links(self, U):
        if self.nc == 3:
            U = np.ascontiguousarray(U, dtype=np.complex128).view(np.float64)
        self._check(self._L.ovl_set_links(self._ctx, _dp(self._as_f64(U, (self.V, 3, 18 if self.nc == 3 else 4)))))

    def get_links(self) -> np.ndarray:
        if self.nc == 3:
            out = np.empty((self.V, 3, 9), np.complex128)
            self._check(self._L.ovl_get_links(self._ctx, _dp(out.view(np.float64))))
            return out
        out = np.empty((self.V, 3, 4))
        self._check(self._L.ovl_get_links(self._ctx, _dp(out)))
        return out

    def set_efield(self, E):
        self._check(self._L.ovl_set_efield(self._ctx, _dp(self._as_f64(E, (self.V, 3, self.nc * self.nc - 1)))))

    def set_u1(self, u1):
        """U(1) background phases complex[N1, N0, 2] (QED::U layout), or None to remove."""
        if u1 is None:
            self._check(self._L.ovl_set_u1(self._ctx, None))
            return
        a = np.ascontiguousarray(u1, dtype=np.complex128)
        if a.size != 2 * self.N[0] * self.N[1]:
            raise ValueError("u1 must hold 2*N0*N1 complex phases")
        self._check(self._L.ovl_set_u1(self._ctx, _dp(a.view(np.float64))))

    def get_efield(self) -> np.ndarray:
        out = np.empty((self.V, 3, self.nc * self.nc - 1))
        self._check(self._L.ovl_get_efield(self._ctx, _dp(out)))
        return out

    def set_modes(self, psi=None, psimid=None, first: int = 0):
        """psi / psimid: complex128[count, V, Nc, 4] in the reference layout."""
        arrs = []
        count = None
        for a in (psi, psimid):
            if a is None:
                arrs.append(None)
                continue
            a = np.ascontiguousarray(a, dtype=np.complex128)
            count = a.shape[0]
            if a.size != count * self.V * 4 * self.nc:
                raise ValueError(f"modes must be complex[count, V, {self.nc}, 4]")
            arrs.append(a)
        if count is None:
            return
        ptrs = [None if a is None else a.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)) for a in arrs]
        self._check(self._L.ovl_set_modes(self._ctx, first, count, ptrs[0], ptrs[1]))

    def get_modes(self, first: int = 0, count: int | None = None):
        count = self.n_modes - first if count is None else count
        psi = np.empty((count, self.V, self.nc, 4), np.complex128)
        mid = np.empty_like(psi)
        self._check(self._L.ovl_get_modes(self._ctx, first, count, _dp(psi.view(np.float64)), _dp(mid.view(np.float64))))
        return psi, mid

    def set_free_fermions(self) -> int:
        bad = C.c_int(0)
        self._check(self._L.ovl_set_free_fermions(self._ctx, C.byref(bad)))
        return bad.value

    # ------------------------------------------------------------- operator
    def set_spectral_bounds(self, pairs):
        """(lambda_min, lambda_max) of h_W^2 per overlap application, in order;
        one pair serves every application (replaces ComputeRitzEigenvalues)."""
        a = np.ascontiguousarray(np.asarray(pairs, dtype=np.float64).reshape(-1, 2))
        self._check(self._L.ovl_set_spectral_bounds(self._ctx, _dp(a), a.shape[0]))

    def apply(self, phi) -> np.ndarray:
        """-i h phi (Wilson or overlap) for modes complex[count, V, Nc, 4]."""
        a = np.ascontiguousarray(phi, dtype=np.complex128)
        out = np.empty_like(a)
        self._check(self._L.ovl_apply(self._ctx, a.shape[0], _dp(a.view(np.float64)), _dp(out.view(np.float64))))
        return out

    def autotune(self):
        """Times the hop-kernel variants on this context's fields (state unchanged)
        and keeps the fastest: returns (variant, [ms per half step of each])."""
        v = C.c_int(0)
        ms = np.zeros(_lib.HOP_VARIANTS)
        self._check(self._L.ovl_autotune(self._ctx, C.byref(v), _dp(ms)))
        return v.value, ms.tolist()

    def set_stochastic_modes(self, seed: int = 0, total_pairs: int = 0):
        """Z2-noise vacuum modes (pairs sqrt(V / pairs) (P+ eta, P- eta)) in place of plane waves."""
        self._check(self._L.ovl_set_stochastic_modes(self._ctx, int(seed) & (2**64 - 1), int(total_pairs)))

    def pipeline_selftest(self) -> int:
        """ovl_pipeline_selftest: the status a timed-out pipelined wait produces
        (OVL_E_TIMEOUT = 4 when the detection works)."""
        code = C.c_int(0)
        self._check(self._L.ovl_pipeline_selftest(self._ctx, C.byref(code)))
        return code.value

    def tuning(self) -> tuple[int, int]:
        """(hop variant, mode blocks per group) in use; -1 before the autotuner ran."""
        v, g = C.c_int(-1), C.c_int(-1)
        self._check(self._L.ovl_tuning(self._ctx, C.byref(v), C.byref(g)))
        return v.value, g.value

    def solver_stats(self) -> dict:
        o = (C.c_int * 3)()
        self._check(self._L.ovl_solver_stats(self._ctx, o))
        return {"iterations": o[0], "max_mode_iterations": o[1], "not_converged": o[2]}

    # ------------------------------------------------------------- evolution
    def step(self, nsteps: int = 1):
        self._check(self._L.ovl_step(self._ctx, int(nsteps)))

    @property
    def step_count(self) -> int:
        v = C.c_int(0)
        self._check(self._L.ovl_get_step_count(self._ctx, C.byref(v)))
        return v.value

    @step_count.setter
    def step_count(self, n: int):
        self._check(self._L.ovl_set_step_count(self._ctx, int(n)))

    def update_links(self, dt_step: float):
        self._check(self._L.ovl_update_links(self._ctx, float(dt_step)))

    def update_efield(self, dt_step: float):
        self._check(self._L.ovl_update_efield(self._ctx, float(dt_step)))

    def synchronize(self):
        self._check(self._L.ovl_synchronize(self._ctx))

    # ----------------------------------------------------------- observables
    def currents(self) -> dict:
        V = self.V
        out = {k: np.empty((V, 4)) for k in ("jV", "jA", "jVw", "jAw")}
        out["PS"] = np.empty(V)
        out["WA"] = np.empty(V)
        self._check(self._L.ovl_currents(self._ctx, *(_dp(out[k]) for k in ("jV", "jA", "jVw", "jAw", "PS", "WA"))))
        return out

    def step_observe(self, nsteps: int = 1) -> dict:
        """nsteps leapfrog steps, returning {NV, N5, PS} of the modes at the end,
        summed inside the last half step in the fused Wilson form (ovl_step_observe)."""
        o = np.empty(3)
        self._check(self._L.ovl_step_observe(self._ctx, int(nsteps), _dp(o)))
        return {"NV": o[0], "N5": o[1], "PS": o[2]}

    @staticmethod
    def _pinned_view(a, size, what):
        """The float64 buffer of `a` itself (no copy: the copy queued from it
        runs after the call returns)."""
        if not isinstance(a, np.ndarray) or a.dtype not in (np.float64, np.complex128) or not a.flags.c_contiguous:
            raise ValueError(f"{what}: a C-contiguous float64/complex128 array in page-locked memory")
        v = a.view(np.float64)
        if v.size != size:
            raise ValueError(f"{what}: expected {size} doubles, got {v.size}")
        return v

    def upload_gauge_async(self, links=None, efield=None):
        """ovl_upload_gauge_async: links and/or E from page-locked arrays (e.g.
        torch.empty(..., pin_memory=True).numpy()) copied on the context's
        stream; keep them unchanged until the stream has passed the copy."""
        nl = self.V * 3 * (18 if self.nc == 3 else 4)
        ne = self.V * 3 * (self.nc * self.nc - 1)
        lp = _dp(self._pinned_view(links, nl, "links")) if links is not None else None
        ep = _dp(self._pinned_view(efield, ne, "efield")) if efield is not None else None
        self._check(self._L.ovl_upload_gauge_async(self._ctx, lp, ep))

    def step_observe_async(self, nsteps: int, out) -> None:
        """ovl_step_observe_async: queues nsteps leapfrog steps; {NV, N5, PS} of
        the modes at the end land in `out` (3 doubles, page-locked) once the
        stream has passed the call."""
        self._check(self._L.ovl_step_observe_async(self._ctx, int(nsteps), _dp(self._pinned_view(out, 3, "out"))))

    def charges(self) -> dict:
        o = np.empty(4)
        self._check(self._L.ovl_charges(self._ctx, _dp(o)))
        return {"NV": o[0], "N5": o[1], "PS": o[2], "WA": o[3]}

    def ncsdot(self) -> float:
        o = np.empty(1)
        self._check(self._L.ovl_ncsdot(self._ctx, _dp(o)))
        return float(o[0])

    def ncs_update(self):
        """ChernSimonsNumber::CoolingMethod::Update(1) without cooling: returns
        (change since the previous call, running sum)."""
        d = np.zeros(1)
        t = np.zeros(1)
        self._check(self._L.ovl_ncs_update(self._ctx, _dp(d), _dp(t)))
        return float(d[0]), float(t[0])

    def ritz_bounds(self, start: np.ndarray | None = None) -> dict:
        """ComputeRitzEigenvalues on the GPU: {"bounds": (MinEValue, MaxEValue),
        "raw": (lambda_min, lambda_max), "iters": (n_min, n_max)}; start is one
        mode [V, Nc, 4] complex (None: drawn from the context's generator)."""
        out, raw = np.empty(2), np.empty(2)
        it = (C.c_int * 2)()
        sp = None
        if start is not None:
            start = np.ascontiguousarray(start, dtype=np.complex128)
            if start.size != 4 * self.nc * volume(self.params.N):
                raise ValueError(f"start must hold one mode (V x {self.nc} x 4 complex)")
            sp = _dp(start.view(np.float64))
        self._check(self._L.ovl_ritz_bounds(self._ctx, sp, _dp(out), _dp(raw), it))
        return {"bounds": (float(out[0]), float(out[1])), "raw": (float(raw[0]), float(raw[1])),
                "iters": (int(it[0]), int(it[1]))}

    def color_force(self) -> np.ndarray:
        """dH_F/dtheta^a_mu(x) as [V, 3 (mu), Nc^2 - 1 (a)] (Wilson fermions)."""
        o = np.empty((volume(self.params.N), 3, self.nc * self.nc - 1))
        self._check(self._L.ovl_color_force(self._ctx, _dp(o)))
        return o

    def fermion_energy(self) -> float:
        """H_F = (1/2V) sum_m w_m Re <psi_m, h_W psi_m> (Wilson fermions)."""
        o = np.empty(1)
        self._check(self._L.ovl_fermion_energy(self._ctx, _dp(o)))
        return float(o[0])

    def set_qed_eigenmodes(self, hamiltonian: bool = False):
        """InitialConditions::SetOverlapQEDEigenfunctions on the device: the modes
        become eigenmodes of the overlap Hamiltonian in the context's U(1)
        background.  Returns (eigenvalues ascending, n_bad[, h_ov [D, D]])."""
        D = 8 * self.V
        w = np.empty(D)
        h = np.empty(2 * D * D) if hamiltonian else None
        bad = C.c_int(0)
        self._check(self._L.ovl_set_qed_eigenmodes(self._ctx, _dp(w), _dp(h) if h is not None else None, C.byref(bad)))
        if hamiltonian:
            return w, bad.value, h.view(np.complex128).reshape(D, D).T  # column-major -> [row, column]
        return w, bad.value

    def set_quasi_particles(self, n0: float, qs: float, seed: int, gauss_max_iter: int = 10000) -> int:
        """InitialConditions::SetQuasiParticles on the device (quasi-particle links and E,
        then Gauss's law restored unless gauss_max_iter is 0); returns the restoration's
        iterations.  Noise from the counter-based generator of ovl_set_quasi_particles."""
        it = C.c_int(0)
        self._check(self._L.ovl_set_quasi_particles(self._ctx, float(n0), float(qs), int(seed) & (2**64 - 1),
                                                    int(gauss_max_iter), C.byref(it)))
        return it.value

    def set_handmade_sphaleron(self, r_sphaleron: float, t_sphaleron: float, final_links: bool = False):
        """InitialConditions::HandmadeSphaleron::Setup on the device: unit links and
        the E field that carries them to the pure gauge G(x) G(x+mu)^+ in the time
        t_sphaleron.  Returns the final links [V, 3, 4] when asked."""
        out = np.empty((self.V, 3, 4)) if final_links else None
        self._check(self._L.ovl_set_handmade_sphaleron(self._ctx, float(r_sphaleron), float(t_sphaleron),
                                                       _dp(out) if out is not None else None))
        return out

    def gauss_restore(self, max_iter: int = 10000, tol: float = 1e-14) -> dict:
        """GaussLawRestoration::Restore on the device: {"iterations", "max", "avg"}."""
        n = C.c_int(0)
        o = np.empty(2)
        self._check(self._L.ovl_gauss_restore(self._ctx, int(max_iter), float(tol), C.byref(n), _dp(o)))
        return {"iterations": n.value, "max": float(o[0]), "avg": float(o[1])}

    def bulk(self) -> dict:
        o = np.empty(10)
        self._check(self._L.ovl_bulk(self._ctx, _dp(o)))
        keys = ("T00", "TXX", "TYY", "TZZ", "electric", "magnetic", "gauss_max", "gauss_avg", "unitarity_max", "unitarity_avg")
        return dict(zip(keys, o.tolist()))

    def cool(self, calibration_steps: int, standard_steps: int = 0, standard_blocking: int = 0,
             calibration_blocking: int = 2, block_frequency: int = 32) -> dict:
        """Gradient-flow cooling of a copy of the links and the Chern-Simons
        calibration along it (ovl_cool: CoolingMethod's standard cooling, then
        its calibration; GRADIENTFLOW/Cooling.cpp).  Returns the calibration log
        (rows: cooling time, magnetic, electric, Delta N_CS so far, vacuum
        N_CS), Delta N_CS along the calibration path, the final cooling time and
        blocking level, and the links after the standard phase."""
        log = np.empty((calibration_steps + 1, 5))
        rows, out = C.c_int(0), np.empty(3)
        cooled = np.empty(self.V * 3 * (18 if self.nc == 3 else 4))
        dims = (C.c_int * 3)()
        self._check(self._L.ovl_cool(self._ctx, int(standard_steps), int(standard_blocking), int(calibration_steps),
                                     int(calibration_blocking), int(block_frequency), _dp(log), C.byref(rows),
                                     _dp(out), _dp(cooled), dims))
        Nc = tuple(dims)
        Vc = Nc[0] * Nc[1] * Nc[2]
        links = cooled[:Vc * 3 * (18 if self.nc == 3 else 4)]
        links = links.view(np.complex128).reshape(Vc, 3, 9) if self.nc == 3 else links.reshape(Vc, 3, 4)
        return {"log": log[:rows.value], "delta_ncs": float(out[0]), "cooling_time": float(out[1]),
                "blocking": int(out[2]), "cooled_N": Nc, "cooled_links": links.copy()}

    def save_configuration(self, u_path=None, e_path=None):
        """Writes the links and E as the reference's configuration text files
        (ovl_save_configuration, IO/SaveConfiguration.cpp); None skips a file."""
        enc = lambda q: None if q is None else str(q).encode()
        self._check(self._L.ovl_save_configuration(self._ctx, enc(u_path), enc(e_path)))

    def load_configuration(self, u_path=None, e_path=None):
        """Reads links and E from the reference's configuration text files
        (ovl_load_configuration, IO/LoadConfiguration.cpp); None skips a field."""
        enc = lambda q: None if q is None else str(q).encode()
        self._check(self._L.ovl_load_configuration(self._ctx, enc(u_path), enc(e_path)))

    def device_modes(self):
        psi, mid, nbytes = C.c_void_p(), C.c_void_p(), C.c_size_t()
        self._check(self._L.ovl_device_modes(self._ctx, C.byref(psi), C.byref(mid), C.byref(nbytes)))
        return psi.value, mid.value, nbytes.value

    def profile(self, on: bool = True):
        """Starts (clearing) or stops per-kernel CUDA-event timing."""
        self._check(self._L.ovl_profile_enable(self._ctx, 1 if on else 0))

    def profile_read(self) -> dict:
        """{kind: (total ms, launches)} for kinds hop, axpy, links, obs."""
        ms = np.zeros(len(_lib.PROF_KINDS))
        n = (C.c_uint64 * len(_lib.PROF_KINDS))()
        self._check(self._L.ovl_profile_read(self._ctx, _dp(ms), n))
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(_lib.PROF_KINDS)}

    @property
    def launch_count(self) -> int:
        v = C.c_uint64(0)
        self._check(self._L.ovl_launch_count(self._ctx, C.byref(v)))
        return v.value


class Ensemble:
    """Independent trajectories of mixed lattice sizes stepped together
    (ovl_ensemble_*): one batched launch per half step and per link update,
    one CUDA graph per leapfrog step.  members: a list of Params (Wilson, fused
    form, one precision).  ens[i] is member i's Context (set links, modes,
    measure); step(n) advances all of them."""

    def __init__(self, members):
        self._L = _lib.lib()
        self.params = [m if isinstance(m, Params) else Params(**m) for m in members]
        arr = (_lib.ovl_params * len(self.params))(*[p.to_c() for p in self.params])
        self._e = C.c_void_p()
        rc = self._L.ovl_ensemble_create(arr, len(self.params), C.byref(self._e))
        if rc != 0:
            raise OvlError(rc, self._L.ovl_ensemble_last_error(None).decode())
        self.members = []
        for i, p in enumerate(self.params):
            h = C.c_void_p()
            self._check(self._L.ovl_ensemble_member(self._e, i, C.byref(h)))
            self.members.append(Context._member(h, p, self))

    def _check(self, rc: int):
        if rc != 0:
            raise OvlError(rc, self._L.ovl_ensemble_last_error(self._e).decode())

    def __len__(self):
        return len(self.members)

    def __getitem__(self, i) -> Context:
        return self.members[i]

    def step(self, nsteps: int = 1):
        self._check(self._L.ovl_ensemble_step(self._e, int(nsteps)))

    def add(self, params) -> Context:
        """Admits a member (continuous batching); returns its Context."""
        p = params if isinstance(params, Params) else Params(**params)
        cp = p.to_c()
        idx = C.c_int(0)
        self._check(self._L.ovl_ensemble_add(self._e, C.byref(cp), C.byref(idx)))
        h = C.c_void_p()
        self._check(self._L.ovl_ensemble_member(self._e, idx.value, C.byref(h)))
        m = Context._member(h, p, self)
        self.params.append(p)
        self.members.append(m)
        return m

    def remove(self, index: int):
        """Retires member `index` (its context is destroyed; later members move down)."""
        m = self.members[index]
        self._check(self._L.ovl_ensemble_remove(self._e, int(index)))
        m._ctx = C.c_void_p()
        del self.members[index]
        del self.params[index]

    def charges(self) -> np.ndarray:
        """[members, 4]: N_V, N_5, PS, WA of each member."""
        o = np.empty((len(self.members), 4))
        self._check(self._L.ovl_ensemble_charges(self._e, _dp(o)))
        return o

    def set_tile(self, sites: int):
        """Tile shape of the batched hop: 0 tune on the next step, 8 or 4 sites per
        CTA, 16 packed-pair tiles (8 sites x 256 modes per CTA; FP32 two-colour members)."""
        self._check(self._L.ovl_ensemble_set_tile(self._e, int(sites)))

    def info(self) -> dict:
        sites, launches = C.c_int(0), C.c_uint64(0)
        ms = np.zeros(_lib.ENSEMBLE_TILES)
        self._check(self._L.ovl_ensemble_info(self._e, C.byref(sites), _dp(ms), C.byref(launches)))
        return {"sites": sites.value, "tile_ms": {8: float(ms[0]), 4: float(ms[1]), 16: float(ms[2])},
                "launches": launches.value}

    def synchronize(self):
        self._check(self._L.ovl_ensemble_synchronize(self._e))

    @property
    def stream(self) -> int:
        return int(self._L.ovl_ensemble_stream(self._e))

    def close(self):
        if self._e:
            for m in self.members:
                m._ctx = C.c_void_p()
            self._L.ovl_ensemble_destroy(self._e)
            self._e = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
