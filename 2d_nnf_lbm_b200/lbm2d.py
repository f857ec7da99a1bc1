"""ctypes binding of the C ABI declared in include/lbm2d.h.

The reference drives its hot path from PROGRAM MAIN by direct subroutine
calls (1_Disk_Newtonian/D2Q9_1P_Validated_20190530.f90:97-399).  This module
exposes the same sequence as a ``Simulation`` object: create (set-up and
INITIALIZE, C1:110-215), ``set_particles`` (the particle read, C1:170-179),
``step`` (the time-loop body, C1:241-319) and getters for the particle state,
fields and time series that the reference writes to its output files.
Errors come back as ``LbmError`` carrying the library's negative status code,
the way the reference STOPs on an invalid relaxation time (C1:127-130).
"""

from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))

# ---- constants mirrored from include/lbm2d.h -------------------------------
LBM_OK = 0
ERRORS = {
    -1: "LBM_E_INVALID",
    -2: "LBM_E_TAU",
    -3: "LBM_E_NOMEM",
    -4: "LBM_E_CUDA",
    -5: "LBM_E_NAN",
    -6: "LBM_E_TIMEOUT",
    -7: "LBM_E_OVERFLOW",
    -8: "LBM_E_STATE",
    -9: "LBM_E_PARTICLE",
    -10: "LBM_E_ABI",
    -11: "LBM_E_SCRATCH",
    -12: "LBM_E_BOUNDS",
}
LBM_FP64, LBM_FP32_SHIFTED = 0, 1
LBM_BC_ZOUHE, LBM_BC_HALFWAY_BB, LBM_BC_EQUILIBRIUM = 0, 1, 2
LBM_MOTION_FREE, LBM_MOTION_OSCILLATE = 0, 1
LBM_STRAIN_MEQ, LBM_STRAIN_FEQ = 0, 1
LBM_NEWTONIAN, LBM_BINGHAM, LBM_CASSON = 0, 1, 2
LBM_RATES_FIXED_Q, LBM_RATES_Q_OF_OMEGA = 0, 1
LBM_WALL_MIRROR, LBM_WALL_OFFSET, LBM_WALL_NONE = 0, 1, 2
LBM_COLLISION_MRT, LBM_COLLISION_BGK = 0, 1
LBM_CONTACT_DPP, LBM_CONTACT_STALE_DPW = 0, 1
LBM_PIN, LBM_POUT, LBM_STATE_PER = 8, 16, 20
LBM_SERIES_HEAD, LBM_SERIES_PER = 2, 12
LBM_OBJ_X, LBM_OBJ_Y, LBM_OBJ_U, LBM_OBJ_V, LBM_OBJ_W = 0, 1, 3, 4, 5
LBM_GRAD_TAU_Y, LBM_GRAD_NU, LBM_GRAD_HEAD, LBM_GRAD_PER = 0, 1, 2, 3
LBM_ADJ_MAX_PARTICLES = 64
FIELDS = {
    "ux": 0, "uy": 1, "rho": 2, "phi": 3, "gx": 4, "gy": 5,
    "tau11": 6, "tau22": 7, "tau12": 8, "omega": 9,
}


def r4(x) -> float:
    """Value a Fortran default-kind REAL(4) literal holds, widened to double.

    ``PI=3.14159265359`` in a DOUBLE PRECISION PARAMETER holds
    3.1415927410125732 (C1:3); the same rule applies to every literal
    without a D exponent (C1:23, C1:881, C1:1229, C6:939).
    """
    return float(np.float32(x))


def r4div(a, b) -> float:
    """REAL(4) quotient of two REAL(4) literals, e.g. ``1./36.`` (C1:881)."""
    return float(np.float32(a) / np.float32(b))


class LbmParams(ctypes.Structure):
    """Mirror of ``lbm_params`` (include/lbm2d.h)."""

    _fields_ = [
        ("struct_size", ctypes.c_int32),
        ("nx", ctypes.c_int32),
        ("ny", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("bc", ctypes.c_int32),
        ("rheology", ctypes.c_int32),
        ("rate_set", ctypes.c_int32),
        ("wall_model", ctypes.c_int32),
        ("contact_test", ctypes.c_int32),
        ("integrate_angle", ctypes.c_int32),
        ("series_every", ctypes.c_int32),
        ("series_particles", ctypes.c_int32),
        ("series_capacity", ctypes.c_int32),
        ("record_stress", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("motion", ctypes.c_int32),
        ("nu", ctypes.c_double),
        ("rho0", ctypes.c_double),
        ("s_e", ctypes.c_double),
        ("s_eps", ctypes.c_double),
        ("s_q", ctypes.c_double),
        ("d_mrt", ctypes.c_double),
        ("inv_six", ctypes.c_double),
        ("w_init", ctypes.c_double * 3),
        ("pi", ctypes.c_double),
        ("zeta", ctypes.c_double),
        ("gravity", ctypes.c_double),
        ("tau_y", ctypes.c_double),
        ("m_pap", ctypes.c_double),
        ("gamma_min", ctypes.c_double),
        ("rep_zeta", ctypes.c_double),
        ("eps_p", ctypes.c_double),
        ("eps_w", ctypes.c_double),
        ("e_p", ctypes.c_double),
        ("e_w", ctypes.c_double),
        ("c_ij", ctypes.c_double),
        ("wall_mirror_top", ctypes.c_double),
        ("wall_mirror_left", ctypes.c_double),
        ("osc_u", ctypes.c_double),
        ("osc_period", ctypes.c_double),
        ("strain_model", ctypes.c_int32),
        ("collision", ctypes.c_int32),
    ]

    def __init__(self, **kw):
        super().__init__()
        self.struct_size = ctypes.sizeof(LbmParams)
        fill_c1_defaults(self)
        for k, v in kw.items():
            setattr(self, k, v)

    def copy(self, **kw) -> "LbmParams":
        p = LbmParams()
        ctypes.memmove(ctypes.byref(p), ctypes.byref(self), ctypes.sizeof(LbmParams))
        for k, v in kw.items():
            setattr(p, k, v)
        return p

    def omega(self) -> float:
        """OMEGA = 1.0/(3.*NU+0.5) (C1:112)."""
        return 1.0 / (3.0 * self.nu + 0.5)

    def as_dict(self) -> dict:
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            d[name] = list(v) if name == "w_init" else v
        return d


def fill_c1_defaults(p: LbmParams) -> None:
    """Constants of 1_Disk_Newtonian as the compiled Fortran holds them.

    Same values as ``lbm_params_init`` in the library (C1:2-93, C1:1035-1042,
    C1:701-703, C1:157-168).
    """
    p.nx, p.ny = 240, 720
    p.precision = LBM_FP64
    p.bc = LBM_BC_ZOUHE
    p.rheology = LBM_NEWTONIAN
    p.rate_set = LBM_RATES_FIXED_Q
    p.wall_model = LBM_WALL_MIRROR
    p.contact_test = LBM_CONTACT_STALE_DPW
    p.integrate_angle = 0
    p.series_every = 1
    p.series_particles = 1
    p.series_capacity = 4096
    p.record_stress = 0
    p.device = 0
    p.nu = r4(0.05)
    p.rho0 = 1.0
    p.s_e, p.s_eps, p.s_q = r4(1.1), 1.0, r4(1.2)
    p.d_mrt = r4div(1.0, 36.0)
    p.inv_six = r4div(1.0, 6.0)
    p.w_init[0] = r4div(2.0, 9.0)
    p.w_init[1] = r4div(1.0, 18.0)
    p.w_init[2] = r4div(1.0, 36.0)
    p.pi = r4(3.14159265359)
    p.zeta = 1.0
    # A_G = -9.81/C_G with C_L = 0.25/30, C_T = C_L**2*NU/0.1, C_G = C_L*0.01/C_T**2
    c_l = r4(0.25) / 30.0
    c_t = (c_l * c_l) * p.nu / r4(0.1)
    c_g = c_l * r4(0.01) / (c_t * c_t)
    p.gravity = -r4(9.81) / c_g
    p.tau_y = 1.0 * p.nu * 1.0 / 30.0
    p.m_pap = r4(1.0e8)
    p.gamma_min = r4(1.0e-15)
    p.rep_zeta = 2.0
    p.eps_p = r4(1.0e5)
    p.eps_w = 0.5 * p.eps_p
    p.e_p = r4(2.0e5)
    p.e_w = 0.5 * p.e_p
    p.c_ij = glowinski_cij(r4(1.25), 1.0, p.gravity, p.pi, 30.0)
    edge3 = 0.5 * float(p.ny) + 0.5 * (2.0 * float(p.ny))
    edge4 = 0.5 * float(p.nx) - 0.5 * (2.0 * float(p.nx))
    p.wall_mirror_top = 2.0 * edge3
    p.wall_mirror_left = 2.0 * edge4


def glowinski_cij(rho_s: float, rho_f: float, a_g: float, pi: float, diam: float) -> float:
    """CIJ=-(RHO_S-RHO_F)*A_G*PI*0.5*D*0.5*D, evaluated left to right (C1:701)."""
    return -((((((rho_s - rho_f) * a_g) * pi) * 0.5) * diam) * 0.5) * diam


def mirror_edges(p: LbmParams) -> None:
    """Recompute 2*WALL%EDGE(3), 2*WALL%EDGE(4) for the current NX, NY (C1:157-164)."""
    edge3 = 0.5 * float(p.ny) + 0.5 * (2.0 * float(p.ny))
    edge4 = 0.5 * float(p.nx) - 0.5 * (2.0 * float(p.nx))
    p.wall_mirror_top = 2.0 * edge3
    p.wall_mirror_left = 2.0 * edge4


class LbmObjective(ctypes.Structure):
    """lbm_objective: J = mean of record field `component` of disk `particle`
    over steps n0..n1."""
    _fields_ = [
        ("struct_size", ctypes.c_int32),
        ("particle", ctypes.c_int32),
        ("component", ctypes.c_int32),
        ("checkpoint_every", ctypes.c_int32),
        ("n0", ctypes.c_int64),
        ("n1", ctypes.c_int64),
    ]


class LbmError(RuntimeError):
    def __init__(self, code: int, where: str, detail: str = ""):
        self.code = code
        name = ERRORS.get(code, str(code))
        super().__init__(f"{where}: {name} ({code}){(': ' + detail) if detail else ''}")


def library_path() -> str:
    """liblbm2d.so of the package directory, or the library LBM2D_LIBRARY
    names (e.g. the checked build, liblbm2d_checked.so)."""
    return os.environ.get("LBM2D_LIBRARY") or os.path.join(_HERE, "liblbm2d.so")


_LIB = None


def load_library():
    """Load liblbm2d.so from the package directory; raise if it is missing."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not os.path.exists(path):
        raise OSError(
            f"{path} is missing: build it with python -c 'import __graft_entry__ as g; g.build()' "
            "(there is no CPU fallback)"
        )
    lib = ctypes.CDLL(path)
    P = ctypes.POINTER
    vp = ctypes.c_void_p
    dp = P(ctypes.c_double)
    ip = P(ctypes.c_int32)
    sigs = {
        "lbm_params_init": ([P(LbmParams)], ctypes.c_int),
        "lbm_create": ([P(LbmParams), P(vp)], ctypes.c_int),
        "lbm_destroy": ([vp], ctypes.c_int),
        "lbm_set_particles": ([vp, ctypes.c_int32, dp], ctypes.c_int),
        "lbm_step": ([vp, ctypes.c_int32], ctypes.c_int),
        "lbm_get_step": ([vp, P(ctypes.c_int64)], ctypes.c_int),
        "lbm_get_particles": ([vp, dp], ctypes.c_int),
        "lbm_get_field": ([vp, ctypes.c_int32, dp], ctypes.c_int),
        "lbm_get_image": ([vp, ip], ctypes.c_int),
        "lbm_get_series": ([vp, dp, ctypes.c_int32, ip], ctypes.c_int),
        "lbm_series_record_len": ([vp, ip], ctypes.c_int),
        "lbm_get_mean_density": ([vp, dp], ctypes.c_int),
        "lbm_compute_error": ([vp, dp], ctypes.c_int),
        "lbm_get_state": ([vp, dp, dp, dp], ctypes.c_int),
        "lbm_set_state": ([vp, ctypes.c_int64, dp, dp, ctypes.c_int32, dp], ctypes.c_int),
        "lbm_get_status": ([vp], ctypes.c_int),
        "lbm_selftest_wait": ([vp, ctypes.c_int32], ctypes.c_int),
        "lbm_get_stream": ([vp, P(vp)], ctypes.c_int),
        "lbm_profile": ([vp, ctypes.c_int32], ctypes.c_int),
        "lbm_profile_read": ([vp, dp, P(ctypes.c_int64)], ctypes.c_int),
        "lbm_strerror": ([ctypes.c_int], ctypes.c_char_p),
        "lbm_checked_build": ([], ctypes.c_int32),
        "lbm_fields_noalloc": ([P(LbmParams), vp, ctypes.c_int32, vp, vp, vp], ctypes.c_int),
        "lbm_adjoint": ([vp, P(LbmObjective), dp, dp], ctypes.c_int),
        "lbm_batch_create": ([P(LbmParams), ctypes.c_int32, P(vp)], ctypes.c_int),
        "lbm_batch_sim": ([vp, ctypes.c_int32], vp),
        "lbm_batch_step": ([vp, ctypes.c_int32], ctypes.c_int),
        "lbm_batch_tuning": ([vp, ip, ip, ip], ctypes.c_int),
        "lbm_batch_set_tuning": ([vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32], ctypes.c_int),
        "lbm_batch_destroy": ([vp], ctypes.c_int),
        "lbm_batch_stream": ([vp, P(vp)], ctypes.c_int),
    }
    for name, (args, res) in sigs.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _LIB = lib
    return lib


def _dptr(a: Optional[np.ndarray]):
    if a is None:
        return ctypes.POINTER(ctypes.c_double)()
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Simulation:
    """One lattice + particle system on one GPU, driven through the C ABI."""

    def __init__(self, params: LbmParams, _handle=None):
        self.lib = load_library()
        self.params = params.copy()
        self._owned = _handle is None
        self._h = ctypes.c_void_p()
        if _handle is None:
            self._check(self.lib.lbm_create(ctypes.byref(self.params), ctypes.byref(self._h)),
                        "lbm_create")
        else:
            self._h = ctypes.c_void_p(_handle)
        self.np = 0
        self.n1x, self.n1y = params.nx + 1, params.ny + 1

    def _check(self, rc: int, where: str) -> None:
        if rc != LBM_OK:
            msg = self.lib.lbm_strerror(rc)
            raise LbmError(rc, where, msg.decode() if msg else "")

    def close(self) -> None:
        if self._h and self._owned:
            self.lib.lbm_destroy(self._h)
        self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- particles --------------------------------------------------------
    def set_particles(self, pin: np.ndarray) -> None:
        """pin: (np, 8) array of x, y, angle, u, v, omega, diam, rho_p."""
        pin = np.ascontiguousarray(pin, dtype=np.float64).reshape(-1, LBM_PIN)
        self._check(self.lib.lbm_set_particles(self._h, pin.shape[0], _dptr(pin)), "lbm_set_particles")
        self.np = pin.shape[0]

    def step(self, nsteps: int = 1) -> None:
        self._check(self.lib.lbm_step(self._h, int(nsteps)), "lbm_step")

    @property
    def kk(self) -> int:
        v = ctypes.c_int64()
        self._check(self.lib.lbm_get_step(self._h, ctypes.byref(v)), "lbm_get_step")
        return v.value

    def particles(self) -> np.ndarray:
        out = np.zeros((max(self.np, 1), LBM_POUT))
        self._check(self.lib.lbm_get_particles(self._h, _dptr(out)), "lbm_get_particles")
        return out[: self.np]

    def field(self, name: str) -> np.ndarray:
        """Field as (NY+1, NX+1) array, i.e. out[j, i] = F(i, j)."""
        out = np.zeros(self.n1x * self.n1y)
        self._check(self.lib.lbm_get_field(self._h, FIELDS[name], _dptr(out)), "lbm_get_field")
        return out.reshape(self.n1y, self.n1x)

    def image(self) -> np.ndarray:
        out = np.zeros(self.n1x * self.n1y, dtype=np.int32)
        self._check(
            self.lib.lbm_get_image(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))),
            "lbm_get_image",
        )
        return out.reshape(self.n1y, self.n1x)

    def series(self, max_records: int = 1 << 20) -> np.ndarray:
        ln = ctypes.c_int32()
        self._check(self.lib.lbm_series_record_len(self._h, ctypes.byref(ln)), "lbm_series_record_len")
        chunks = []
        cap = min(4096, max(64, int(self.params.series_capacity)))
        while True:
            buf = np.empty((cap, ln.value))
            n = ctypes.c_int32()
            self._check(self.lib.lbm_get_series(self._h, _dptr(buf), cap, ctypes.byref(n)), "lbm_get_series")
            if n.value:
                chunks.append(buf[: n.value])
            if n.value < cap or sum(len(c) for c in chunks) >= max_records:
                break
        return np.concatenate(chunks) if chunks else np.zeros((0, ln.value))

    def series_into(self, out: np.ndarray) -> int:
        """lbm_get_series into a caller-kept C-contiguous float64 array of
        shape (records, record length); returns the number of records read."""
        if out.dtype != np.float64 or not out.flags.c_contiguous or out.ndim != 2:
            raise ValueError("out must be a C-contiguous 2-D float64 array")
        n = ctypes.c_int32()
        self._check(self.lib.lbm_get_series(self._h, _dptr(out), out.shape[0], ctypes.byref(n)),
                    "lbm_get_series")
        return n.value

    def series_record_len(self) -> int:
        ln = ctypes.c_int32()
        self._check(self.lib.lbm_series_record_len(self._h, ctypes.byref(ln)), "lbm_series_record_len")
        return ln.value

    def mean_density(self) -> float:
        v = ctypes.c_double()
        self._check(self.lib.lbm_get_mean_density(self._h, ctypes.byref(v)), "lbm_get_mean_density")
        return v.value

    def compute_error(self) -> float:
        """COMPUTEERROR (C1:1592-1612): relative velocity change since the
        previous call (since the initial state on the first call)."""
        v = ctypes.c_double()
        self._check(self.lib.lbm_compute_error(self._h, ctypes.byref(v)), "lbm_compute_error")
        return v.value

    def get_state(self):
        nn = self.n1x * self.n1y
        f = np.zeros(9 * nn)
        om = np.zeros(nn)
        ps = np.zeros((max(self.np, 1), LBM_STATE_PER))
        self._check(self.lib.lbm_get_state(self._h, _dptr(f), _dptr(om), _dptr(ps)), "lbm_get_state")
        return f, om, ps[: self.np]

    def set_state(self, kk: int, f: np.ndarray, omega: Optional[np.ndarray], parts: np.ndarray) -> None:
        f = np.ascontiguousarray(f, dtype=np.float64)
        om = None if omega is None else np.ascontiguousarray(omega, dtype=np.float64)
        parts = np.ascontiguousarray(parts, dtype=np.float64).reshape(-1, LBM_STATE_PER)
        self._check(
            self.lib.lbm_set_state(self._h, int(kk), _dptr(f), _dptr(om), parts.shape[0], _dptr(parts)),
            "lbm_set_state",
        )
        self.np = parts.shape[0]

    def status(self) -> int:
        return int(self.lib.lbm_get_status(self._h))

    def selftest_wait(self, limit: int = 1024) -> None:
        """Run one bounded device wait that cannot complete (the failure path
        of the kernels' waits); afterwards status() is LBM_E_TIMEOUT."""
        self._check(self.lib.lbm_selftest_wait(self._h, int(limit)), "lbm_selftest_wait")

    def stream(self) -> int:
        """The handle's cudaStream_t as an integer (for external events)."""
        s = ctypes.c_void_p()
        self._check(self.lib.lbm_get_stream(self._h, ctypes.byref(s)), "lbm_get_stream")
        return int(s.value or 0)

    def profile(self, enable: bool) -> None:
        self._check(self.lib.lbm_profile(self._h, 1 if enable else 0), "lbm_profile")

    def profile_read(self):
        """(particle_ms, lattice_ms), (particle_launches, lattice_launches)."""
        ms = (ctypes.c_double * 2)()
        n = (ctypes.c_int64 * 2)()
        self._check(self.lib.lbm_profile_read(self._h, ms, n), "lbm_profile_read")
        return (ms[0], ms[1]), (n[0], n[1])

    def adjoint(self, n0: int, n1: int, particle: int = 0, component: int = LBM_OBJ_V,
                checkpoint_every: int = 0):
        """lbm_adjoint from step 0: J = mean of `component` of disk `particle`
        over steps n0..n1 and its gradient, a dict with tau_y, nu and per-disk
        arrays rho_p, x0, y0.  The simulation is left at step n1."""
        obj = LbmObjective(ctypes.sizeof(LbmObjective), particle, component, checkpoint_every,
                           n0, n1)
        g = np.zeros(LBM_GRAD_HEAD + LBM_GRAD_PER * max(self.np, 1))
        v = ctypes.c_double()
        self._check(self.lib.lbm_adjoint(self._h, ctypes.byref(obj), ctypes.byref(v), _dptr(g)),
                    "lbm_adjoint")
        per = g[LBM_GRAD_HEAD:LBM_GRAD_HEAD + LBM_GRAD_PER * self.np].reshape(-1, LBM_GRAD_PER)
        return v.value, {"tau_y": g[LBM_GRAD_TAU_Y], "nu": g[LBM_GRAD_NU],
                         "rho_p": per[:, 0].copy(), "x0": per[:, 1].copy(), "y0": per[:, 2].copy()}


class Batch:
    """lbm_batch_*: independent simulations advanced together, one launch per
    kernel per step.  ``sims[i]`` is a Simulation view of simulation i (set
    its particles, read its state); the batch owns the handles."""

    def __init__(self, params_list):
        self.lib = load_library()
        arr = (LbmParams * len(params_list))(*[p.copy() for p in params_list])
        self._b = ctypes.c_void_p()
        rc = self.lib.lbm_batch_create(arr, len(params_list), ctypes.byref(self._b))
        if rc != LBM_OK:
            raise LbmError(rc, "lbm_batch_create")
        self.sims = [Simulation(p, _handle=self.lib.lbm_batch_sim(self._b, i))
                     for i, p in enumerate(params_list)]

    def step(self, nsteps: int) -> None:
        rc = self.lib.lbm_batch_step(self._b, int(nsteps))
        if rc != LBM_OK:
            raise LbmError(rc, "lbm_batch_step")

    def tuning(self):
        """(tile_x, tile_y, blocks_per_sm); zeros before the first step."""
        v = [ctypes.c_int32() for _ in range(3)]
        self.lib.lbm_batch_tuning(self._b, *[ctypes.byref(x) for x in v])
        return tuple(x.value for x in v)

    def set_tuning(self, tile_x: int, tile_y: int = 0, blocks_per_sm: int = 0) -> None:
        rc = self.lib.lbm_batch_set_tuning(self._b, tile_x, tile_y, blocks_per_sm)
        if rc != LBM_OK:
            raise LbmError(rc, "lbm_batch_set_tuning")

    def batch_stream(self) -> int:
        """The batch's own cudaStream_t (as an integer)."""
        s = ctypes.c_void_p()
        rc = self.lib.lbm_batch_stream(self._b, ctypes.byref(s))
        if rc != LBM_OK:
            raise LbmError(rc, "lbm_batch_stream")
        return int(s.value or 0)

    def close(self) -> None:
        if self._b:
            for s in self.sims:
                s._h = ctypes.c_void_p()
            self.lib.lbm_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
