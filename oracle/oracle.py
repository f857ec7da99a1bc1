"""ctypes wrapper of the CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, as the checker.  The product package never imports it.
"""

from __future__ import annotations

import ctypes
import importlib
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_lbm = importlib.import_module("2d_nnf_lbm_b200.lbm2d")
LbmParams = _lbm.LbmParams


class OracleOpts(ctypes.Structure):
    _fields_ = [
        ("omega_chain", ctypes.c_int32),
        ("phi_on_the_fly", ctypes.c_int32),
        ("stale_dpw_init", ctypes.c_double),
    ]


def lib_path() -> str:
    return os.path.join(_HERE, "liblbm_oracle.so")


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return lib_path()


_LIB = None


def load():
    global _LIB
    if _LIB is None:
        if not os.path.exists(lib_path()):
            build()
        lib = ctypes.CDLL(lib_path())
        P = ctypes.POINTER
        vp = ctypes.c_void_p
        dp = P(ctypes.c_double)
        ip = P(ctypes.c_int32)
        sigs = {
            "oracle_create": ([P(LbmParams), P(OracleOpts), P(vp)], ctypes.c_int),
            "oracle_destroy": ([vp], None),
            "oracle_set_particles": ([vp, ctypes.c_int32, dp], ctypes.c_int),
            "oracle_step": ([vp, ctypes.c_int32], ctypes.c_int),
            "oracle_kk": ([vp], ctypes.c_int64),
            "oracle_get_particles": ([vp, dp], ctypes.c_int),
            "oracle_get_field": ([vp, ctypes.c_int32, dp], ctypes.c_int),
            "oracle_get_image": ([vp, ip], ctypes.c_int),
            "oracle_get_f": ([vp, dp], ctypes.c_int),
            "oracle_get_next_post_collision": ([vp, dp, dp], ctypes.c_int),
            "oracle_get_series": ([vp, dp, ctypes.c_int32, ip], ctypes.c_int),
            "oracle_series_record_len": ([vp], ctypes.c_int),
            "oracle_mean_density": ([vp], ctypes.c_double),
            "oracle_get_state_particles": ([vp, dp], ctypes.c_int),
            "oracle_compute_error": ([vp, dp], ctypes.c_int),
        }
        for name, (args, res) in sigs.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _LIB = lib
    return _LIB


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


# the inputs a tangent run can carry the derivative of (lbm_oracle.h)
SEEDS = {"tau_y": 0, "nu": 1, "rho_p": 2, "x0": 3, "y0": 4}
_TLIB = None


def tangent_lib_path() -> str:
    return os.path.join(_HERE, "liblbm_oracle_tangent.so")


def load_tangent():
    """The tangent build: the oracle's source compiled with every real a
    value and its derivative (oracle_dual.h)."""
    global _TLIB
    if _TLIB is None:
        if not os.path.exists(tangent_lib_path()):
            build()
        lib = ctypes.CDLL(tangent_lib_path())
        P = ctypes.POINTER
        vp = ctypes.c_void_p
        dp = P(ctypes.c_double)
        sigs = {
            "oracle_create_tangent": ([P(LbmParams), P(OracleOpts), ctypes.c_int32, ctypes.c_int32,
                                       P(vp)], ctypes.c_int),
            "oracle_destroy": ([vp], None),
            "oracle_set_particles": ([vp, ctypes.c_int32, dp], ctypes.c_int),
            "oracle_step": ([vp, ctypes.c_int32], ctypes.c_int),
            "oracle_kk": ([vp], ctypes.c_int64),
            "oracle_get_particles": ([vp, dp], ctypes.c_int),
            "oracle_get_particles_tangent": ([vp, dp], ctypes.c_int),
        }
        for name, (args, res) in sigs.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _TLIB = lib
    return _TLIB


class Oracle:
    """Same call sequence as ``Simulation`` but on the CPU restatement."""

    def __init__(self, params, omega_chain: int = 0, phi_on_the_fly: int = 0,
                 stale_dpw_init: float = float("inf")):
        self.lib = load()
        self.params = params.copy()
        self.opts = OracleOpts(omega_chain, phi_on_the_fly, stale_dpw_init)
        self._h = ctypes.c_void_p()
        rc = self.lib.oracle_create(ctypes.byref(self.params), ctypes.byref(self.opts), ctypes.byref(self._h))
        if rc != 0:
            raise _lbm.LbmError(rc, "oracle_create")
        self.n1x, self.n1y = params.nx + 1, params.ny + 1
        self.np = 0

    def close(self):
        if self._h:
            self.lib.oracle_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_particles(self, pin):
        pin = np.ascontiguousarray(pin, dtype=np.float64).reshape(-1, _lbm.LBM_PIN)
        rc = self.lib.oracle_set_particles(self._h, pin.shape[0], _dp(pin))
        if rc != 0:
            raise _lbm.LbmError(rc, "oracle_set_particles")
        self.np = pin.shape[0]

    def step(self, n=1):
        rc = self.lib.oracle_step(self._h, int(n))
        if rc != 0:
            raise _lbm.LbmError(rc, "oracle_step")

    @property
    def kk(self):
        return int(self.lib.oracle_kk(self._h))

    def particles(self):
        out = np.zeros((max(self.np, 1), _lbm.LBM_POUT))
        self.lib.oracle_get_particles(self._h, _dp(out))
        return out[: self.np]

    def state_particles(self):
        out = np.zeros((max(self.np, 1), _lbm.LBM_STATE_PER))
        self.lib.oracle_get_state_particles(self._h, _dp(out))
        return out[: self.np]

    def field(self, name):
        out = np.zeros(self.n1x * self.n1y)
        rc = self.lib.oracle_get_field(self._h, _lbm.FIELDS[name], _dp(out))
        if rc != 0:
            raise _lbm.LbmError(rc, "oracle_get_field")
        return out.reshape(self.n1y, self.n1x)

    def image(self):
        out = np.zeros(self.n1x * self.n1y, dtype=np.int32)
        self.lib.oracle_get_image(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
        return out.reshape(self.n1y, self.n1x)

    def f(self):
        out = np.zeros(9 * self.n1x * self.n1y)
        self.lib.oracle_get_f(self._h, _dp(out))
        return out

    def next_post_collision(self):
        out = np.zeros(9 * self.n1x * self.n1y)
        om = np.zeros(self.n1x * self.n1y)
        self.lib.oracle_get_next_post_collision(self._h, _dp(out), _dp(om))
        return out, om

    def series(self):
        ln = self.lib.oracle_series_record_len(self._h)
        chunks = []
        while True:
            buf = np.zeros((4096, ln))
            n = ctypes.c_int32()
            self.lib.oracle_get_series(self._h, _dp(buf), 4096, ctypes.byref(n))
            if n.value:
                chunks.append(buf[: n.value].copy())
            if n.value < 4096:
                break
        return np.concatenate(chunks) if chunks else np.zeros((0, ln))

    def mean_density(self):
        return float(self.lib.oracle_mean_density(self._h))

    def compute_error(self):
        er = ctypes.c_double()
        rc = self.lib.oracle_compute_error(self._h, ctypes.byref(er))
        if rc != 0:
            raise _lbm.LbmError(rc, "oracle_compute_error")
        return er.value


class TangentOracle(Oracle):
    """The oracle run in forward-mode derivative numbers: the same values as
    ``Oracle`` and, beside them, their derivatives with respect to one input
    (``which`` in SEEDS; ``disk`` for rho_p, x0, y0)."""

    def __init__(self, params, which: str, disk: int = -1, omega_chain: int = 0):
        self.lib = load_tangent()
        self.params = params.copy()
        self.opts = OracleOpts(omega_chain, 0, float("inf"))
        self._h = ctypes.c_void_p()
        rc = self.lib.oracle_create_tangent(ctypes.byref(self.params), ctypes.byref(self.opts),
                                            SEEDS[which], int(disk), ctypes.byref(self._h))
        if rc != 0:
            raise _lbm.LbmError(rc, "oracle_create_tangent")
        self.n1x, self.n1y = params.nx + 1, params.ny + 1
        self.np = 0

    def particles_tangent(self):
        out = np.zeros((max(self.np, 1), _lbm.LBM_POUT))
        self.lib.oracle_get_particles_tangent(self._h, _dp(out))
        return out[: self.np]
