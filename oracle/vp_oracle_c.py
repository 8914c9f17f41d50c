"""ctypes front end of the OpenMP C restatement (oracle/vp_oracle_c.c).

TEST INFRASTRUCTURE ONLY: used as the timed CPU baseline in bench.py and as a faster checker in
the tests. Build it with ``make -C oracle``.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libvporacle.so")
_lib = None

_D = ctypes.POINTER(ctypes.c_double)


class _Grid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("nv", ctypes.c_int), ("xs", _D), ("vs", _D),
                ("dx", ctypes.c_double), ("dv", ctypes.c_double),
                ("period_x", ctypes.c_double), ("period_v", ctypes.c_double)]


def _load():
    global _lib
    if _lib is None and os.path.exists(_LIB_PATH):
        lib = ctypes.CDLL(_LIB_PATH)
        lib.vpo_threads.restype = ctypes.c_int
        lib.vpo_forward.argtypes = [ctypes.POINTER(_Grid), ctypes.c_double, _D, _D, _D, ctypes.c_int,
                                    _D, _D, _D, _D]
        lib.vpo_backward.argtypes = [ctypes.POINTER(_Grid), ctypes.c_double, _D, _D, _D, ctypes.c_int,
                                     _D, _D, _D, _D, _D, _D, _D]
        _lib = lib
    return _lib


def available() -> bool:
    return _load() is not None


def threads() -> int:
    return int(_load().vpo_threads())


def _p(a):
    return None if a is None else a.ctypes.data_as(_D)


def _c(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


class _Bound:
    def __init__(self, g):
        self.xs = _c(g.xs)
        self.vs = _c(g.vs)
        self.s = _Grid(int(g.nx), int(g.nv), _p(self.xs), _p(self.vs), float(g.dx), float(g.dv),
                       float(g.period_x), float(g.period_v))


def forward(g, dt, f_eq, f_iv, H, n_steps):
    """Legacy forward loop: (f_final, f_hist, E_hist, ee_hist), float64."""
    lib = _load()
    b = _Bound(g)
    nx, nv = int(g.nx), int(g.nv)
    f_eq, f_iv, H = _c(f_eq), _c(f_iv), _c(H)
    f_final = np.empty((nx, nv))
    f_hist = np.empty((max(n_steps, 1), nx, nv))
    E_hist = np.empty((n_steps, nx))
    ee_hist = np.empty(n_steps)
    rc = lib.vpo_forward(ctypes.byref(b.s), float(dt), _p(f_eq), _p(f_iv), _p(H), int(n_steps),
                         _p(f_final), _p(f_hist), _p(E_hist), _p(ee_hist))
    if rc != 0:
        raise MemoryError("vpo_forward failed")
    if n_steps == 0:
        f_final = f_iv.copy()
    return f_final, f_hist[:n_steps], E_hist, ee_hist


def backward(g, dt, f_eq, f_iv, H, n_steps, f_hist, g_f_final, g_f_hist, g_E_hist, g_ee_hist):
    """Legacy adjoint: (g_f_iv, g_H), float64."""
    lib = _load()
    b = _Bound(g)
    nx, nv = int(g.nx), int(g.nv)
    f_eq, f_iv, H, f_hist = _c(f_eq), _c(f_iv), _c(H), _c(f_hist)
    g_ff, g_fh, g_Eh, g_ee = _c(g_f_final), _c(g_f_hist), _c(g_E_hist), _c(g_ee_hist)
    g_fiv = np.empty((nx, nv))
    g_H = np.empty(nx)
    rc = lib.vpo_backward(ctypes.byref(b.s), float(dt), _p(f_eq), _p(f_iv), _p(H), int(n_steps),
                          _p(f_hist), _p(g_ff), _p(g_fh), _p(g_Eh), _p(g_ee), _p(g_fiv), _p(g_H))
    if rc != 0:
        raise MemoryError("vpo_backward failed")
    return g_fiv, g_H


def forward_backward(g, dt, f_eq, f_iv, H, n_steps):
    """Forward plus the adjoint of J = sum(ee)*dt (the benchmark's unit of work)."""
    fwd = forward(g, dt, f_eq, f_iv, H, n_steps)
    backward(g, dt, f_eq, f_iv, H, n_steps, fwd[1], None, None, None, np.full(n_steps, float(dt)))
    return n_steps
