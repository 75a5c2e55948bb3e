"""ctypes wrapper of the CPU oracle (test infrastructure only).

Used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as
the parity checker; the product (smaug_b200) never imports it.
"""
import ctypes
import os

import numpy as np

from . import build as _build

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _build.LIB
        if not os.path.exists(path):
            path = _build.build()
        L = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        L.or_grid_metric.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int32), dp, dp]
        L.or_boundary.argtypes = [ctypes.c_void_p, dp]
        L.or_cmax.argtypes = [ctypes.c_void_p, dp, dp]
        L.or_advance.argtypes = [ctypes.c_void_p, dp, dp, dp, ctypes.c_int, dp, dp]
        L.or_num_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _dp(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def grid_metric(ndim, n, pos):
    """initgrid restatement: returns (pos_rewritten, delx)."""
    pos = np.ascontiguousarray(pos, dtype=np.float64).copy()
    delx = np.zeros_like(pos)
    nn = (ctypes.c_int32 * 3)(*(list(n) + [1] * (3 - len(n))))
    rc = lib().or_grid_metric(ndim, nn, _dp(pos), _dp(delx))
    if rc:
        raise RuntimeError("or_grid_metric failed: %d" % rc)
    return pos, delx


def boundary(params, w):
    w = np.ascontiguousarray(w, dtype=np.float64).copy()
    rc = lib().or_boundary(ctypes.byref(params), _dp(w))
    if rc:
        raise RuntimeError("or_boundary failed: %d" % rc)
    return w


def cmax(params, w):
    w = np.ascontiguousarray(w, dtype=np.float64)
    out = np.zeros(3)
    rc = lib().or_cmax(ctypes.byref(params), _dp(w), _dp(out))
    if rc:
        raise RuntimeError("or_cmax failed: %d" % rc)
    return out[: params.ndim]


class OracleRun:
    """State of one oracle run: w (reference slot 1 after boundaries)."""

    def __init__(self, params, w, pos):
        self.p = params
        self.pos, self.delx = grid_metric(params.ndim, list(params.n)[: params.ndim], pos)
        self.w = boundary(params, w)
        self.state = np.array([params.dt, 0.0, 0.0])  # dt, t, step counter
        self.cmax = np.zeros(3)
        self.it = 0

    def advance(self, nsteps):
        rc = lib().or_advance(ctypes.byref(self.p), _dp(self.w), _dp(self.pos),
                              _dp(self.delx), int(nsteps), _dp(self.state), _dp(self.cmax))
        if rc:
            raise RuntimeError("or_advance failed: %d" % rc)
        self.it += nsteps
        return self

    @property
    def dt(self):
        return float(self.state[0])

    @property
    def t(self):
        return float(self.state[1])


def num_threads():
    return int(lib().or_num_threads())
