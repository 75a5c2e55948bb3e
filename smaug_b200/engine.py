"""Python binding of the engine's C ABI (include/smaug_b200.h).

Mirrors the reference's host flow (src/iosmaug.c): create from an initial
state (cuinit + initgrid + boundaries), step, copy back (cuupdate), write
.out snapshots (writevacconfig).  All compute runs in libsmaug_b200.so on the
GPU; there is no CPU path.  Errors raise SmaugError with the library message.
"""
import ctypes
import os

import numpy as np

from . import params as _params

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libsmaug_b200.so")

EXPORTS = [
    "smaug_params_default", "smaug_create", "smaug_step", "smaug_get_state", "smaug_get_fields",
    "smaug_set_state", "smaug_get_time", "smaug_get_cmax", "smaug_write_out",
    "smaug_destroy", "smaug_last_error", "smaug_version", "smaug_read_ini",
    "smaug_write_out_host", "smaug_grid_metric", "smaug_step_async", "smaug_sync",
    "smaug_set_stream", "smaug_euler_step_noalloc", "smaug_batch_create", "smaug_batch_step",
    "smaug_batch_get_state", "smaug_batch_get_time", "smaug_batch_launch_shape",
    "smaug_batch_destroy", "smaug_batch_step_async", "smaug_batch_sync", "smaug_batch_set_stream",
    "smaug_adj_create", "smaug_adj_set_driver", "smaug_adj_forward", "smaug_adj_backward",
    "smaug_adj_tape_reserve", "smaug_adj_forward_tape", "smaug_adj_backward_tape",
    "smaug_adj_destroy", "smaug_write_out_async", "smaug_wait_writes",
    "smaug_adj_backward_tape_range", "smaug_batch_tile_shape", "smaug_batch_pin_tile_shape",
    "smaug_batch_persistent", "smaug_batch_pin_form", "smaug_staging", "smaug_set_staging",
]

ERRORS = {1: "invalid", 2: "cuda", 3: "nomem", 4: "io", 5: "format", 6: "unsupported",
          7: "nonfinite"}


class SmaugError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("smaug error %d (%s): %s" % (code, ERRORS.get(code, "?"), msg))
        self.code = code


_lib = None


def lib():
    """Load the engine library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise ImportError("libsmaug_b200.so not built (run __graft_entry__.build() "
                              "or python smaug_b200/build.py)")
        L = ctypes.CDLL(LIBPATH)
        dp = ctypes.POINTER(ctypes.c_double)
        vp = ctypes.c_void_p
        L.smaug_params_default.argtypes = [vp, ctypes.c_int32]
        L.smaug_create.argtypes = [vp, dp, dp, ctypes.POINTER(vp)]
        L.smaug_step.argtypes = [vp, ctypes.c_int32]
        L.smaug_step_async.argtypes = [vp, ctypes.c_int32]
        L.smaug_sync.argtypes = [vp]
        L.smaug_set_stream.argtypes = [vp, vp]
        L.smaug_euler_step_noalloc.argtypes = [vp, vp, vp, dp, dp, vp]
        L.smaug_get_state.argtypes = [vp, dp]
        L.smaug_get_fields.argtypes = [vp, dp, ctypes.c_int32, ctypes.c_int32]
        L.smaug_set_state.argtypes = [vp, dp]
        L.smaug_get_time.argtypes = [vp, ctypes.POINTER(ctypes.c_int64), dp, dp]
        L.smaug_get_cmax.argtypes = [vp, dp]
        L.smaug_staging.argtypes = [vp, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]
        L.smaug_set_staging.argtypes = [vp, ctypes.c_int32]
        L.smaug_write_out.argtypes = [vp, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int32,
                                      ctypes.c_double]
        L.smaug_write_out_async.argtypes = [vp, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int32,
                                            ctypes.c_double]
        L.smaug_wait_writes.argtypes = [vp]
        L.smaug_destroy.argtypes = [vp]
        L.smaug_last_error.restype = ctypes.c_char_p
        L.smaug_version.restype = ctypes.c_char_p
        L.smaug_read_ini.argtypes = [ctypes.c_char_p, ctypes.c_int32,
                                     ctypes.POINTER(ctypes.c_int32), dp, dp,
                                     ctypes.POINTER(ctypes.c_int32), dp]
        L.smaug_write_out_host.argtypes = [ctypes.c_char_p, vp, dp, dp, ctypes.c_char_p,
                                           ctypes.c_int32, ctypes.c_double]
        L.smaug_grid_metric.argtypes = [ctypes.c_int32, ctypes.POINTER(ctypes.c_int32), dp, dp]
        L.smaug_batch_create.argtypes = [ctypes.c_int32, ctypes.POINTER(vp), ctypes.POINTER(dp),
                                         ctypes.POINTER(dp), ctypes.POINTER(vp)]
        L.smaug_batch_step.argtypes = [vp, ctypes.c_int32]
        L.smaug_batch_step_async.argtypes = [vp, ctypes.c_int32]
        L.smaug_batch_sync.argtypes = [vp]
        L.smaug_batch_set_stream.argtypes = [vp, vp]
        L.smaug_batch_get_state.argtypes = [vp, ctypes.c_int32, dp]
        L.smaug_batch_get_time.argtypes = [vp, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64), dp, dp]
        L.smaug_batch_tile_shape.argtypes = [vp, ctypes.POINTER(ctypes.c_int32),
                                             ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_float)]
        L.smaug_batch_pin_tile_shape.argtypes = [vp, ctypes.c_int32, ctypes.c_int32]
        L.smaug_batch_persistent.argtypes = [vp, ctypes.POINTER(ctypes.c_int32),
                                             ctypes.POINTER(ctypes.c_int32),
                                             ctypes.POINTER(ctypes.c_float)]
        L.smaug_batch_pin_form.argtypes = [vp, ctypes.c_int32]
        L.smaug_batch_launch_shape.argtypes = [vp, ctypes.POINTER(ctypes.c_int32),
                                               ctypes.POINTER(ctypes.c_int32),
                                               ctypes.POINTER(ctypes.c_float)]
        L.smaug_batch_destroy.argtypes = [vp]
        L.smaug_adj_create.argtypes = [vp, dp, dp, ctypes.POINTER(vp)]
        L.smaug_adj_set_driver.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.smaug_adj_forward.argtypes = [vp, vp, vp, ctypes.c_double, vp]
        L.smaug_adj_backward.argtypes = [vp, vp, vp, vp, vp, ctypes.c_double, vp]
        L.smaug_adj_tape_reserve.argtypes = [vp, ctypes.c_int32]
        L.smaug_adj_forward_tape.argtypes = [vp, vp, vp, ctypes.c_double, ctypes.c_int32, vp]
        L.smaug_adj_backward_tape.argtypes = [vp, ctypes.c_int32, vp, vp, vp, ctypes.c_double, vp]
        L.smaug_adj_backward_tape_range.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, vp, vp, vp,
                                                    ctypes.c_double, ctypes.c_int32, vp]
        L.smaug_adj_destroy.argtypes = [vp]
        _lib = L
    return _lib


def _check(rc):
    if rc:
        raise SmaugError(rc, lib().smaug_last_error().decode())


def _dp(a):
    if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
        raise TypeError("expected a C-contiguous float64 array")
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def version():
    return lib().smaug_version().decode()


def grid_metric(ndim, n, pos):
    """Host restatement of initgrid: returns (rewritten positions, delx)."""
    pos = np.array(pos, dtype=np.float64, order="C")
    delx = np.zeros_like(pos)
    nn = (ctypes.c_int32 * 3)(*(list(n) + [1] * (3 - len(n))))
    _check(lib().smaug_grid_metric(ndim, nn, _dp(pos), _dp(delx)))
    return pos, delx


def read_ini(path, ndim, n):
    nvar = 4 + 3 * ndim
    shape = tuple(reversed(list(n)[:ndim]))
    w = np.zeros((nvar,) + shape)
    pos = np.zeros((ndim,) + shape)
    nn = (ctypes.c_int32 * 3)(*(list(n) + [1] * (3 - len(n))))
    it = ctypes.c_int32(0)
    t = ctypes.c_double(0.0)
    _check(lib().smaug_read_ini(path.encode(), ndim, nn, _dp(w), _dp(pos), ctypes.byref(it),
                                ctypes.byref(t)))
    return w, pos, int(it.value), float(t.value)


class Engine:
    """One simulation on the current CUDA device."""

    def __init__(self, params, w, pos):
        self.p = params
        self.shape = (params.nvar,) + params.shape
        w = np.ascontiguousarray(w, dtype=np.float64)
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        if w.shape != self.shape:
            raise ValueError("state shape %s, expected %s" % (w.shape, self.shape))
        if pos.shape != (params.ndim,) + params.shape:
            raise ValueError("positions shape %s" % (pos.shape,))
        h = ctypes.c_void_p()
        _check(lib().smaug_create(ctypes.byref(params), _dp(w), _dp(pos), ctypes.byref(h)))
        self.h = h

    def step(self, n=1):
        _check(lib().smaug_step(self.h, int(n)))
        return self

    def step_async(self, n=1):
        """Enqueue n steps on the engine's stream without waiting."""
        _check(lib().smaug_step_async(self.h, int(n)))
        return self

    def sync(self):
        _check(lib().smaug_sync(self.h))

    def set_stream(self, stream_handle):
        """Launch on the given cudaStream_t (an int handle, e.g.
        torch.cuda.current_stream().cuda_stream); None restores the engine's own."""
        _check(lib().smaug_set_stream(self.h, ctypes.c_void_p(stream_handle or None)))

    def state(self, out=None):
        """Copy the state to the host (into `out`, e.g. a pinned buffer, if given)."""
        w = np.zeros(self.shape) if out is None else out
        if w.shape != self.shape:
            raise ValueError("out has shape %s, expected %s" % (w.shape, self.shape))
        _check(lib().smaug_get_state(self.h, _dp(w)))
        return w

    def fields(self, f0, nf, out=None):
        """Copy fields [f0, f0+nf) of the state to the host (into `out`, whose
        leading dimension is nf, if given)."""
        shape = (nf,) + self.shape[1:]
        w = np.zeros(shape) if out is None else out
        if w.shape != shape or not w.flags["C_CONTIGUOUS"]:
            raise ValueError("out has shape %s, expected contiguous %s" % (w.shape, shape))
        _check(lib().smaug_get_fields(self.h, _dp(w), int(f0), int(nf)))
        return w

    def set_state(self, w):
        w = np.ascontiguousarray(w, dtype=np.float64)
        _check(lib().smaug_set_state(self.h, _dp(w)))

    def time(self):
        it = ctypes.c_int64(0)
        t = ctypes.c_double(0)
        dt = ctypes.c_double(0)
        _check(lib().smaug_get_time(self.h, ctypes.byref(it), ctypes.byref(t), ctypes.byref(dt)))
        return int(it.value), float(t.value), float(dt.value)

    def cmax(self):
        c = np.zeros(3)
        _check(lib().smaug_get_cmax(self.h, _dp(c)))
        return c[: self.p.ndim]

    def staging(self):
        """(tma, available): how the 2D stage tiles are staged (0 per-thread
        loads, 1 bulk tensor copies in a persistent grid, 2 bulk tensor
        copies with a block per tile), and whether the grid admits copies."""
        on, av = ctypes.c_int32(0), ctypes.c_int32(0)
        _check(lib().smaug_staging(self.h, ctypes.byref(on), ctypes.byref(av)))
        return int(on.value), bool(av.value)

    def set_staging(self, tma):
        """Staging of the 2D tiles from the next launch on (0 / False
        per-thread loads, 1 / True bulk tensor copies in a persistent grid, 2
        bulk tensor copies with a block per tile); bitwise-identical results."""
        _check(lib().smaug_set_staging(self.h, int(tma)))

    def write_out(self, path, name="test1", it=None, t=None):
        i, tt, _ = self.time()
        _check(lib().smaug_write_out(self.h, path.encode(), name.encode(),
                                     int(i if it is None else it), float(tt if t is None else t)))

    def write_out_async(self, path, name="test1", it=None, t=None):
        """Snapshot the current state to a .out file without waiting: the copy
        is queued on the engine's stream and a host thread writes the file
        (errors surface in wait_writes)."""
        if it is None or t is None:   # smaug_get_time waits for the engine's stream
            i, tt, _ = self.time()
            it = i if it is None else it
            t = tt if t is None else t
        _check(lib().smaug_write_out_async(self.h, path.encode(), name.encode(), int(it), float(t)))

    def wait_writes(self):
        """Wait for the pending write_out_async files; raises the first write error."""
        _check(lib().smaug_wait_writes(self.h))

    def close(self):
        if getattr(self, "h", None):
            lib().smaug_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Batch:
    """An ensemble of independent 2D runs advanced together (RK4): one launch
    per stage for all runs or one persistent launch for several steps, a
    6-step cycle replayed from a CUDA graph; the first 10 steps choose the
    tile shape and the launch shape or form by timing."""

    def __init__(self, params_list, w_list, pos_list):
        n = len(params_list)
        if not (n == len(w_list) == len(pos_list)) or n == 0:
            raise ValueError("params, states and positions must be non-empty lists of one length")
        self.params = list(params_list)
        self.w = [np.ascontiguousarray(w, dtype=np.float64) for w in w_list]
        self.pos = [np.ascontiguousarray(p, dtype=np.float64) for p in pos_list]
        for p, w, x in zip(self.params, self.w, self.pos):
            if w.shape != (p.nvar,) + p.shape or x.shape != (p.ndim,) + p.shape:
                raise ValueError("state/positions shape does not match its parameter block")
        vp = ctypes.c_void_p
        dp = ctypes.POINTER(ctypes.c_double)
        pa = (vp * n)(*[ctypes.cast(ctypes.byref(p), vp) for p in self.params])
        wa = (dp * n)(*[_dp(w) for w in self.w])
        xa = (dp * n)(*[_dp(x) for x in self.pos])
        h = vp()
        _check(lib().smaug_batch_create(n, pa, wa, xa, ctypes.byref(h)))
        self.h = h
        self.n = n

    def step(self, nsteps=1):
        _check(lib().smaug_batch_step(self.h, int(nsteps)))
        return self

    def step_async(self, nsteps=1):
        _check(lib().smaug_batch_step_async(self.h, int(nsteps)))
        return self

    def sync(self):
        _check(lib().smaug_batch_sync(self.h))

    def set_stream(self, stream_handle):
        _check(lib().smaug_batch_set_stream(self.h, ctypes.c_void_p(stream_handle or None)))

    def state(self, run):
        p = self.params[run]
        w = np.zeros((p.nvar,) + p.shape)
        _check(lib().smaug_batch_get_state(self.h, int(run), _dp(w)))
        return w

    def time(self, run):
        it = ctypes.c_int64(0)
        t = ctypes.c_double(0)
        dt = ctypes.c_double(0)
        _check(lib().smaug_batch_get_time(self.h, int(run), ctypes.byref(it), ctypes.byref(t),
                                          ctypes.byref(dt)))
        return int(it.value), float(t.value), float(dt.value)

    def launch_shape(self):
        g = ctypes.c_int32(0)
        cand = (ctypes.c_int32 * 4)()
        ms = (ctypes.c_float * 4)()
        _check(lib().smaug_batch_launch_shape(self.h, ctypes.byref(g), cand, ms))
        return {"grid": int(g.value), "candidates": list(cand), "ms": [float(v) for v in ms]}

    def tile_shape(self):
        """The tile shape the autotuner chose ((0, 0) before the first steps)
        and the step time of every (tile shape, grid) candidate."""
        tx, ty = ctypes.c_int32(0), ctypes.c_int32(0)
        ms = (ctypes.c_float * 8)()
        _check(lib().smaug_batch_tile_shape(self.h, ctypes.byref(tx), ctypes.byref(ty), ms))
        return {"tile": (int(tx.value), int(ty.value)),
                "ms": {"32x8": [float(v) for v in ms[:4]], "16x16": [float(v) for v in ms[4:]]}}

    def pin_tile_shape(self, tx, ty):
        """Use only the tile shape tx x ty (32x8 or 16x16); before the first step."""
        _check(lib().smaug_batch_pin_tile_shape(self.h, int(tx), int(ty)))
        return self

    def persistent(self):
        """Whether the tuner chose the persistent launch, and per tile shape
        (32x8, 16x16) its resident grid and step time."""
        on = ctypes.c_int32(0)
        grid = (ctypes.c_int32 * 2)()
        ms = (ctypes.c_float * 2)()
        _check(lib().smaug_batch_persistent(self.h, ctypes.byref(on), grid, ms))
        return {"on": bool(on.value), "grid": {"32x8": int(grid[0]), "16x16": int(grid[1])},
                "ms": {"32x8": float(ms[0]), "16x16": float(ms[1])}}

    def pin_form(self, form):
        """Restrict the tuner: "persistent" (one launch for several steps),
        "per-stage" (one launch per stage) or None (both); before the first
        step."""
        code = {None: -1, "per-stage": 0, "persistent": 1}[form]
        _check(lib().smaug_batch_pin_form(self.h, code))
        return self

    def close(self):
        if getattr(self, "h", None):
            lib().smaug_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def euler_step_noalloc(params, w_in_ptr, w_out_ptr, delx1d, dt, stream=None):
    """One Euler step on caller-owned device buffers (integer device
    pointers), allocating nothing; delx1d = widths along dim 0 then dim 1
    (host); returns this step's dt."""
    delx1d = np.ascontiguousarray(delx1d, dtype=np.float64)
    d = ctypes.c_double(dt)
    _check(lib().smaug_euler_step_noalloc(ctypes.byref(params), ctypes.c_void_p(w_in_ptr),
                                          ctypes.c_void_p(w_out_ptr), _dp(delx1d),
                                          ctypes.byref(d), ctypes.c_void_p(stream)))
    return d.value


def make_params(**kw):
    return _params.make_params(**kw)
