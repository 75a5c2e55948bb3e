"""Differentiable time advance: the hand-written adjoint of one RK4 step
(smaug_adj_* in include/smaug_b200.h) as a torch.autograd.Function, and a
checkpointed rollout.

The step is u -> U' (2D, FP64, dt = params.dt held fixed, params.moddton = 0);
its adjoint gives the gradients with respect to the state and to the driver
parameters theta = (amplitude, period, centre along dim 1).  A rollout of N
steps keeps only every `checkpoint_every`-th state and recomputes the states
inside a segment during the backward pass (torch.utils.checkpoint).
States are CUDA float64 tensors of the evolved fields, shape (6, n1, n0); the
background fields come from the state given at construction.
"""
import ctypes

import numpy as np
import torch
import torch.utils.checkpoint

from . import engine as _engine


class StepAdjoint:
    """Handle of the step and its adjoint for one grid and parameter block."""

    def __init__(self, params, w, pos):
        w = np.ascontiguousarray(w, dtype=np.float64)
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        if w.shape != (params.nvar,) + params.shape:
            raise ValueError("state shape %s, expected %s" % (w.shape, (params.nvar,) + params.shape))
        self.params = params
        self.dt = float(params.dt)
        h = ctypes.c_void_p()
        _engine._check(_engine.lib().smaug_adj_create(ctypes.byref(params), _engine._dp(w),
                                                      _engine._dp(pos), ctypes.byref(h)))
        self.h = h

    @staticmethod
    def _ptr(t):
        if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
            raise TypeError("expected a contiguous CUDA float64 tensor")
        return ctypes.c_void_p(t.data_ptr())

    def set_driver(self, amp, period, x0):
        _engine._check(_engine.lib().smaug_adj_set_driver(self.h, float(amp), float(period), float(x0)))

    def forward(self, u, t):
        out = torch.empty_like(u)
        st = torch.cuda.current_stream(u.device).cuda_stream
        _engine._check(_engine.lib().smaug_adj_forward(self.h, self._ptr(u), self._ptr(out), float(t),
                                                       ctypes.c_void_p(st)))
        return out

    def backward(self, u, ubar_next, t):
        ubar = torch.empty_like(u)
        thbar = torch.empty(3, dtype=torch.float64, device=u.device)
        st = torch.cuda.current_stream(u.device).cuda_stream
        _engine._check(_engine.lib().smaug_adj_backward(
            self.h, self._ptr(u), self._ptr(ubar_next.contiguous()), self._ptr(ubar), self._ptr(thbar),
            float(t), ctypes.c_void_p(st)))
        return ubar, thbar

    def close(self):
        if getattr(self, "h", None):
            _engine.lib().smaug_adj_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Step(torch.autograd.Function):
    """U' = step(u; theta) at time t, differentiable in u and theta."""

    @staticmethod
    def forward(ctx, theta, u, t, sa):
        sa.set_driver(*theta.detach().cpu().tolist())
        out = sa.forward(u.detach(), t)
        ctx.save_for_backward(theta, u)
        ctx.t = t
        ctx.sa = sa
        return out

    @staticmethod
    def backward(ctx, gout):
        theta, u = ctx.saved_tensors
        sa = ctx.sa
        sa.set_driver(*theta.detach().cpu().tolist())
        ubar, thbar = sa.backward(u.detach(), gout, ctx.t)
        return thbar.to(theta.device, theta.dtype), ubar, None, None


def rollout(sa, theta, u0, nsteps, loss_fn, t0=0.0, checkpoint_every=20):
    """sum over steps n = 1..nsteps of loss_fn(u_n, n), differentiable in
    theta and u0; the states inside each segment of `checkpoint_every` steps
    are recomputed in the backward pass."""
    dt = sa.dt

    def segment(theta_, u_, n0, n1):
        acc = torch.zeros((), dtype=torch.float64, device=u_.device)
        for n in range(n0, n1):
            u_ = Step.apply(theta_, u_, t0 + n * dt, sa)
            acc = acc + loss_fn(u_, n + 1)
        return acc, u_

    total = torch.zeros((), dtype=torch.float64, device=u0.device)
    u = u0
    for s in range(0, nsteps, checkpoint_every):
        e = min(nsteps, s + checkpoint_every)
        part, u = torch.utils.checkpoint.checkpoint(segment, theta, u, s, e, use_reentrant=False)
        total = total + part
    return total
