"""Differentiable time advance: the hand-written adjoint of one RK4 step
(smaug_adj_* in include/smaug_b200.h) as a torch.autograd.Function, and a
checkpointed rollout.

The step is u -> U' (2D, FP64, dt = params.dt held fixed, params.moddton = 0);
its adjoint gives the gradients with respect to the state and to the driver
parameters theta = (amplitude, period, centre along dim 1).  A rollout of N
steps keeps only every `checkpoint_every`-th state; the backward pass
recomputes one segment at a time into a device tape of the segment's stage
inputs, then runs the step adjoints from the tape (`rollout`).  The same
gradient composed from single-step Functions with torch.utils.checkpoint is
`rollout_autograd`.
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

    def reserve(self, nslots):
        _engine._check(_engine.lib().smaug_adj_tape_reserve(self.h, int(nslots)))

    def forward_tape(self, u, t, slot):
        out = torch.empty_like(u)
        st = torch.cuda.current_stream(u.device).cuda_stream
        _engine._check(_engine.lib().smaug_adj_forward_tape(self.h, self._ptr(u), self._ptr(out), float(t),
                                                            int(slot), ctypes.c_void_p(st)))
        return out

    def backward_tape(self, slot, ubar_next, t):
        ubar = torch.empty_like(ubar_next)
        thbar = torch.empty(3, dtype=torch.float64, device=ubar_next.device)
        st = torch.cuda.current_stream(ubar_next.device).cuda_stream
        _engine._check(_engine.lib().smaug_adj_backward_tape(
            self.h, int(slot), self._ptr(ubar_next.contiguous()), self._ptr(ubar), self._ptr(thbar),
            float(t), ctypes.c_void_p(st)))
        return ubar, thbar

    def backward_tape_range(self, slot_lo, nsteps, gsteps, ubar, thbar, t0, n_lo):
        """The step adjoints of slots slot_lo .. slot_lo+nsteps-1 in reverse
        order in one call (steps n_lo.. at t0 + n*dt): ubar is updated in
        place from the adjoint after the last step to the adjoint before the
        first, gsteps[k] (or nothing when None) is added before step k's
        adjoint, thbar accumulates."""
        st = torch.cuda.current_stream(ubar.device).cuda_stream
        gp = None if gsteps is None else self._ptr(gsteps)
        _engine._check(_engine.lib().smaug_adj_backward_tape_range(
            self.h, int(slot_lo), int(nsteps), gp, self._ptr(ubar), self._ptr(thbar), float(t0),
            int(n_lo), ctypes.c_void_p(st)))

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


class _Rollout(torch.autograd.Function):
    """L = sum_n loss_fn(u_n, n) over a rollout, with the hand-written step
    adjoint applied segment by segment from a tape (every > 0: checkpoints
    every `every` steps, each segment recomputed into the tape in the
    backward pass; every == 0: the forward pass records the tape of the whole
    rollout and the backward pass recomputes nothing)."""

    @staticmethod
    def forward(ctx, theta, u0, sa, nsteps, loss_fn, t0, every):
        dt = sa.dt
        sa.set_driver(*theta.detach().cpu().tolist())
        ckpt, states = [], None
        total = torch.zeros((), dtype=torch.float64, device=u0.device)
        u = u0.detach()
        with torch.no_grad():
            if every == 0:
                sa.reserve(nsteps)
                states = [u]
                for n in range(nsteps):
                    u = sa.forward_tape(u, t0 + n * dt, n)
                    states.append(u)
                    total = total + loss_fn(u, n + 1)
            else:
                for n in range(nsteps):
                    if n % every == 0:
                        ckpt.append(u)
                    u = sa.forward(u, t0 + n * dt)
                    total = total + loss_fn(u, n + 1)
        ctx.sa, ctx.nsteps, ctx.loss_fn, ctx.t0, ctx.every = sa, nsteps, loss_fn, t0, every
        ctx.ckpt, ctx.states = ckpt, states
        ctx.theta = theta.detach().cpu().tolist()
        ctx.theta_meta = (theta.dtype, theta.device)
        return total

    @staticmethod
    def _loss_grads(loss_fn, states, s):
        """d loss_fn(u_n, n) / d u_n for the states u_{s+1}.. of a segment, in
        one autograd call (each term depends on its own state only)."""
        with torch.enable_grad():
            us = [x.detach().requires_grad_(True) for x in states[1:]]
            tot = None
            for k, uk in enumerate(us):
                lk = loss_fn(uk, s + k + 1)
                tot = lk if tot is None else tot + lk
            if tot is None or not tot.requires_grad:
                return [None] * len(us)
            return list(torch.autograd.grad(tot, us, allow_unused=True))

    @staticmethod
    def backward(ctx, gL):
        sa, nsteps, every, t0 = ctx.sa, ctx.nsteps, ctx.every, ctx.t0
        dt = sa.dt
        sa.set_driver(*ctx.theta)
        ubar = None
        thbar = torch.zeros(3, dtype=torch.float64, device=gL.device)
        if every == 0:
            segments = [(0, nsteps, ctx.states, 0)]
        else:
            sa.reserve(min(every, nsteps))
            segments = [(si * every, min(nsteps, si * every + every), None, si * every)
                        for si in range(len(ctx.ckpt))]
        for s, e, states, base in reversed(segments):
            if states is None:
                # recompute the segment into the tape (slots 0 .. e-s-1)
                states = [ctx.ckpt[s // every]]
                with torch.no_grad():
                    for n in range(s, e):
                        states.append(sa.forward_tape(states[-1], t0 + n * dt, n - s))
            grads = _Rollout._loss_grads(ctx.loss_fn, states, s)
            gsteps = torch.stack([g if g is not None else torch.zeros_like(states[0]) for g in grads])
            gsteps.mul_(gL)
            if ubar is None:
                ubar = torch.zeros_like(states[0])
            # the segment's step adjoints in one call (gsteps[k] joins before step s+k)
            sa.backward_tape_range(s - base, e - s, gsteps, ubar, thbar, t0, s)
        ctx.states = None
        dtype, device = ctx.theta_meta
        # ubar and thbar already carry the factor gL (it scales every loss gradient)
        return thbar.to(device=device, dtype=dtype), ubar, None, None, None, None, None


def rollout(sa, theta, u0, nsteps, loss_fn, t0=0.0, checkpoint_every=20):
    """sum over steps n = 1..nsteps of loss_fn(u_n, n), differentiable in
    theta and u0.  With checkpoint_every = k > 0 it keeps every k-th state;
    the backward recomputes each segment once into a tape of its stage inputs
    (smaug_adj_forward_tape) and applies the step adjoints from it
    (smaug_adj_backward_tape), so no step is computed more than twice.  With
    checkpoint_every = 0 the forward pass records the tape of all nsteps steps
    (4 x nvar_evolved x cells doubles per step on the device) and the
    backward recomputes nothing.  The loss gradients of a segment are taken
    in one autograd call."""
    every = 0 if not checkpoint_every else max(1, int(checkpoint_every))
    return _Rollout.apply(theta, u0, sa, nsteps, loss_fn, t0, every)


def rollout_autograd(sa, theta, u0, nsteps, loss_fn, t0=0.0, checkpoint_every=20):
    """The same sum composed from single-step Functions (Step) under
    torch.utils.checkpoint: the states inside each segment of
    `checkpoint_every` steps are recomputed in the backward pass, and each
    step adjoint recomputes its stage inputs."""
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
