"""Hand-written adjoint of the 2D RK4 step (smaug_adj_*) and the checkpointed
differentiable rollout (smaug_b200/adjoint.py), against central finite
differences of the forward step on a small stratified driven slab (gravity,
background fields, contcd4/periodic ghosts, hyperdiffusion, Gaussian driver).

Tolerances (relative): 2e-7 for the step's state adjoint without
hyperdiffusion (a smooth operator; central FD with steps of 1e-7 relative
is good to ~1e-8 per term); 1e-6 with hyperdiffusion (the
max-limiters are piecewise smooth: with smooth perturbations of a state
without symmetries, FD steps of 1e-7 relative rarely cross a kink); 1e-5 for the driver-parameter gradient
of a 12-step rollout against central FD with h = 1e-4 relative."""
import numpy as np
import pytest

from smaug_b200 import ic, params as P

pytestmark = pytest.mark.gpu


def slab(nz=32, nx=24, hyper=1, seed=4):
    w, pos, dx = ic.stratified(nz=nz, nx=nx, seed=seed, vz_sigma=10.0)
    p = P.make_params(ndim=2, n=(nz + 4, nx + 4, 1), dx=dx, courant=0.3, dtmax=1.0,
                      integrator=P.INT_RK4, g=(-274.0, 0.0),
                      boundtype=(P.BC_CONTCD4, P.BC_PERIODIC), driver=P.DRIVER_GAUSS,
                      drv_amp=200.0, drv_period=30.0, drv_x0=(0.1e6, 1.0e6),
                      drv_sigma=(0.2e6, 0.2e6), hyperdifmom=hyper)
    return p, w, pos


def fixed_dt(engine_lib, p, w, pos):
    e = engine_lib.Engine(p, w, pos)
    e.step(1)
    dt = e.time()[2]
    e.close()
    q = P.SmaugParams.from_buffer_copy(p)
    q.moddton = 0
    q.dt = 0.5 * dt
    return q


def generic(hyper=1, seed=5):
    """Smooth 2D state without symmetries (a max with exact ties is not
    differentiable, and white noise puts near-ties within any FD step):
    Orszag-Tang with background fields and a smooth oblique modulation of every
    field, gravity, an off-centre driver, contcd4 / periodic ghosts."""
    from tests.util import ot_rect, with_background
    w, pos, dx = ot_rect(40, 32, seed=seed, noise=0.0)
    w = with_background(w)
    X, Y = pos
    for f in range(6):  # smooth, without the Orszag-Tang symmetries
        w[f] *= 1.0 + 2e-2 * np.sin((0.9 + 0.13 * f) * X + (0.6 + 0.07 * f) * Y + 0.3 * f + 0.4)
    p = P.make_params(ndim=2, n=(44, 36, 1), dx=dx, courant=0.3, dtmax=1.0, integrator=P.INT_RK4,
                      g=(0.1, -0.05), boundtype=(P.BC_CONTCD4, P.BC_PERIODIC),
                      driver=P.DRIVER_GAUSS, drv_amp=0.05, drv_period=0.3, drv_x0=(1.3, 2.7),
                      drv_sigma=(0.5, 0.8), hyperdifmom=hyper)
    return p, w, pos


def setup(engine_lib, make, hyper=1):
    import torch
    from smaug_b200.adjoint import StepAdjoint
    p, w, pos = make(hyper=hyper)
    q = fixed_dt(engine_lib, p, w, pos)
    sa = StepAdjoint(q, w, pos)
    u = torch.tensor(w[:6], dtype=torch.float64, device="cuda").contiguous()
    return sa, q, w, pos, u


@pytest.mark.parametrize("hyper,tol", [(0, 2e-7), (1, 1e-6)])
def test_step_adjoint_matches_directional_fd(engine_lib, hyper, tol):
    """<lam, (step(u + eps v) - step(u - eps v)) / 2 eps> against <ubar, v>
    for a smooth perturbation v of each field."""
    import torch
    sa, q, w, pos, u = setup(engine_lib, generic, hyper)
    t = 0.1
    gen = torch.Generator(device="cuda").manual_seed(7)
    scale = u.abs().amax(dim=(1, 2), keepdim=True).clamp_min(1e-30)
    eps = 1e-7
    X = torch.tensor(pos[0], device="cuda", dtype=torch.float64)
    Y = torch.tensor(pos[1], device="cuda", dtype=torch.float64)
    for f in range(6):
        # a smooth direction: random-noise directions move the third
        # differences that nu is built on across their maxima' kinks
        v = torch.zeros_like(u)
        v[f] = u[f] * torch.sin((1.1 + 0.2 * f) * X - (0.8 + 0.1 * f) * Y + 0.5 + f)
        lam = torch.randn(u.shape, generator=gen, device="cuda", dtype=torch.float64) / scale
        lam[:, :2, :] = 0
        lam[:, -2:, :] = 0
        lam[:, :, :2] = 0
        lam[:, :, -2:] = 0
        fd = float(((sa.forward(u + eps * v, t) - sa.forward(u - eps * v, t)) / (2 * eps) * lam).sum())
        ubar, _ = sa.backward(u, lam, t)
        ad = float((ubar * v).sum())
        assert abs(ad - fd) <= tol * abs(fd), (f, ad, fd)
    sa.close()


def test_rollout_parameter_gradient_matches_fd(engine_lib):
    import torch
    from smaug_b200.adjoint import rollout
    sa, q, w, pos, u0 = setup(engine_lib, slab, 1)
    kz = int(np.argmin(np.abs(pos[0][0] - 0.4e6)))  # the row z = 0.4 Mm (dim 0 is vertical)
    rhob = torch.tensor(w[7], device="cuda", dtype=torch.float64)
    theta0 = torch.tensor([200.0, 30.0, 1.0e6], dtype=torch.float64)
    nsteps = 12

    def vz_row(u):
        return u[1, :, kz] / (u[0, :, kz] + rhob[:, kz])

    # target trace from a run with shifted parameters
    with torch.no_grad():
        target = []
        sa.set_driver(*(theta0 * torch.tensor([1.05, 0.9, 1.02], dtype=torch.float64)).tolist())
        u = u0
        for n in range(nsteps):
            u = sa.forward(u, n * q.dt)
            target.append(vz_row(u).clone())

    def loss_fn(u, n):
        return ((vz_row(u) - target[n - 1]) ** 2).sum()

    theta = theta0.clone().requires_grad_(True)
    L = rollout(sa, theta, u0, nsteps, loss_fn, checkpoint_every=5)
    assert float(L.detach()) > 0
    L.backward()
    g = theta.grad.clone()
    for k in range(3):
        h = 1e-4 * float(theta0[k])
        vals = []
        for s in (1, -1):
            th = theta0.clone()
            th[k] += s * h
            with torch.no_grad():
                vals.append(float(rollout(sa, th, u0, nsteps, loss_fn, checkpoint_every=5)))
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(float(g[k]) - fd) <= 1e-5 * abs(fd) + 1e-30, (k, float(g[k]), fd)
    sa.close()


def test_adjoint_rejects(engine_lib):
    from smaug_b200.adjoint import StepAdjoint
    p, w, pos = slab()
    with pytest.raises(engine_lib.SmaugError) as e:
        StepAdjoint(p, w, pos)          # moddton = 1: dt would depend on the state
    assert e.value.code == 6


def test_taped_rollout_equals_checkpointed_composition(engine_lib):
    """rollout (segment recompute into a tape, step adjoints from the tape)
    and rollout_autograd (single-step Functions under torch.utils.checkpoint,
    each adjoint recomputing its stages) give the same loss and gradients
    with respect to the parameters and the initial state."""
    import torch
    from smaug_b200.adjoint import rollout, rollout_autograd
    sa, q, w, pos, u0 = setup(engine_lib, slab, 1)
    kz = int(np.argmin(np.abs(pos[0][0] - 0.4e6)))
    rhob = torch.tensor(w[7], device="cuda", dtype=torch.float64)
    theta0 = torch.tensor([200.0, 30.0, 1.0e6], dtype=torch.float64)

    def loss_fn(u, n):
        v = u[1, :, kz] / (u[0, :, kz] + rhob[:, kz])
        return (v ** 2).sum() * (1.0 + 0.1 * n)

    out = []
    for fn in (rollout, rollout_autograd):
        th = theta0.clone().requires_grad_(True)
        u = u0.clone().requires_grad_(True)
        L = fn(sa, th, u, 9, loss_fn, checkpoint_every=4)
        L.backward()
        out.append((float(L), th.grad.clone(), u.grad.clone()))
    (L1, g1, u1), (L2, g2, u2) = out
    assert abs(L1 - L2) <= 1e-13 * abs(L2)
    assert float((g1 - g2).abs().max()) <= 1e-10 * float(g2.abs().max())
    assert float((u1 - u2).norm()) <= 1e-10 * float(u2.norm())
    assert float(u2.norm()) > 0
    sa.close()


def test_full_tape_rollout_equals_checkpointed(engine_lib):
    """checkpoint_every = 0 (the forward pass records the tape of every step,
    the backward recomputes nothing) gives the loss of the checkpointed
    rollout exactly and its gradients to rounding (the same stage inputs and
    step adjoints; the adjoint's reductions add in hardware order)."""
    import torch
    from smaug_b200.adjoint import rollout
    sa, q, w, pos, u0 = setup(engine_lib, slab, 1)
    kz = int(np.argmin(np.abs(pos[0][0] - 0.4e6)))
    rhob = torch.tensor(w[7], device="cuda", dtype=torch.float64)
    theta0 = torch.tensor([200.0, 30.0, 1.0e6], dtype=torch.float64)

    def loss_fn(u, n):
        v = u[1, :, kz] / (u[0, :, kz] + rhob[:, kz])
        return (v ** 2).sum() * (1.0 + 0.1 * n)

    out = []
    for every in (4, 0):
        th = theta0.clone().requires_grad_(True)
        u = u0.clone().requires_grad_(True)
        L = rollout(sa, th, u, 9, loss_fn, checkpoint_every=every)
        L.backward()
        out.append((float(L), th.grad.clone(), u.grad.clone()))
    (L1, g1, u1), (L2, g2, u2) = out
    assert L1 == L2
    assert float((g1 - g2).abs().max()) <= 1e-12 * float(g2.abs().max())
    assert float((u1 - u2).norm()) <= 1e-12 * float(u2.norm())
    assert float(u2.norm()) > 0
    sa.close()


def test_parameter_gradient_matches_oracle_fd(engine_lib, oracle):
    """The adjoint's driver-parameter gradient against central differences of
    the same loss computed by the CPU oracle (pinned to the reference's own
    outputs), so that the check does not rest on the CUDA forward: a 32 x 24
    stratified driven slab, 20 RK4 steps at fixed dt, loss = sum over steps of
    sum_x (v_z - target)^2 on the row z = 0.4 Mm, target from an oracle run
    with shifted parameters.  Tolerances: the two losses agree to 1e-10
    (FP64 forwards of the same operator); the gradient agrees with central FD
    at h = 1e-6 relative to 1e-7 relative.  (The FD of the driver centre
    converges as -5.90591e-4, -5.898722e-4, -5.8986471e-4, -5.89864712e-4 for
    h = 1e-3 .. 1e-6 relative: at h = 1e-4 its truncation error is still
    1.3e-5, the Gaussian's width being 0.2 Mm.)"""
    import torch
    from smaug_b200.adjoint import rollout
    sa, q, w, pos, u0 = setup(engine_lib, slab, 1)
    kz = int(np.argmin(np.abs(pos[0][0] - 0.4e6)))
    nsteps = 20
    theta0 = np.array([200.0, 30.0, 1.0e6])

    def oracle_states(theta):
        pp = P.SmaugParams.from_buffer_copy(q)
        pp.drv_amp, pp.drv_period, pp.drv_x0[1] = theta
        run = oracle.OracleRun(pp, w, pos)
        out = []
        for _ in range(nsteps):
            run.advance(1)
            out.append(run.w[1, :, kz] / (run.w[0, :, kz] + run.w[7, :, kz]))
        return out

    target = oracle_states(theta0 * np.array([1.05, 0.9, 1.02]))

    def oracle_loss(theta):
        return sum(float(np.sum((v - t) ** 2)) for v, t in zip(oracle_states(theta), target))

    rhob = torch.tensor(w[7], device="cuda", dtype=torch.float64)
    tgt = [torch.tensor(t, device="cuda", dtype=torch.float64) for t in target]

    def loss_fn(u, n):
        return ((u[1, :, kz] / (u[0, :, kz] + rhob[:, kz]) - tgt[n - 1]) ** 2).sum()

    theta = torch.tensor(theta0, dtype=torch.float64).requires_grad_(True)
    L = rollout(sa, theta, u0, nsteps, loss_fn, checkpoint_every=5)
    L.backward()
    g = theta.grad.detach().numpy()
    L0 = oracle_loss(theta0)
    assert L0 > 0
    assert abs(float(L.detach()) - L0) <= 1e-10 * L0, (float(L.detach()), L0)
    for k in range(3):
        h = 1e-6 * theta0[k]
        tp, tm = theta0.copy(), theta0.copy()
        tp[k] += h
        tm[k] -= h
        fd = (oracle_loss(tp) - oracle_loss(tm)) / (2 * h)
        assert abs(g[k] - fd) <= 1e-7 * abs(fd), (k, g[k], fd)
    sa.close()
