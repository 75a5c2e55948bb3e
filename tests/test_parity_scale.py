"""Parity of the CUDA engine with the CPU oracle at the benchmark sizes.

The benchmark's own workloads, run through the C ABI and compared with the
oracle on the same seeded inputs:
  - 2D Orszag-Tang 4096^2 with 1e-3 seeded rho noise, classical RK4, 2 steps
    (the headline bandwidth configuration);
  - 3D stratified atmosphere 128^3 (2 x 2 x 6 Mm, contcd4 vertically and
    periodic horizontally, gravity, Gaussian v_z driver, hyperdiffusion),
    classical RK4, 3 steps;
  - the same atmosphere at its benchmark size 256^3, one Euler step.
Tolerance: relative L2 per evolved field <= 1e-12 (FP64 on both sides,
reordered and contracted sums), and equal step time and dt to 1e-13.
Each case runs the oracle for one to two minutes on the host's cores.
"""
import numpy as np
import pytest

from smaug_b200 import ic, params as P
from tests.util import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-12


def ot(N, seed=1):
    w, pos, dx = ic.orszag_tang(N, noise=1e-3, seed=seed)
    p = P.make_params(ndim=2, n=(N + 4, N + 4, 1), dx=dx, courant=0.3, dtmax=1.0,
                      integrator=P.INT_RK4)
    return p, w, pos


def tube(N, integrator, seed=1):
    """The benchmark's 3D stratified atmosphere, N^3 interior cells."""
    w, pos, dx = ic.stratified(nz=N, nx=N, ny=N, seed=seed)
    p = P.make_params(ndim=3, n=(N + 4, N + 4, N + 4), dx=dx, courant=0.3, dtmax=1.0,
                      integrator=integrator, g=(-274.0, 0.0, 0.0),
                      boundtype=(P.BC_CONTCD4, P.BC_PERIODIC, P.BC_PERIODIC),
                      driver=P.DRIVER_GAUSS, drv_amp=200.0, drv_period=30.0,
                      drv_x0=(0.1e6, 1.0e6, 1.0e6), drv_sigma=(0.2e6, 0.2e6, 0.2e6))
    return p, w, pos


def check(engine_lib, oracle, p, w, pos, steps, nev):
    e = engine_lib.Engine(p, w, pos)
    e.step(steps)
    got = e.state()
    it, t, dt = e.time()
    e.close()
    ref = oracle.OracleRun(p, w, pos).advance(steps)
    errs = [rel_l2(got[f], ref.w[f]) for f in range(nev)]
    assert max(errs) <= TOL, errs
    assert np.array_equal(got[nev:], ref.w[nev:])
    assert it == steps
    assert abs(t - ref.t) <= 1e-13 * abs(ref.t)
    assert abs(dt - ref.dt) <= 1e-13 * abs(ref.dt)


def test_ot4096_rk4(engine_lib, oracle):
    p, w, pos = ot(4096)
    check(engine_lib, oracle, p, w, pos, 2, 6)


def test_tube128_rk4(engine_lib, oracle):
    p, w, pos = tube(128, P.INT_RK4)
    check(engine_lib, oracle, p, w, pos, 3, 8)


def test_tube256_euler(engine_lib, oracle):
    p, w, pos = tube(256, P.INT_EULER)
    check(engine_lib, oracle, p, w, pos, 1, 8)
