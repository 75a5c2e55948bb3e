"""Mixed precision form (perturbations stored and hyperdiffusion computed in
float; backgrounds, fluxes, pressure recovery, CFL and the compensated RK4
accumulation in double) against the FP64 oracle on identical inputs.

Tolerance: relative L2 per evolved field <= 1e-5 after the stated number of
steps (the accuracy bar of the mixed form); the errors are also required to
be well above FP64 rounding, i.e. the float path really runs."""
import numpy as np
import pytest

from smaug_b200 import params as P
from tests.util import ot_rect, params3, params_for, rel_l2, state3d, with_background

pytestmark = pytest.mark.gpu
TOL = 1e-5


def errors(engine_lib, oracle, w, pos, p, steps, nevo):
    e = engine_lib.Engine(p, w, pos)
    e.step(steps)
    got = e.state()
    it, t, dt = e.time()
    e.close()
    pf = P.SmaugParams.from_buffer_copy(p)
    pf.precision = P.PREC_FP64
    ref = oracle.OracleRun(pf, w, pos).advance(steps)
    errs = [rel_l2(got[f], ref.w[f]) for f in range(nevo)]
    assert np.array_equal(got[nevo:], ref.w[nevo:])
    return errs, (t, dt), ref


@pytest.mark.parametrize("integ", [P.INT_RK4, P.INT_EULER])
def test_mixed_ot128_short(engine_lib, oracle, integ):
    """Orszag-Tang 128^2, 25 steps: within the 1e-5 bar."""
    w, pos, dx = ot_rect(128, 128, seed=1)
    p = params_for(w, dx, integrator=integ, precision=P.PREC_MIXED)
    errs, (t, dt), ref = errors(engine_lib, oracle, w, pos, p, 25, 6)
    assert max(errs) <= TOL, errs
    assert max(errs) > 1e-12, errs
    assert abs(t - ref.t) <= 1e-6 * ref.t


def test_mixed_ot128_200_steps_within_fp64_sensitivity(engine_lib, oracle):
    """Orszag-Tang 128^2, 200 RK4 steps (the small benchmark configuration).
    The FP64 solution itself is chaotic at this horizon: rounding only the
    initial state to float moves the FP64 result by ~3e-3 after 200 steps
    (and a 1e-12 relative perturbation by ~4e-6), so no float-storage form
    can meet 1e-5 there.  The mixed form must stay within 3x of that
    FP64 sensitivity."""
    w, pos, dx = ot_rect(128, 128, seed=1)
    p = params_for(w, dx, integrator=P.INT_RK4, precision=P.PREC_MIXED)
    errs, _, ref = errors(engine_lib, oracle, w, pos, p, 200, 6)
    pf = params_for(w, dx, integrator=P.INT_RK4)
    wf = w.copy()
    wf[:6] = w[:6].astype(np.float32).astype(np.float64)
    rounded = oracle.OracleRun(pf, wf, pos).advance(200)
    sens = max(rel_l2(rounded.w[f], ref.w[f]) for f in range(6))
    assert max(errs) <= 3 * sens, (errs, sens)


@pytest.mark.parametrize("integ", [P.INT_RK4, P.INT_EULER])
def test_mixed_background_2d(engine_lib, oracle, integ):
    w, pos, dx = ot_rect(48, 40, seed=5)
    w = with_background(w)
    p = params_for(w, dx, integrator=integ, g=(0.1, -0.05), precision=P.PREC_MIXED,
                   boundtype=(P.BC_CONTCD4, P.BC_PERIODIC))
    errs, _, _ = errors(engine_lib, oracle, w, pos, p, 40, 6)
    assert max(errs) <= TOL, errs


@pytest.mark.parametrize("integ", [P.INT_RK4, P.INT_EULER])
def test_mixed_fixed_and_antisymmetric(engine_lib, oracle, integ):
    """Fixed ghosts live in every float buffer; antisymmetric images."""
    w, pos, dx = ot_rect(40, 36, seed=6)
    p = params_for(w, dx, integrator=integ, precision=P.PREC_MIXED,
                   boundtype=(P.BC_FIXED, P.BC_PERIODIC))
    errs, _, _ = errors(engine_lib, oracle, w, pos, p, 20, 6)
    assert max(errs) <= TOL, errs
    w3, pos3, dx3 = state3d(10, 9, 8, seed=9)
    p3 = params3(w3, dx3, integrator=integ, precision=P.PREC_MIXED,
                 boundtype=(P.BC_ASYMM, P.BC_FIXED, P.BC_PERIODIC))
    errs, _, _ = errors(engine_lib, oracle, w3, pos3, p3, 10, 8)
    assert max(errs) <= TOL, errs


@pytest.mark.parametrize("integ", [P.INT_RK4, P.INT_EULER])
def test_mixed_3d(engine_lib, oracle, integ):
    w, pos, dx = state3d(16, 12, 10, seed=7)
    p = params3(w, dx, integrator=integ, g=(-0.1, 0, 0), precision=P.PREC_MIXED,
                boundtype=(P.BC_CONTCD4, P.BC_PERIODIC, P.BC_PERIODIC),
                driver=P.DRIVER_GAUSS, drv_amp=0.02, drv_period=0.01,
                drv_x0=(0.02, 0.05, 0.05), drv_sigma=(0.02, 0.03, 0.03))
    errs, _, _ = errors(engine_lib, oracle, w, pos, p, 30, 8)
    assert max(errs) <= TOL, errs


def test_mixed_matches_fp64_engine_1024(engine_lib):
    """1024^2 Orszag-Tang, 20 RK4 steps: mixed against the FP64 engine."""
    w, pos, dx = ot_rect(1024, 1024, seed=3)
    out = {}
    for prec in (P.PREC_FP64, P.PREC_MIXED):
        p = params_for(w, dx, integrator=P.INT_RK4, precision=prec)
        e = engine_lib.Engine(p, w, pos)
        e.step(20)
        out[prec] = e.state()
        e.close()
    errs = [rel_l2(out[P.PREC_MIXED][f], out[P.PREC_FP64][f]) for f in range(6)]
    assert max(errs) <= TOL, errs


def test_mixed_roundtrip_and_determinism(engine_lib):
    w, pos, dx = ot_rect(40, 33, seed=4)
    p = params_for(w, dx, integrator=P.INT_RK4, precision=P.PREC_MIXED)
    a = engine_lib.Engine(p, w, pos)
    a.step(5)
    s5 = a.state()
    a.step(5)
    s10 = a.state()
    b = engine_lib.Engine(p, w, pos)
    b.step(5)
    b.set_state(s5)       # FP64 in, split into the float pair: exact round trip
    assert np.array_equal(b.state(), s5)
    b.step(5)
    # the restart recomputes the CFL maxima from hi+lo rather than from the
    # stage sum, so dt may differ in the last bits
    s10b = b.state()
    for f in range(6):
        assert rel_l2(s10b[f], s10[f]) <= 1e-12
    a.close()
    b.close()


@pytest.mark.parametrize("integ", [P.INT_RK4, P.INT_EULER])
def test_mixed_fixed_ghost_updates(engine_lib, oracle, integ):
    """2D fixed boundaries with gravity, background fields and the driver:
    the mixed form's fixed ghost layers (fixed_ghost2d_kernel with float
    storage) follow the FP64 oracle within the 1e-5 bar, ghost cells
    included."""
    w, pos, dx = ot_rect(30, 26, seed=11)
    w = with_background(w)
    p = params_for(w, dx, integrator=integ, precision=P.PREC_MIXED,
                   boundtype=(P.BC_FIXED, P.BC_FIXED), g=(0.2, -0.1), driver=P.DRIVER_GAUSS,
                   drv_amp=0.05, drv_period=0.4, drv_x0=(0.8, 2.0), drv_sigma=(1.5, 2.0))
    errs, _, ref = errors(engine_lib, oracle, w, pos, p, 10, 6)
    assert max(errs) <= TOL, errs
    assert max(errs) > 1e-12, errs
