"""Parity of the CUDA engine (through the C ABI) with the CPU oracle on
identical seeded inputs.

Tolerance: relative L2 per evolved field <= 1e-12 after the stated number of
steps (FP64 on both sides; the engine contracts multiply-adds into FMAs, the
oracle does not, so agreement is to rounding, observed ~1e-16)."""
import numpy as np
import pytest

from smaug_b200 import params as P
from tests.util import ot_rect, params_for, rel_l2, with_background

pytestmark = pytest.mark.gpu
TOL = 1e-12


def run_both(engine_lib, oracle, w, pos, p, steps):
    e = engine_lib.Engine(p, w, pos)
    e.step(steps)
    got = e.state()
    it, t, dt = e.time()
    cm = e.cmax()
    e.close()
    ref = oracle.OracleRun(p, w, pos).advance(steps)
    return got, (it, t, dt), cm, ref


def assert_parity(got, ref, tol=TOL):
    for f in range(6):
        err = rel_l2(got[f], ref.w[f])
        assert err <= tol, "field %d: rel L2 %.3e" % (f, err)
    # backgrounds untouched
    assert np.array_equal(got[6:], ref.w[6:])


CASES = [
    # (nx, ny, steps, extra params)
    (64, 64, 10, {}),
    (48, 40, 10, {}),
    (37, 29, 6, {}),                        # partial tiles in both dims
    (5, 5, 3, {}),                          # minimum interior
    (96, 17, 4, {}),
    (40, 40, 5, {"boundtype": (P.BC_CONTCD4, P.BC_CONTCD4)}),
    (40, 40, 5, {"boundtype": (P.BC_CONT, P.BC_PERIODIC)}),
    (40, 40, 5, {"boundtype": (P.BC_SYMM, P.BC_CONTCD4)}),
    (40, 40, 5, {"boundtype": (P.BC_FIXED, P.BC_PERIODIC)}),
    (36, 40, 5, {"boundtype": (P.BC_PERIODIC, P.BC_FIXED)}),
    (40, 38, 5, {"boundtype": (P.BC_FIXED, P.BC_CONTCD4)}),
    (33, 30, 4, {"boundtype": (P.BC_FIXED, P.BC_FIXED)}),
    (38, 34, 5, {"boundtype": (P.BC_SYMM, P.BC_FIXED)}),
    (34, 38, 5, {"boundtype": (P.BC_FIXED, P.BC_CONT)}),
    (40, 40, 5, {"g": (-0.3, 0.2)}),
    (40, 40, 5, {"pad_model": P.PAD_ZERO}),
    (40, 40, 5, {"hyperdifmom": 0}),
    (40, 40, 5, {"chyp": [0.3, 0.1, 0.25, 0.2, 0.05, 0.15, 0, 0, 0, 0]}),
    (40, 40, 5, {"moddton": 0, "dt": 0.004}),
    (40, 40, 5, {"dtmax": 0.005}),           # CFL candidate rejected: dt stays
]


@pytest.mark.parametrize("integ", [P.INT_EULER, P.INT_RK4])
@pytest.mark.parametrize("nx,ny,steps,kw", CASES)
def test_parity(engine_lib, oracle, nx, ny, steps, kw, integ):
    w, pos, dx = ot_rect(nx, ny, seed=nx * 31 + ny)
    p = params_for(w, dx, integrator=integ, **kw)
    got, (it, t, dt), cm, ref = run_both(engine_lib, oracle, w, pos, p, steps)
    assert_parity(got, ref)
    assert it == steps
    assert abs(t - ref.t) <= 1e-13 * abs(ref.t)
    assert abs(dt - ref.dt) <= 1e-13 * abs(ref.dt)


@pytest.mark.parametrize("integ", [P.INT_EULER, P.INT_RK4])
def test_parity_background_fields(engine_lib, oracle, integ):
    """Nonzero energyb/rhob/b1b/b2b: split-form coupling terms
    (addenergyterms_cd2) and background pressure in every flux."""
    w, pos, dx = ot_rect(36, 28, seed=5)
    w = with_background(w)
    p = params_for(w, dx, integrator=integ, g=(0.1, -0.05),
                   boundtype=(P.BC_CONTCD4, P.BC_PERIODIC))
    got, _, _, ref = run_both(engine_lib, oracle, w, pos, p, 6)
    assert_parity(got, ref)


@pytest.mark.parametrize("integ", [P.INT_EULER, P.INT_RK4])
def test_parity_driver(engine_lib, oracle, integ):
    """Gaussian vertical-velocity driver (user source term)."""
    w, pos, dx = ot_rect(40, 32, seed=9)
    p = params_for(w, dx, integrator=integ, driver=P.DRIVER_GAUSS, drv_amp=0.05,
                   drv_period=0.3, drv_x0=(1.0, 3.0), drv_sigma=(0.5, 0.8))
    got, _, _, ref = run_both(engine_lib, oracle, w, pos, p, 6)
    assert_parity(got, ref)


def test_cmax_matches_oracle(engine_lib, oracle):
    w, pos, dx = ot_rect(50, 30, seed=2)
    p = params_for(w, dx)
    e = engine_lib.Engine(p, w, pos)
    c0 = e.cmax()
    e.step(3)
    c3 = e.cmax()
    st = e.state()
    e.close()
    ref0 = oracle.cmax(p, oracle.boundary(p, w))
    assert np.allclose(c0, ref0, rtol=1e-14, atol=0)
    assert np.allclose(c3, oracle.cmax(p, st), rtol=1e-14, atol=0)


def test_large_grid_against_oracle(engine_lib, oracle):
    """1024^2 Orszag-Tang (the benchmark's size class), 2 Euler steps."""
    w, pos, dx = ot_rect(1024, 1024, seed=3)
    p = params_for(w, dx)
    got, _, _, ref = run_both(engine_lib, oracle, w, pos, p, 2)
    assert_parity(got, ref)


def small_perturbation(w, scale=0.01):
    """Evolved fields scaled down on top of large backgrounds, so that the
    negated images of antisymmetric boundaries keep the total density and
    energy positive."""
    w = w.copy()
    ny, nx = w.shape[1:]
    w[:6] *= scale
    w[6] = 2.0
    w[7] = 1.0
    w[8] = 0.1
    w[9] = 0.05
    return w


@pytest.mark.parametrize("integ", [P.INT_EULER, P.INT_RK4])
@pytest.mark.parametrize("bt", [(P.BC_ASYMM, P.BC_PERIODIC), (P.BC_CONTCD4, P.BC_ASYMM),
                                (P.BC_ASYMM, P.BC_CONT), (P.BC_SYMM, P.BC_ASYMM)])
def test_parity_antisymmetric(engine_lib, oracle, bt, integ):
    """Antisymmetric ghosts (src/gradops.cu:1397-1465) alone and beside the
    other types, corners included."""
    w, pos, dx = ot_rect(34, 30, seed=17)
    w = small_perturbation(w)
    p = params_for(w, dx, integrator=integ, boundtype=bt)
    got, (it, t, dt), _, ref = run_both(engine_lib, oracle, w, pos, p, 5)
    assert_parity(got, ref)
    assert abs(dt - ref.dt) <= 1e-13 * abs(ref.dt)


@pytest.mark.parametrize("integ", [P.INT_EULER, P.INT_RK4])
def test_fixed_ghosts_keep_initial_values(engine_lib, integ):
    """Fixed boundaries: the two ghost layers along that dimension (corners
    included) hold the initial values after any number of steps."""
    w, pos, dx = ot_rect(30, 26, seed=8)
    p = params_for(w, dx, integrator=integ, boundtype=(P.BC_FIXED, P.BC_PERIODIC))
    e = engine_lib.Engine(p, w, pos)
    e.step(7)
    got = e.state()
    e.close()
    for f in range(6):
        for cols in (slice(0, 2), slice(-2, None)):
            assert np.array_equal(got[f][2:-2, cols], w[f][2:-2, cols])
    # corners: the periodic images of the fixed columns
    ny = w.shape[1]
    for f in range(6):
        assert np.array_equal(got[f][0:2, 0:2], w[f][ny - 4:ny - 2, 0:2])
        assert np.array_equal(got[f][ny - 2:, -2:], w[f][2:4, -2:])


FIXED_UPDATE_CASES = [
    # (boundary types, gravity, background fields, driver)
    ((P.BC_FIXED, P.BC_PERIODIC), (0.2, -0.1), False, False),
    ((P.BC_PERIODIC, P.BC_FIXED), (-0.15, 0.25), False, False),
    ((P.BC_FIXED, P.BC_CONTCD4), (0.0, 0.0), True, False),
    ((P.BC_CONTCD4, P.BC_FIXED), (0.1, 0.1), True, False),
    ((P.BC_FIXED, P.BC_PERIODIC), (0.0, 0.0), False, True),
    ((P.BC_FIXED, P.BC_FIXED), (0.2, -0.1), True, True),
    ((P.BC_SYMM, P.BC_FIXED), (0.1, -0.2), True, True),
]


@pytest.mark.parametrize("integ", [P.INT_EULER, P.INT_RK4])
@pytest.mark.parametrize("bt,g,bg,drv", FIXED_UPDATE_CASES)
def test_parity_fixed_ghost_updates(engine_lib, oracle, bt, g, bg, drv, integ):
    """2D fixed boundaries with gravity, background fields or the driver: the
    reference's gravity and energy-coupling kernels also update the two low
    ghost layers, its driver every ghost layer, and the fixed boundary keeps
    those values (src/centdiff2.cu:587-872); the engine's fixed ghost layers
    follow, ghost cells and CFL maxima included."""
    w, pos, dx = ot_rect(30, 26, seed=11)
    if bg:
        w = with_background(w)
    kw = dict(driver=P.DRIVER_GAUSS, drv_amp=0.05, drv_period=0.4, drv_x0=(0.8, 2.0),
              drv_sigma=(1.5, 2.0)) if drv else {}
    p = params_for(w, dx, integrator=integ, boundtype=bt, g=g, **kw)
    got, (it, t, dt), cm, ref = run_both(engine_lib, oracle, w, pos, p, 6)
    assert_parity(got, ref)
    assert abs(dt - ref.dt) <= 1e-13 * abs(ref.dt)
    # the fixed ghost layers did change
    w0 = oracle.boundary(p, w)
    ny, nx = w.shape[1:]
    mask = np.zeros((ny, nx), bool)
    if bt[0] == P.BC_FIXED:
        mask[:, [0, 1, nx - 2, nx - 1]] = True
    if bt[1] == P.BC_FIXED:
        mask[[0, 1, ny - 2, ny - 1], :] = True
    assert any(not np.array_equal(got[f][mask], w0[f][mask]) for f in range(6))


def test_fixed_ghost_updates_refused_by_batches(engine_lib):
    """Batches keep fixed ghost layers constant; runs whose fixed layers the
    reference would update are refused with a clear error."""
    w, pos, dx = ot_rect(20, 20, seed=2)
    p = params_for(w, dx, integrator=P.INT_RK4, boundtype=(P.BC_FIXED, P.BC_PERIODIC), g=(0.2, 0.0))
    with pytest.raises(engine_lib.SmaugError) as e:
        engine_lib.Batch([p], [w], [pos])
    assert "fixed ghost" in str(e.value)


def test_fixed_ghost_updates_need_order4(engine_lib):
    w, pos, dx = ot_rect(20, 20, seed=2)
    p = params_for(w, dx, boundtype=(P.BC_FIXED, P.BC_PERIODIC), g=(0.2, 0.0), stencil_order=6)
    with pytest.raises(engine_lib.SmaugError, match="4th-order"):
        engine_lib.Engine(p, w, pos)
