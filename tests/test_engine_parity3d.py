"""3D: parity of the CUDA engine (through the C ABI) with the CPU oracle on
identical seeded inputs, and against the reference's own 3D outputs.

Tolerance: relative L2 per evolved field <= 1e-12 after the stated number of
steps (FP64 on both sides; sums per cell are reordered and contracted into
FMAs, so agreement is to rounding)."""
import numpy as np
import pytest

from smaug_b200 import params as P
from tests import golden_util as G
from tests.util import params3, rel_l2, state3d

pytestmark = pytest.mark.gpu
TOL = 1e-12

C4, PER, CONT, SYM = P.BC_CONTCD4, P.BC_PERIODIC, P.BC_CONT, P.BC_SYMM
FIX, ASYM = P.BC_FIXED, P.BC_ASYMM


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
    for f in range(8):
        err = rel_l2(got[f], ref.w[f])
        assert err <= tol, "field %d: rel L2 %.3e" % (f, err)
    assert np.array_equal(got[8:], ref.w[8:])


CASES = [
    # (nx, ny, nz, steps, background, extra params)
    (12, 12, 8, 6, True, {"g": (-0.1, 0.0, 0.0)}),
    (16, 12, 9, 5, True, {"boundtype": (PER, PER, PER)}),
    (9, 7, 6, 5, True, {"boundtype": (C4, PER, CONT)}),        # partial tiles everywhere
    (4, 4, 4, 4, True, {}),                                     # minimum interior
    (20, 8, 5, 4, True, {"boundtype": (SYM, C4, PER), "g": (0.0, 0.05, -0.02)}),
    (10, 10, 10, 5, False, {"boundtype": (PER, PER, PER)}),    # no background fields
    (11, 9, 13, 4, True, {"pad_model": P.PAD_ZERO}),
    (11, 9, 13, 4, True, {"hyperdifmom": 0}),
    (10, 12, 7, 4, True, {"chyp": [0.3, 0.1, 0.25, 0.2, 0.15, 0.05, 0.12, 0.18, 0, 0, 0, 0, 0]}),
    (10, 10, 8, 4, True, {"moddton": 0, "dt": 1e-3}),
    (10, 10, 8, 4, True, {"dtmax": 5e-4}),                     # CFL candidate rejected
    (12, 10, 8, 4, True, {"boundtype": (FIX, PER, C4)}),
    (9, 10, 7, 4, True, {"boundtype": (ASYM, FIX, PER)}),
    (10, 8, 9, 4, True, {"boundtype": (C4, ASYM, SYM)}),
]


@pytest.mark.parametrize("integ", [P.INT_EULER, P.INT_RK4])
@pytest.mark.parametrize("nx,ny,nz,steps,bg,kw", CASES)
def test_parity3d(engine_lib, oracle, nx, ny, nz, steps, bg, kw, integ):
    w, pos, dx = state3d(nx, ny, nz, seed=nx * 97 + ny * 13 + nz, background=bg)
    p = params3(w, dx, integrator=integ, **kw)
    got, (it, t, dt), cm, ref = run_both(engine_lib, oracle, w, pos, p, steps)
    assert_parity(got, ref)
    assert it == steps
    assert abs(t - ref.t) <= 1e-13 * abs(ref.t)
    assert abs(dt - ref.dt) <= 1e-13 * abs(ref.dt)


@pytest.mark.parametrize("integ", [P.INT_EULER, P.INT_RK4])
def test_parity3d_driver(engine_lib, oracle, integ):
    """Gaussian driver on m along dim 0 (the vertical axis)."""
    w, pos, dx = state3d(14, 10, 8, seed=6)
    p = params3(w, dx, integrator=integ, boundtype=(C4, PER, PER), g=(-0.1, 0, 0),
                driver=P.DRIVER_GAUSS, drv_amp=0.02, drv_period=0.01,
                drv_x0=(0.02, 0.05, 0.05), drv_sigma=(0.02, 0.03, 0.03))
    got, _, _, ref = run_both(engine_lib, oracle, w, pos, p, 5)
    assert_parity(got, ref)


def test_cmax3d_matches_oracle(engine_lib, oracle):
    w, pos, dx = state3d(13, 9, 7, seed=2)
    p = params3(w, dx)
    e = engine_lib.Engine(p, w, pos)
    c0 = e.cmax()
    e.step(2)
    c2 = e.cmax()
    st = e.state()
    e.close()
    assert np.allclose(c0, oracle.cmax(p, oracle.boundary(p, w)), rtol=1e-14, atol=0)
    assert np.allclose(c2, oracle.cmax(p, st), rtol=1e-14, atol=0)


def test_larger_grid3d_against_oracle(engine_lib, oracle):
    """64 x 48 x 40 interior (many blocks in every direction), 2 RK4 steps."""
    w, pos, dx = state3d(64, 48, 40, seed=3)
    p = params3(w, dx, integrator=P.INT_RK4, boundtype=(C4, PER, PER), g=(-0.1, 0, 0))
    got, _, _, ref = run_both(engine_lib, oracle, w, pos, p, 2)
    assert_parity(got, ref)


@pytest.mark.parametrize("name", G.STRICT3 + G.ORDER6_3D)
def test_engine_matches_reference_run_3d(engine_lib, name):
    """Every field at every saved step of the reference's 3D build."""
    d = G.load(name)
    p = G.params(d)
    e = engine_lib.Engine(p, d["w0full"], d["pos"])
    done = 0
    for k, ref in zip(d["steps"], d["states"]):
        e.step(int(k) - done)
        done = int(k)
        got = e.state()
        for f in range(13):
            assert rel_l2(got[f], ref[f]) <= 1e-13, (name, k, f, rel_l2(got[f], ref[f]))
    e.close()
