"""The 6th-order flux derivative (stencil_order = 6): the reference's
-DUSE_DORDER3 build of grad3dn (src/gradops.cu:450-453), defined on the
index range (2, n-3) of each direction and 0 elsewhere.

Parity of the CUDA engine (through the C ABI) with the CPU oracle on
identical seeded inputs, 2D and 3D, Euler and RK4.  Tolerance: relative L2
per evolved field <= 1e-12 after the stated number of steps (FP64; the
engine multiplies by reciprocals and contracts FMAs, the oracle divides)."""
import numpy as np
import pytest

from smaug_b200 import params as P
from tests.util import ot_rect, params3, params_for, rel_l2, state3d, with_background

pytestmark = pytest.mark.gpu
TOL = 1e-12
C4, PER, CONT, SYM, FIX = P.BC_CONTCD4, P.BC_PERIODIC, P.BC_CONT, P.BC_SYMM, P.BC_FIXED


def run_both(engine_lib, oracle, w, pos, p, steps):
    e = engine_lib.Engine(p, w, pos)
    e.step(steps)
    got = e.state()
    it, t, dt = e.time()
    e.close()
    ref = oracle.OracleRun(p, w, pos).advance(steps)
    return got, (it, t, dt), ref


def assert_parity(got, ref, nevo, tol=TOL):
    for f in range(nevo):
        err = rel_l2(got[f], ref.w[f])
        assert err <= tol, "field %d: rel L2 %.3e" % (f, err)
    assert np.array_equal(got[nevo:], ref.w[nevo:])


CASES2 = [
    # (nx, ny, steps, background, extra params)
    (64, 64, 8, False, {}),
    (37, 29, 6, False, {}),                                   # partial tiles in both dims
    (5, 5, 3, False, {}),                                     # minimum interior
    (96, 17, 4, False, {}),
    (40, 40, 5, False, {"boundtype": (C4, C4)}),
    (40, 36, 5, False, {"boundtype": (SYM, PER)}),
    (36, 40, 5, False, {"boundtype": (FIX, CONT)}),
    (36, 28, 6, True, {"g": (0.1, -0.05), "boundtype": (C4, PER)}),  # energy coupling terms
    (40, 32, 6, False, {"driver": P.DRIVER_GAUSS, "drv_amp": 0.05, "drv_period": 0.3,
                        "drv_x0": (1.0, 3.0), "drv_sigma": (0.5, 0.8)}),
]


@pytest.mark.parametrize("integ", [P.INT_EULER, P.INT_RK4])
@pytest.mark.parametrize("nx,ny,steps,bg,kw", CASES2)
def test_parity_order6_2d(engine_lib, oracle, nx, ny, steps, bg, kw, integ):
    w, pos, dx = ot_rect(nx, ny, seed=nx * 17 + ny)
    if bg:
        w = with_background(w)
    p = params_for(w, dx, integrator=integ, stencil_order=6, **kw)
    got, (it, t, dt), ref = run_both(engine_lib, oracle, w, pos, p, steps)
    assert_parity(got, ref, 6)
    assert it == steps
    assert abs(t - ref.t) <= 1e-13 * abs(ref.t)


CASES3 = [
    # (nx, ny, nz, steps, background, extra params)
    (12, 12, 8, 5, True, {"g": (-0.1, 0.0, 0.0)}),
    (16, 12, 9, 4, True, {"boundtype": (PER, PER, PER)}),
    (9, 7, 6, 4, True, {"boundtype": (C4, PER, CONT)}),       # partial tiles everywhere
    (10, 10, 10, 4, False, {"boundtype": (PER, PER, PER)}),
    (12, 10, 8, 4, True, {"boundtype": (FIX, PER, C4)}),
]


@pytest.mark.parametrize("integ", [P.INT_EULER, P.INT_RK4])
@pytest.mark.parametrize("nx,ny,nz,steps,bg,kw", CASES3)
def test_parity_order6_3d(engine_lib, oracle, nx, ny, nz, steps, bg, kw, integ):
    w, pos, dx = state3d(nx, ny, nz, seed=nx * 7 + ny * 5 + nz, background=bg)
    p = params3(w, dx, integrator=integ, stencil_order=6, **kw)
    got, (it, t, dt), ref = run_both(engine_lib, oracle, w, pos, p, steps)
    assert_parity(got, ref, 8)
    assert it == steps


def test_order6_mixed_form_tracks_fp64(engine_lib):
    """The mixed precision form with the 6th-order derivative against the
    FP64 engine: 1e-5 per field after 10 RK4 steps."""
    w, pos, dx = ot_rect(96, 80, seed=4)
    out = []
    for prec in (P.PREC_FP64, P.PREC_MIXED):
        p = params_for(w, dx, integrator=P.INT_RK4, stencil_order=6, precision=prec)
        e = engine_lib.Engine(p, w, pos)
        e.step(10)
        out.append(e.state())
        e.close()
    for f in range(6):
        assert rel_l2(out[1][f], out[0][f]) <= 1e-5, f


def test_order6_changes_the_result(engine_lib):
    """The switch reaches the kernels: 4th and 6th order differ after a few
    steps (by the truncation error, far above rounding)."""
    w, pos, dx = ot_rect(48, 48, seed=2)
    out = []
    for order in (4, 6):
        e = engine_lib.Engine(params_for(w, dx, integrator=P.INT_RK4, stencil_order=order), w, pos)
        e.step(3)
        out.append(e.state())
        e.close()
    assert max(rel_l2(out[1][f], out[0][f]) for f in range(6)) > 1e-8


def test_order6_rejections(engine_lib):
    """Orders other than 4 and 6 are invalid; batches and the adjoint are of
    the 4th-order stencil only."""
    import torch
    from smaug_b200.adjoint import StepAdjoint
    w, pos, dx = ot_rect(40, 40, seed=1)
    with pytest.raises(engine_lib.SmaugError) as e:
        engine_lib.Engine(params_for(w, dx, stencil_order=5), w, pos)
    assert e.value.code == 1
    p6 = params_for(w, dx, integrator=P.INT_RK4, stencil_order=6)
    with pytest.raises(engine_lib.SmaugError) as e:
        engine_lib.Batch([p6], [w], [pos])
    assert e.value.code == 6
    q = params_for(w, dx, integrator=P.INT_RK4, stencil_order=6, moddton=0, dt=1e-3)
    with pytest.raises(engine_lib.SmaugError) as e:
        StepAdjoint(q, w, pos)
    assert e.value.code == 6
    assert torch.cuda.is_available()
