"""The 2D stage kernel with bulk-tensor (TMA) staging against the same kernel
with per-thread staging.

Both evaluate the same arithmetic cell by cell, so the states after the same
steps are bitwise identical, as are the step time, dt and the CFL maxima.
The grids are large enough (over 600 tiles) that every block of the
persistent form stages several tiles, so the copy of a block's next tile,
issued during the current tile's stores, is exercised; the small grids
cover the edge tiles.  The engine-oracle parity of the staged kernel is the
bitwise equality with the per-thread staging, which the parity suite pins."""
import numpy as np
import pytest

from smaug_b200 import params as P
from tests.util import ot_rect, params_for, with_background

pytestmark = pytest.mark.gpu


def run(engine_lib, w, pos, p, steps, staging):
    e = engine_lib.Engine(p, w, pos)
    _, avail = e.staging()
    assert avail
    e.set_staging(staging)
    assert e.staging() == (staging, True)
    e.step(steps)
    out = (e.state(), e.time(), e.cmax())
    e.close()
    return out


def assert_same(a, b):
    assert np.array_equal(a[0], b[0])
    assert a[1] == b[1]
    assert np.array_equal(a[2], b[2])


CASES = [
    # (nx, ny, steps, background, extra params)
    (1024, 512, 3, False, {}),
    (1020, 516, 2, True, {"g": (0.1, -0.05), "boundtype": (P.BC_CONTCD4, P.BC_PERIODIC)}),
    (1016, 508, 2, False, {"boundtype": (P.BC_SYMM, P.BC_CONT)}),
    (1020, 500, 2, True, {"g": (0.2, -0.1), "boundtype": (P.BC_FIXED, P.BC_PERIODIC)}),
    (1024, 508, 2, False, {"boundtype": (P.BC_ASYMM, P.BC_FIXED)}),
    (1020, 512, 2, True, {"driver": P.DRIVER_GAUSS, "drv_amp": 0.05, "drv_period": 0.7,
                          "drv_x0": (3.0, 2.5, 0.0), "drv_sigma": (0.6, 0.8, 0.0)}),
]


@pytest.mark.parametrize("prec", [P.PREC_FP64, P.PREC_MIXED])
@pytest.mark.parametrize("integ", [P.INT_EULER, P.INT_RK4])
@pytest.mark.parametrize("nx,ny,steps,bg,kw", CASES)
def test_tma_matches_per_thread_staging(engine_lib, nx, ny, steps, bg, kw, integ, prec):
    w, pos, dx = ot_rect(nx, ny, seed=nx + 7 * ny)
    if bg:
        w = with_background(w)
    p = params_for(w, dx, integrator=integ, precision=prec, **kw)
    ref = run(engine_lib, w, pos, p, steps, 0)
    for staging in (1, 2):
        assert_same(run(engine_lib, w, pos, p, steps, staging), ref)


def test_small_grids_and_edge_tiles(engine_lib):
    """Grids of one or two tile rows and columns (every tile an edge tile,
    tile column 0 holding the single interior column x = 2)."""
    for nx, ny in [(4, 4), (28, 12), (32, 8), (60, 20), (92, 36)]:
        for integ in (P.INT_EULER, P.INT_RK4):
            w, pos, dx = ot_rect(nx, ny, seed=nx * ny + 1)
            p = params_for(w, dx, integrator=integ)
            ref = run(engine_lib, w, pos, p, 4, 0)
            for staging in (1, 2):
                assert_same(run(engine_lib, w, pos, p, 4, staging), ref)


def test_staging_availability(engine_lib):
    # rows of 42 doubles (336 bytes): FP64 yes, float (168 bytes) no
    w, pos, dx = ot_rect(38, 20)
    e = engine_lib.Engine(params_for(w, dx), w, pos)
    assert e.staging() == (0, True)
    e.close()
    e = engine_lib.Engine(params_for(w, dx, precision=P.PREC_MIXED), w, pos)
    assert e.staging() == (0, False)
    with pytest.raises(engine_lib.SmaugError) as ex:
        e.set_staging(1)
    assert ex.value.code == 6
    e.set_staging(0)
    with pytest.raises(engine_lib.SmaugError) as ex:
        e.set_staging(3)
    assert ex.value.code == 1
    e.close()
    # odd row length
    w, pos, dx = ot_rect(37, 20)
    e = engine_lib.Engine(params_for(w, dx), w, pos)
    assert e.staging() == (0, False)
    e.close()
    # the 6th-order stencil keeps the per-thread staging
    w, pos, dx = ot_rect(40, 20)
    e = engine_lib.Engine(params_for(w, dx, stencil_order=6), w, pos)
    assert e.staging() == (0, False)
    e.close()
