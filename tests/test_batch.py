"""Batched ensemble (smaug_batch_*): runs of different sizes, boundary types,
backgrounds and drivers advanced together must reproduce each run stepped
alone through smaug_step.  Tolerance: relative L2 per evolved field <= 1e-12
(FP64) and <= 1e-6 (mixed form: the two launch paths may contract multiply-adds
differently in the float hyperdiffusion)."""
import numpy as np
import pytest

from smaug_b200 import ic, params as P
from tests.util import ot_rect, params_for, rel_l2

pytestmark = pytest.mark.gpu


def slab(nz, nx, period, seed):
    """stratified driven slab (vertical = dim 0), as in the ensemble benchmark"""
    w, pos, dx = ic.stratified(nz=nz, nx=nx, seed=seed, vz_sigma=10.0)
    p = P.make_params(ndim=2, n=(nz + 4, nx + 4, 1), dx=dx, courant=0.3, dtmax=1.0,
                      integrator=P.INT_RK4, g=(-274.0, 0.0),
                      boundtype=(P.BC_CONTCD4, P.BC_PERIODIC), driver=P.DRIVER_GAUSS,
                      drv_amp=200.0, drv_period=period, drv_x0=(0.1e6, 1.0e6),
                      drv_sigma=(0.2e6, 0.2e6))
    return p, w, pos


def ensemble(precision):
    runs = []
    for (nx, ny, seed) in [(64, 64, 1), (96, 80, 2), (37, 29, 3), (128, 128, 4)]:
        w, pos, dx = ot_rect(nx, ny, seed=seed)
        runs.append((params_for(w, dx, integrator=P.INT_RK4, precision=precision), w, pos))
    p, w, pos = slab(48, 64, 30.0, 5)
    p.precision = precision
    runs.append((p, w, pos))
    # fixed and antisymmetric ghosts in the same launch
    w, pos, dx = ot_rect(40, 36, seed=6)
    runs.append((params_for(w, dx, integrator=P.INT_RK4, precision=precision,
                            boundtype=(P.BC_FIXED, P.BC_PERIODIC)), w, pos))
    w, pos, dx = ot_rect(34, 30, seed=7)
    w[:6] *= 0.01
    w[6], w[7], w[8], w[9] = 2.0, 1.0, 0.1, 0.05
    runs.append((params_for(w, dx, integrator=P.INT_RK4, precision=precision,
                            boundtype=(P.BC_ASYMM, P.BC_CONTCD4)), w, pos))
    return runs


@pytest.mark.parametrize("form", [None, "per-stage", "persistent"])
@pytest.mark.parametrize("pin", [None, (32, 8), (16, 16)])
@pytest.mark.parametrize("precision,tol", [(P.PREC_FP64, 1e-12), (P.PREC_MIXED, 1e-6)])
def test_batch_matches_single_runs(engine_lib, precision, tol, pin, form):
    """Every run of a batch against the same run stepped alone, with the tile
    shape chosen by the autotuner or pinned to each built shape (the
    single-run kernel uses 32x8 tiles), and the launch form chosen by the
    autotuner or pinned to per-stage launches or to the persistent launch
    (several steps per launch, a grid barrier between stages)."""
    runs = ensemble(precision)
    b = engine_lib.Batch([r[0] for r in runs], [r[1] for r in runs], [r[2] for r in runs])
    if pin:
        b.pin_tile_shape(*pin)
    b.pin_form(form)
    # up to 10 tuning steps, single steps, a 6-step graph cycle from step 12,
    # single steps
    nfirst = 20
    b.step(nfirst)
    shape = b.launch_shape()
    pers = b.persistent()
    assert pers["on"] == (form == "persistent") or form is None
    if pers["on"]:
        tile = b.tile_shape()["tile"]
        assert shape["grid"] == pers["grid"]["%dx%d" % tile] > 0
    else:
        assert shape["grid"] in shape["candidates"]
    tile = b.tile_shape()
    assert tile["tile"] in ((32, 8), (16, 16))
    if pin:
        assert tile["tile"] == pin
    elif form is None:
        assert all(v > 0 for v in tile["ms"]["32x8"] + tile["ms"]["16x16"])
        assert all(v > 0 for v in pers["ms"].values())
    for i, (p, w, pos) in enumerate(runs):
        e = engine_lib.Engine(p, w, pos)
        e.step(nfirst)
        ref = e.state()
        it, t, dt = e.time()
        e.close()
        got = b.state(i)
        for f in range(6):
            assert rel_l2(got[f], ref[f]) <= tol, (i, f, rel_l2(got[f], ref[f]))
        assert np.array_equal(got[6:], ref[6:])
        bit, bt, bdt = b.time(i)
        assert bit == it == nfirst
        assert abs(bt - t) <= 1e-12 * abs(t)
    b.step(7)  # continues from a step that is not 0 mod 6
    for i, (p, w, pos) in enumerate(runs[:2]):
        e = engine_lib.Engine(p, w, pos)
        e.step(nfirst + 7)
        ref = e.state()
        e.close()
        got = b.state(i)
        for f in range(6):
            assert rel_l2(got[f], ref[f]) <= tol
    b.close()


def test_batch_rejects(engine_lib):
    w, pos, dx = ot_rect(32, 32, seed=1)
    pe = params_for(w, dx, integrator=P.INT_EULER)
    with pytest.raises(engine_lib.SmaugError) as e:
        engine_lib.Batch([pe], [w], [pos])
    assert e.value.code == 6
    p64 = params_for(w, dx, integrator=P.INT_RK4)
    pmx = params_for(w, dx, integrator=P.INT_RK4, precision=P.PREC_MIXED)
    with pytest.raises(engine_lib.SmaugError) as e:
        engine_lib.Batch([p64, pmx], [w, w], [pos, pos])
    assert e.value.code == 6


def test_batch_pin_tile_shape_rejects(engine_lib):
    """Only built tile shapes can be pinned, and only before the first step."""
    w, pos, dx = ot_rect(40, 40, seed=1)
    p = params_for(w, dx, integrator=P.INT_RK4)
    b = engine_lib.Batch([p], [w], [pos])
    with pytest.raises(engine_lib.SmaugError) as e:
        b.pin_tile_shape(8, 8)
    assert e.value.code == 1
    assert b.tile_shape()["tile"] == (0, 0)
    b.step(1)
    with pytest.raises(engine_lib.SmaugError) as e:
        b.pin_tile_shape(16, 16)
    assert e.value.code == 1
    with pytest.raises(engine_lib.SmaugError) as e:
        b.pin_form("persistent")
    assert e.value.code == 1
    b.close()
