"""The allocation-free Euler step (smaug_euler_step_noalloc) against the
engine's regular Euler step, through the C ABI.

The entry point serves callers that cannot call cudaMalloc -- applications that
reserve their device memory up front, plugins whose host forbids allocating in
its step callback, loops that cudaFree's device-wide synchronisation would
stall -- so its scratch lives in one static device array.  The test owns the device buffers (torch), calls the
entry point twice in a row (the second call reuses the array with the first
call's leftovers), and checks both outputs against two regular steps:
relative L2 per evolved field <= 1e-12, the same tolerance as the parity tests.
This file is named to be collected last.
"""
import numpy as np
import pytest

from tests.util import ot_rect, params_for, rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-12


def test_noalloc_two_steps_match_engine(engine_lib):
    import torch
    w, pos, dx = ot_rect(45, 38, seed=21)
    p = params_for(w, dx)
    eng = engine_lib.Engine(p, w, pos)
    s0 = eng.state()                      # initial state with ghost layers filled
    eng.step(1)
    s1 = eng.state()
    dt1 = eng.time()[2]
    eng.step(1)
    s2 = eng.state()
    dt2 = eng.time()[2]
    eng.close()

    _, delx = engine_lib.grid_metric(2, (p.n[0], p.n[1]), pos)
    delx1d = np.concatenate([delx[0][2, :], delx[1][:, 2]])
    dev = torch.device("cuda", torch.cuda.current_device())
    a = torch.from_numpy(s0).to(dev)
    b = torch.empty_like(a)
    c = torch.empty_like(a)
    torch.cuda.synchronize()
    dt = engine_lib.euler_step_noalloc(p, a.data_ptr(), b.data_ptr(), delx1d, p.dt)
    got1 = b.cpu().numpy()
    dt = engine_lib.euler_step_noalloc(p, b.data_ptr(), c.data_ptr(), delx1d, dt)
    got2 = c.cpu().numpy()
    for got, ref in ((got1, s1), (got2, s2)):
        for f in range(6):
            assert rel_l2(got[f], ref[f]) <= TOL, (f, rel_l2(got[f], ref[f]))
        assert np.array_equal(got[6:], ref[6:])
    assert abs(dt - dt2) <= 1e-14 * dt2


def test_noalloc_rejects_oversize_grid(engine_lib):
    p = params_for(np.zeros((10, 16, 9000)), (0.1, 0.1))
    with pytest.raises(engine_lib.SmaugError) as e:
        engine_lib.euler_step_noalloc(p, 1, 2, np.ones(9016), 1e-3)
    assert e.value.code == 6 and "8192" in str(e.value)
