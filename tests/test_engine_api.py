"""C-ABI behaviour: errors, state round trips, determinism, chunking,
non-finite detection, .out output."""
import ctypes

import numpy as np
import pytest

from smaug_b200 import formats, params as P
from tests.util import ot_rect, params_for

pytestmark = pytest.mark.gpu


def test_invalid_params_rejected(engine_lib):
    w, pos, dx = ot_rect(16, 16)
    for kw, code in [({"integrator": 7}, 1), ({"pad_model": 9}, 1), ({"boundtype": (1, 0)}, 6),
                     ({"gamma": 1.0}, 1)]:
        p = params_for(w, dx, **kw)
        with pytest.raises(engine_lib.SmaugError) as e:
            engine_lib.Engine(p, w, pos)
        assert e.value.code == code, kw
    p = params_for(w, dx)
    p.version = 99
    with pytest.raises(engine_lib.SmaugError) as e:
        engine_lib.Engine(p, w, pos)
    assert e.value.code == 1
    p = params_for(w, dx)
    p.n[0] = 7
    with pytest.raises((engine_lib.SmaugError, ValueError)):
        engine_lib.Engine(p, w[:, :, :7].copy(), pos[:, :, :7].copy())


def test_null_handle(engine_lib):
    L = engine_lib.lib()
    assert L.smaug_step(None, 1) == 1
    assert L.smaug_destroy(None) == 0


def test_state_roundtrip_and_determinism(engine_lib):
    w, pos, dx = ot_rect(40, 33, seed=4)
    p = params_for(w, dx, integrator=P.INT_RK4)
    a = engine_lib.Engine(p, w, pos)
    s0 = a.state()
    assert np.array_equal(s0[6:], w[6:])
    a.step(4)
    b = engine_lib.Engine(p, w, pos)
    b.step(1).step(3)
    assert np.array_equal(a.state(), b.state())          # chunking
    assert a.time() == b.time()
    mid = a.state()
    a.set_state(mid)
    a.step(2)
    b.step(2)
    assert np.array_equal(a.state(), b.state())          # set_state is exact
    a.close()
    b.close()


def test_zero_steps(engine_lib):
    w, pos, dx = ot_rect(12, 12)
    e = engine_lib.Engine(params_for(w, dx), w, pos)
    s = e.state()
    e.step(0)
    assert np.array_equal(s, e.state())
    assert e.time()[0] == 0


def test_nonfinite_detected(engine_lib):
    w, pos, dx = ot_rect(20, 20)
    w[0, 10, 10] = np.nan
    p = params_for(w, dx, moddton=0, dt=1e-3)
    e = engine_lib.Engine(p, w, pos)
    with pytest.raises(engine_lib.SmaugError) as err:
        e.step(1)
    assert err.value.code == 7
    e.close()


def test_write_out(engine_lib, tmp_path):
    w, pos, dx = ot_rect(10, 9, seed=8)
    p = params_for(w, dx)
    e = engine_lib.Engine(p, w, pos)
    e.step(2)
    path = str(tmp_path / "s.out")
    e.write_out(path, name="test1", it=2, t=0.5)
    w2, pos2, hdr = formats.read_out(path)
    assert np.array_equal(w2, e.state())
    assert hdr["it"] == 2 and hdr["t"] == 0.5 and hdr["n"] == [14, 13]
    e.close()


def test_3d_roundtrip_and_write_out(engine_lib, tmp_path):
    from tests.util import params3, state3d
    w, pos, dx = state3d(9, 7, 6, seed=4)
    p = params3(w, dx)
    e = engine_lib.Engine(p, w, pos)
    e.step(2)
    st = e.state()
    assert st.shape == (13, 10, 11, 13)
    assert np.array_equal(st[8:], w[8:])          # backgrounds carried unchanged
    e.set_state(st)
    assert np.array_equal(e.state(), st)
    path = str(tmp_path / "s3.out")
    e.write_out(path, name="tube", it=2, t=0.25)
    w2, pos2, hdr = formats.read_out(path)
    assert np.array_equal(w2, st)
    assert hdr["ndim"] == 3 and hdr["nw"] == 13 and hdr["n"] == [13, 11, 10]
    e.close()


def test_3d_too_small_is_rejected(engine_lib):
    p = P.make_params(ndim=3, n=(12, 12, 7))
    with pytest.raises(engine_lib.SmaugError) as e:
        engine_lib.Engine(p, np.zeros((13, 7, 12, 12)), np.zeros((3, 7, 12, 12)))
    assert e.value.code == 1


def test_noalloc_rejects_3d(engine_lib):
    """Rejected on the parameter block, before any pointer is used."""
    p = P.make_params(ndim=3, n=(12, 12, 12))
    d = np.zeros(36)
    with pytest.raises(engine_lib.SmaugError) as e:
        engine_lib.euler_step_noalloc(p, 1, 2, d, 1e-3)
    assert e.value.code == 6


def test_get_fields_subsets(engine_lib):
    """smaug_get_fields: any contiguous range of fields equals the same rows of
    smaug_get_state, across the evolved/background boundary too."""
    w, pos, dx = ot_rect(24, 20, seed=3)
    w[7] = 0.1
    e = engine_lib.Engine(params_for(w, dx, integrator=P.INT_RK4), w, pos)
    e.step(2)
    full = e.state()
    for f0, nf in [(0, 6), (0, 10), (3, 1), (5, 3), (6, 4), (9, 1)]:
        got = e.fields(f0, nf)
        assert np.array_equal(got, full[f0:f0 + nf]), (f0, nf)
    with pytest.raises(engine_lib.SmaugError):
        e.fields(8, 3)
    e.close()

