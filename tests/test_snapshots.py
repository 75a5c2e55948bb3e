"""Asynchronous .out snapshots (smaug_write_out_async / smaug_wait_writes):
the files equal, byte for byte, those of the synchronous writer at the same
steps, while the engine keeps stepping between the calls; write errors
surface in smaug_wait_writes."""
import pytest

from smaug_b200 import params as P
from tests.util import ot_rect, params_for

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [P.PREC_FP64, P.PREC_MIXED])
def test_async_snapshots_equal_sync(engine_lib, tmp_path, prec):
    w, pos, dx = ot_rect(48, 40, seed=3)
    p = params_for(w, dx, integrator=P.INT_RK4, precision=prec)
    a = engine_lib.Engine(p, w, pos)
    b = engine_lib.Engine(p, w, pos)
    plan = [2, 3, 1, 4, 2]  # steps before each snapshot; the third reuses the first buffer
    for k, n in enumerate(plan):
        a.step_async(n)
        a.write_out_async(str(tmp_path / ("a%d.out" % k)), name="snap", it=k, t=0.25 * k)
        b.step(n)
        b.write_out(str(tmp_path / ("b%d.out" % k)), name="snap", it=k, t=0.25 * k)
    a.wait_writes()
    a.sync()
    for k in range(len(plan)):
        fa = (tmp_path / ("a%d.out" % k)).read_bytes()
        fb = (tmp_path / ("b%d.out" % k)).read_bytes()
        assert len(fa) > 0 and fa == fb, k
    a.close()
    b.close()


def test_async_snapshot_error_is_reported(engine_lib, tmp_path):
    w, pos, dx = ot_rect(24, 24, seed=1)
    e = engine_lib.Engine(params_for(w, dx), w, pos)
    e.step(1)
    e.write_out_async(str(tmp_path / "missing_dir" / "x.out"), it=1, t=0.0)
    e.write_out_async(str(tmp_path / "ok.out"), it=1, t=0.0)
    with pytest.raises(engine_lib.SmaugError) as err:
        e.wait_writes()
    assert err.value.code == 4          # SMAUG_E_IO
    assert (tmp_path / "ok.out").stat().st_size > 0
    e.wait_writes()                     # the error was reported once
    e.close()
