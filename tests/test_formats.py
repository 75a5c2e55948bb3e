"""Format boundary: .ini reader and .out writer of the library (host code,
CPU-safe) against the reference layouts (src/readwrite.c:160-366,975-1082;
.out read layout of python/smaug-read2.py:24-61)."""
import ctypes
import os
import struct

import numpy as np
import pytest

from smaug_b200 import formats
from tests.util import ot_rect, params_for

from oracle.build_ref import REFROOT  # noqa: E402  (SMAUG_REFERENCE overrides)

REF_TILE = os.path.join(REFROOT, "configs", "zero1_ot_asc_252_np0202_000.ini")


def test_ini_roundtrip_c_reader(engine_lib, tmp_path):
    w, pos, dx = ot_rect(13, 9)
    path = str(tmp_path / "a.ini")
    formats.write_ini(path, w, pos)
    w2, pos2, it, t = engine_lib.read_ini(path, 2, (17, 13))
    assert np.array_equal(w, w2) and np.array_equal(pos, pos2)
    assert it == 0 and t == 0.0


def test_ini_python_reader_matches(engine_lib, tmp_path):
    w, pos, dx = ot_rect(11, 10)
    path = str(tmp_path / "b.ini")
    formats.write_ini(path, w, pos)
    w2, pos2, hdr = formats.read_ini(path, 2)
    assert np.array_equal(w, w2) and np.array_equal(pos, pos2)
    assert hdr["n"] == [15, 14]


def test_ini_errors(engine_lib, tmp_path):
    w, pos, dx = ot_rect(8, 8)
    path = str(tmp_path / "c.ini")
    formats.write_ini(path, w, pos)
    with pytest.raises(engine_lib.SmaugError) as e:
        engine_lib.read_ini(path, 2, (13, 12))        # wrong grid
    assert e.value.code == 5
    lines = open(path).read().splitlines()
    open(path, "w").write("\n".join(lines[:-3]) + "\n")  # truncated
    with pytest.raises(engine_lib.SmaugError) as e:
        engine_lib.read_ini(path, 2, (12, 12))
    assert e.value.code == 5
    with pytest.raises(engine_lib.SmaugError) as e:
        engine_lib.read_ini(str(tmp_path / "missing.ini"), 2, (12, 12))
    assert e.value.code == 4


def test_out_writer_layout(engine_lib, tmp_path):
    w, pos, dx = ot_rect(7, 6)
    p = params_for(w, dx, g=(0.5, -0.25))
    path = str(tmp_path / "x.out")
    dp = ctypes.POINTER(ctypes.c_double)
    rc = engine_lib.lib().smaug_write_out_host(
        path.encode(), ctypes.byref(p), w.ctypes.data_as(dp), pos.ctypes.data_as(dp),
        b"test1", 42, 1.25)
    assert rc == 0
    buf = open(path, "rb").read()
    # 79 name | int it | double t | 3 ints | 2 ints | 6 doubles | 79 names | data | '\n'
    assert buf[:5] == b"test1" and buf[5:79] == b"\0" * 74
    assert struct.unpack_from("<i", buf, 79)[0] == 42
    assert struct.unpack_from("<d", buf, 83)[0] == 1.25
    assert struct.unpack_from("<3i", buf, 91) == (2, 6, 10)
    assert struct.unpack_from("<2i", buf, 103) == (11, 10)
    assert struct.unpack_from("<6d", buf, 111) == (p.gamma, 0.0, 0.5, -0.25, 0.0, 0.0)
    assert buf[159:159 + 38] == b"x y rho mx my e bx by  gamma eta g1 g2"
    ncell = 11 * 10
    assert len(buf) == 238 + 12 * ncell * 8 + 1 and buf[-1:] == b"\n"
    w2, pos2, hdr = formats.read_out(path)
    assert np.array_equal(w2, w) and np.array_equal(pos2, pos)
    assert hdr["it"] == 42 and hdr["t"] == 1.25 and hdr["n"] == [11, 10]


def test_python_out_writer_matches_c(engine_lib, tmp_path):
    w, pos, dx = ot_rect(5, 7)
    p = params_for(w, dx)
    a, b = str(tmp_path / "a.out"), str(tmp_path / "b.out")
    dp = ctypes.POINTER(ctypes.c_double)
    assert engine_lib.lib().smaug_write_out_host(a.encode(), ctypes.byref(p),
                                                 w.ctypes.data_as(dp), pos.ctypes.data_as(dp),
                                                 b"run", 3, 0.5) == 0
    formats.write_out(b, w, pos, p.gamma, it=3, t=0.5, name="run")
    assert open(a, "rb").read() == open(b, "rb").read()


@pytest.mark.skipif(not os.path.exists(REF_TILE), reason="reference checkout not present")
def test_reads_reference_ot_tile(engine_lib):
    """One of the reference's own 126x126 OT tiles (no ghost layers): both
    readers agree and the values carry the documented OT constants."""
    w, pos, hdr = formats.read_ini(REF_TILE, 2)
    assert hdr["n"] == [126, 126] and hdr["name"].startswith("opozmf_mhd22")
    assert w.shape == (10, 126, 126)
    assert np.allclose(w[0], 25.0 / (36.0 * np.pi), rtol=1e-9)
    assert abs(pos[0, 0, 0] - 1.0 / 504.0) < 1e-12 and abs(pos[1, 0, 0] - 1.0 / 504.0) < 1e-12
    assert abs(hdr["eqpar"][0] - 1.66667) < 1e-5
    w2, pos2, it, t = engine_lib.read_ini(REF_TILE, 2, (126, 126))
    assert np.array_equal(w2, w) and np.array_equal(pos2, pos)
