"""The CUDA engine against the reference's own outputs (tests/golden/),
through the C ABI.  Tolerance: relative L2 per evolved field <= 1e-13."""
import numpy as np
import pytest

from tests import golden_util as G
from tests.util import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-13


@pytest.mark.parametrize("name", G.STRICT + G.BOUNDARY)
def test_engine_matches_reference_run(engine_lib, name):
    d = G.load(name)
    p = G.params(d)
    e = engine_lib.Engine(p, d["w0full"], d["pos"])
    done = 0
    for k, ref in zip(d["steps"], d["states"]):
        e.step(int(k) - done)
        done = int(k)
        got = e.state()
        for f in range(6):
            assert rel_l2(got[f], ref[f]) <= TOL, (name, k, f, rel_l2(got[f], ref[f]))
    e.close()


@pytest.mark.parametrize("name", G.ONESTEP)
def test_engine_one_step_multiblock(engine_lib, name):
    d = G.load(name)
    p = G.params(d)
    n0 = d["w0"].shape[2]
    mask = np.ones(d["w0"].shape[1:], bool)
    mask[:, [1, n0 - 3]] = False
    for a in range(len(d["steps"]) - 1):
        e = engine_lib.Engine(p, G.full(d["states"][a]), d["pos"])
        e.step(1)
        got = e.state()
        e.close()
        for f in range(6):
            assert rel_l2(got[f][mask], d["states"][a + 1][f][mask]) <= TOL
