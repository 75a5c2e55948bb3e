"""Grid metric (initgrid restatement): the library's host implementation
agrees bit for bit with the oracle, including the reference's asymmetric
extrapolation of ghost positions (src/init.cu:2502-3060)."""
import numpy as np

from tests.util import ot_rect


def test_metric_uniform_matches_oracle(engine_lib, oracle):
    w, pos, dx = ot_rect(20, 12)
    pe, de = engine_lib.grid_metric(2, (24, 16), pos)
    po, do = oracle.grid_metric(2, (24, 16), pos)
    assert np.array_equal(pe, po) and np.array_equal(de, do)
    assert np.allclose(de[0], dx[0], rtol=1e-12) and np.allclose(de[1], dx[1], rtol=1e-12)


def test_metric_stretched_matches_oracle(engine_lib, oracle):
    n0, n1 = 18, 14
    x = np.cumsum(0.1 + 0.01 * np.arange(n0) ** 1.5)
    y = np.cumsum(0.2 + 0.02 * np.sin(np.arange(n1)))
    X, Y = np.meshgrid(x, y, indexing="xy")
    pos = np.stack([X, Y])
    pe, de = engine_lib.grid_metric(2, (n0, n1), pos)
    po, do = oracle.grid_metric(2, (n0, n1), pos)
    assert np.array_equal(pe, po) and np.array_equal(de, do)
    # interior: centred half-differences of the file positions
    assert np.allclose(de[0][5, 3:-3], 0.5 * (X[5, 4:-2] - X[5, 2:-4]), rtol=1e-14)
    # dim 0 lower: only index 0 is extrapolated (from 1, 2); dims > 0:
    # indices 0 and 1 (from 2, 3); upper: n-2, n-1 (from n-3, n-4)
    r = 4
    assert pe[0][r, 1] == X[r, 1]
    assert np.isclose(pe[0][r, 0], 2 * X[r, 1] - X[r, 2], rtol=1e-14)
    assert np.isclose(pe[0][r, n0 - 2], 2 * X[r, n0 - 3] - X[r, n0 - 4], rtol=1e-14)
    assert np.isclose(pe[0][r, n0 - 1], 3 * X[r, n0 - 3] - 2 * X[r, n0 - 4], rtol=1e-14)
    c = 3
    assert np.isclose(pe[1][1, c], 2 * Y[2, c] - Y[3, c], rtol=1e-14)
    assert np.isclose(pe[1][0, c], 3 * Y[2, c] - 2 * Y[3, c], rtol=1e-14)
    assert np.isclose(pe[1][n1 - 1, c], 3 * Y[n1 - 3, c] - 2 * Y[n1 - 4, c], rtol=1e-14)
