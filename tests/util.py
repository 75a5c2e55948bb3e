"""Helpers shared by the tests: initial states and error norms."""
import math

import numpy as np

from smaug_b200 import ic, params as P
import smaug_b200.ic as I


def rel_l2(a, b):
    """relative L2 error of a against reference b (absolute if b == 0)."""
    n = float(np.sqrt(np.sum(np.asarray(b, dtype=np.float64) ** 2)))
    d = float(np.sqrt(np.sum((np.asarray(a, dtype=np.float64) - b) ** 2)))
    return d / n if n > 0 else d


def ot_rect(nx, ny, seed=1, noise=1e-3, gamma=5.0 / 3.0):
    """Orszag-Tang on [0,2pi]^2 with nx x ny interior cells and seeded rho noise."""
    x, dx = I._axis(nx, 0, 2 * math.pi)
    y, dy = I._axis(ny, 0, 2 * math.pi)
    X, Y = np.meshgrid(x, y, indexing="xy")
    rng = np.random.default_rng(seed)
    rho = 25 / (36 * math.pi) * (1 + noise * rng.standard_normal(X.shape))
    b0 = 1 / math.sqrt(4 * math.pi)
    w = np.zeros((10,) + X.shape)
    w[0] = rho
    w[1] = -rho * np.sin(Y)
    w[2] = rho * np.sin(X)
    w[4] = -b0 * np.sin(Y)
    w[5] = b0 * np.sin(2 * X)
    w[3] = 5 / (12 * math.pi) / (gamma - 1) + 0.5 * (w[1] ** 2 + w[2] ** 2) / rho \
        + 0.5 * (w[4] ** 2 + w[5] ** 2)
    return w, np.stack([X, Y]), (dx, dy)


def with_background(w, seed=3, amp=0.05):
    """Add smooth nonzero background fields (energyb, rhob, b1b, b2b) and keep
    the total state the same, exercising the split-form coupling terms."""
    w = w.copy()
    ny, nx = w.shape[1:]
    jj, ii = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    rb = 0.1 * (1 + 0.2 * np.sin(2 * math.pi * ii / nx))
    w[7] = rb
    w[0] = w[0] - rb
    w[8] = amp * np.cos(2 * math.pi * jj / ny)
    w[9] = amp * 0.5
    w[6] = 0.05 + 0.01 * np.cos(2 * math.pi * ii / nx)
    w[3] = w[3] - w[6]
    return w


def params_for(w, dx, **kw):
    n = list(reversed(w.shape[1:]))
    kw.setdefault("courant", 0.3)
    kw.setdefault("dtmax", 1.0)
    return P.make_params(ndim=2, n=(n[0], n[1], 1), dx=dx, **kw)


def state3d(nx, ny, nz, seed=0, background=True):
    """3D state on [0,0.1]^3 (the generator of the 3D golden fixtures):
    nonzero backgrounds, or with background=False the same total state folded
    into the perturbation fields.  Returns (w[13], pos[3], dx)."""
    from tests.golden.make_golden import L3, tube_state
    w, pos = tube_state(nx, ny, nz, seed)
    if not background:
        w[0] += w[9]
        w[4] += w[8]
        for c in range(3):
            w[5 + c] += w[10 + c]
        w[8:] = 0.0
    return w, pos, (L3 / nx, L3 / ny, L3 / nz)


def params3(w, dx, boundtype=(P.BC_CONTCD4,) * 3, **kw):
    n = list(reversed(w.shape[1:]))
    kw.setdefault("courant", 0.3)
    kw.setdefault("dtmax", 1.0)
    return P.make_params(ndim=3, n=tuple(n), dx=dx, boundtype=boundtype, **kw)
