"""Initial-condition generators for the benchmark configurations.

The reference ships only initial-state .ini fixtures and its IDL generators
(magfield/make_ini_file_2D_murawski1.pro); the single-GPU Orszag-Tang input
(configs/zero1_ot_asc.ini) is absent from the checkout, so these generators
produce the reference-format arrays directly: w[NVAR, ...] in the field order
of include/iotypes.h:209-216 and pos[NDIM, ...] cell positions, ghosts
included (2 layers per side).  Arrays are numpy, shape (nvar, [n2,] n1, n0).
"""
import math

import numpy as np

from .params import field_ids


def _axis(n, lo, hi):
    """cell centres of an n-cell interior on [lo, hi] plus 2 ghost layers."""
    dx = (hi - lo) / n
    return lo + (np.arange(n + 4) - 2 + 0.5) * dx, dx


def orszag_tang(N=128, L=2.0 * math.pi, gamma=5.0 / 3.0, noise=0.0, seed=0):
    """2D Orszag-Tang vortex on [0,L]^2, N x N interior cells.

    rho = 25/(36 pi), p = 5/(12 pi), v = (-sin y, sin x),
    B = (-sin y, sin 2x)/sqrt(4 pi) with x,y scaled to [0, 2 pi); background
    fields zero.  `noise` adds seeded relative white noise to rho
    (numpy default_rng(seed)).
    Returns (w, pos, dx) with w shape (10, N+4, N+4).
    """
    ids = field_ids(2)
    x, dx = _axis(N, 0.0, L)
    y, dy = _axis(N, 0.0, L)
    X, Y = np.meshgrid(x, y, indexing="xy")        # shape (n1, n0): [j, i]
    k = 2.0 * math.pi / L
    rho = np.full_like(X, 25.0 / (36.0 * math.pi))
    if noise:
        rng = np.random.default_rng(seed)
        rho = rho * (1.0 + noise * rng.standard_normal(rho.shape))
    p = 5.0 / (12.0 * math.pi)
    vx = -np.sin(k * Y)
    vy = np.sin(k * X)
    b0 = 1.0 / math.sqrt(4.0 * math.pi)
    bx = -b0 * np.sin(k * Y)
    by = b0 * np.sin(2.0 * k * X)
    e = p / (gamma - 1.0) + 0.5 * rho * (vx * vx + vy * vy) + 0.5 * (bx * bx + by * by)
    w = np.zeros((10,) + X.shape)
    w[ids["rho"]] = rho
    w[ids["mom1"]] = rho * vx
    w[ids["mom2"]] = rho * vy
    w[ids["energy"]] = e
    w[ids["b1"]] = bx
    w[ids["b2"]] = by
    pos = np.stack([X, Y])
    return w, pos, (dx, dy)


MU0 = 4.0e-7 * math.pi
KB = 1.380649e-23
MP = 1.67262192e-27


def temperature_profile(z, t_low=6.0e3, t_high=1.0e6, z_tr=2.0e6, width=0.2e6):
    """T(z) = t_low + (t_high - t_low) * 0.5 * (1 + tanh((z - z_tr)/width))."""
    return t_low + (t_high - t_low) * 0.5 * (1.0 + np.tanh((z - z_tr) / width))


def hydrostatic(z, rho0=2.7e-4, mu=0.6, g=274.0, **tkw):
    """rho_b(z), p_b(z) by integrating dp/dz = -rho g with p = rho kB T/(mu mp)
    upward from rho(z[0]) = rho0 (trapezoidal in ln p)."""
    T = temperature_profile(z, **tkw)
    H = KB * T / (mu * MP * g)          # pressure scale height
    lnp = np.empty_like(z)
    lnp[0] = math.log(rho0 * KB * T[0] / (mu * MP))
    for i in range(1, len(z)):
        lnp[i] = lnp[i - 1] - 0.5 * (z[i] - z[i - 1]) * (1.0 / H[i] + 1.0 / H[i - 1])
    p = np.exp(lnp)
    rho = p * mu * MP / (KB * T)
    return rho, p


def stratified(nz=256, nx=256, ny=None, zrange=(0.0, 6.0e6), xrange=(0.0, 2.0e6),
               yrange=(0.0, 2.0e6), gamma=5.0 / 3.0, b_gauss=10.0, seed=None,
               vz_sigma=0.0, smooth_cells=3):
    """Stratified solar atmosphere, vertical axis = dimension 0 (SMAUG's
    convention for gravity along x, models/iosmaugparams.h.fluxtube1).

    2D when ny is None: shape (10, nx+4, nz+4); 3D: (13, ny+4, nx+4, nz+4).
    Background: rho_b, e_b = p_b/(gamma-1) + B_b^2/2 with a uniform vertical
    B_b = b_gauss * 1e-4 T / sqrt(mu0) (SAC units,
    magfield/make_ini_file_2D_murawski1.pro:128-130,230).  Perturbations zero,
    except an optional seeded Gaussian-smoothed vertical velocity with
    standard deviation vz_sigma [m/s].
    """
    ndim = 2 if ny is None else 3
    ids = field_ids(ndim)
    z, dz = _axis(nz, *zrange)
    x, dxx = _axis(nx, *xrange)
    rho_b, p_b = hydrostatic(z)
    bz = b_gauss * 1.0e-4 / math.sqrt(MU0)
    eb = p_b / (gamma - 1.0) + 0.5 * bz * bz
    if ndim == 2:
        shape = (nx + 4, nz + 4)
        Z = np.broadcast_to(z[None, :], shape).copy()
        X = np.broadcast_to(x[:, None], shape).copy()
        pos = np.stack([Z, X])
        dx = (dz, dxx)
    else:
        y, dy = _axis(ny, *yrange)
        shape = (ny + 4, nx + 4, nz + 4)
        Z = np.broadcast_to(z[None, None, :], shape).copy()
        X = np.broadcast_to(x[None, :, None], shape).copy()
        Y = np.broadcast_to(y[:, None, None], shape).copy()
        pos = np.stack([Z, X, Y])
        dx = (dz, dxx, dy)
    w = np.zeros((4 + 3 * ndim,) + shape)
    bshape = (1,) * (ndim - 1) + (nz + 4,)
    w[ids["rhob"]] = rho_b.reshape(bshape)
    w[ids["energyb"]] = eb.reshape(bshape)
    w[ids["b1b"]] = bz
    if vz_sigma and seed is not None:
        rng = np.random.default_rng(seed)
        v = rng.standard_normal(shape).astype(np.float32).astype(np.float64)
        v = _gauss_smooth(v, smooth_cells)
        v *= vz_sigma / max(np.std(v), 1e-300)
        w[ids["mom1"]] = v * w[ids["rhob"]]
    return w, pos, dx


def _gauss_smooth(a, s):
    if s <= 0:
        return a
    r = int(3 * s)
    k = np.exp(-0.5 * (np.arange(-r, r + 1) / s) ** 2)
    k /= k.sum()
    out = a
    for ax in range(a.ndim):
        out = np.apply_along_axis(lambda v: np.convolve(np.pad(v, r, mode="wrap"), k, "valid"),
                                  ax, out)
    return out
