"""Generate the golden fixtures of tests/golden/ from the reference itself.

The reference (mikeg64/smaug) has no tests and ships no golden outputs, so
these fixtures are produced by running the reference's own GPU binary (built
from its sources by oracle/build_ref.py) on a B200, on inputs written here:

  python tests/golden/make_golden.py prepare   # here: .ini inputs + reference builds
  python tests/golden/make_golden.py run --runs DIR      # on a GPU machine: run the binaries
  python tests/golden/make_golden.py collect --runs DIR  # here: .out files -> *.npz fixtures
(an optional comma-separated list of case names after the command selects cases)

Cases (Orszag-Tang on [0,2pi]^2, seeded 1e-3 rho noise, the reference OT
model parameters with PGAMMA 1.66666667, courant 0.3, DT 1, moddton on):
  g16      16x16 interior, 20 steps   -- one thread block: race-free
  g18x12   18x12 interior, 20 steps   -- one thread block: race-free
  ot64     64x64 interior, 11 steps   -- multi-block (17 thread blocks)
  ot24x20  24x20 interior, steps 0-5  -- multi-block, consecutive steps for
           one-step parity away from the column the pad race can touch
  ot128    128x128 interior, steps 1, 50, 200 -- the 128^2/200-step
           configuration (34 blocks), run twice on the GPU box
The reference launches one thread per cell in 512-thread blocks; its
hyperdifvisc1r_parallel stores tmp6 through the wrong index (encode3) into
the padded array while the same launch zeroes it.  Inside one block the
stray store lands last; across blocks the order is not fixed, which can
change nu_r in the last interior column along dim 0.
Each .npz holds the evolved fields (rho m1 m2 e b1 b2, ghosts included) of
the initial state and of the saved steps, the positions, and the header
times of the reference's .out files.

3D cases (flux-tube model build, -DUSE_SAC_3D, contcd4 ghosts in every
dimension, domain [0,0.1]^3, gravity -0.1 along dim 0, nonzero background
fields, DT 1, courant 0.3, chyp 0.2, PGAMMA 1.66666667):
  t3s      4x4x4 interior (8^3 = 512 cells: one thread block), 20 steps
  t3a      12x12x8 interior (16x16x12 = 6 blocks), steps 0-5 and 10
  t3b      20x12x8 interior (24x16x12 = 9 blocks), steps 0-3
6th-order flux derivative (the reference built with -DUSE_DORDER3,
src/gradops.cu:450-453; one thread block each):
  d16      2D, as g16 with seed 15, 20 steps
  d3s      3D, as t3s with seed 25, 20 steps
Every 3D grid holds a whole number of 512-thread blocks: the reference's
contcd4 ghost kernels (models/boundary.cu.fluxtube1:16-85) have no
cell-count guard, so a partial last block would write past the state array.
The 3D fixtures hold all 13 fields (the backgrounds included).
"""
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

WORK = os.path.join(HERE, "_inputs")          # git-ignored; travels to the GPU box
# directory holding the reference runs' .out files (one sub-directory per
# case): `run` writes it on the GPU machine, `collect` reads it here after the
# caller has copied it back.  `--runs DIR` or SMAUG_GOLDEN_RUNS selects it;
# the default is git-ignored.
RUNS = os.environ.get("SMAUG_GOLDEN_RUNS", os.path.join(HERE, "_runs"))

# name: (nx, ny, seed, NT, steps kept[, boundary types per dim])
CASES = {
    "g16": (16, 16, 11, 21, [1, 2, 3, 5, 10, 20]),
    "g18x12": (18, 12, 12, 21, [1, 2, 3, 5, 10, 20]),
    "ot64": (64, 64, 1, 12, [1, 11]),
    "ot24x20": (24, 20, 5, 12, [0, 1, 2, 3, 4, 5]),
    # the small benchmark configuration: 128^2, 200 steps (34 thread blocks)
    "ot128": (128, 128, 2, 201, [1, 50, 200]),
    # fixed (5) ghosts: the OT model's cuboundary (src/boundary.cu:231-252)
    # dispatches periodic only, so type 5 leaves the ghost layers as read
    # from the .ini; the gradient edge zeroing of non-periodic types applies
    "f16x": (16, 16, 13, 21, [1, 2, 3, 5, 10, 20], (5, 0)),
    "f18y": (18, 12, 14, 21, [1, 2, 3, 5, 10, 20], (0, 5)),
}
GAMMA_REF = 1.66666667  # models/iosmaugparams.h.ot PGAMMA
TWICE = ("ot128",)      # run twice: the multi-block pad race makes runs differ

# 3D: name: ((nx, ny, nz), seed, NT, steps kept, runs); runs > 1 repeats the
# multi-block cases to expose order-dependent results
L3 = 0.1
G3 = -0.1
CASES3 = {
    "t3s": ((4, 4, 4), 21, 21, [1, 2, 3, 5, 10, 20], 1),
    "t3a": ((12, 12, 8), 22, 12, [0, 1, 2, 3, 4, 5, 10], 2),
    "t3b": ((20, 12, 8), 23, 5, [0, 1, 2, 3], 2),
    # fixed ghosts along dim 0: the flux-tube model's cuboundary leaves type 3
    # untouched at run time (models/boundary.cu.fluxtube1:1137-1277), which
    # is the engine's fixed type (5)
    "t3f": ((4, 4, 4), 24, 21, [1, 2, 3, 5, 10, 20], 1, (3, 4, 4), (5, 4, 4)),
}


# the reference built with -DUSE_DORDER3 (same tuple layouts as CASES / CASES3)
CASES_O6 = {"d16": (16, 16, 15, 21, [1, 2, 3, 5, 10, 20])}

# The user source term of the reference's spicule1 model
# (models/usersource.cu.spicule1:3-137, built with -DUSE_USERSOURCE into the
# Orszag-Tang build): m_1 += dt vvz (rho + rho_b) with
# vvz = 200 exp(-(z-xc1)^2/dz^2) exp(-(x-xc2)^2/dx^2), z = xmin_0 + i dx_0,
# x = xmin_1 + j dx_1 (ghosts included), xc1 = 0.0174 Mm, xc2 = 1.998046 Mm,
# dz = dx = 1 km, applied in the step whose counter p->it is 1 only.  The
# domain is placed around the driver's centre in metres with 1 km cells, so
# that the term reaches several cells: dim 0 [8, 26] km, dim 1
# [1990, 2008] km, 18 x 18 interior cells (one thread block: race-free).  The
# state is an Orszag-Tang pattern in solar units with a uniform background
# density and pressure (energyb) and positions equal to the source's own
# z and x, so that the engine's Gaussian driver with the same centre and
# width reproduces the term.
# fs18: the same with fixed (5) ghosts along dim 0 and the domain moved so
# that the driver's centre lies on ghost column 1: the reference's driver acts
# on every cell, and a fixed boundary keeps the ghost values it leaves.
# name: (nx, ny, seed, NT, steps kept, XMIN XMAX YMIN YMAX [m], boundary types)
DRV_DOMAIN = (8.0e3, 26.0e3, 1.99e6, 2.008e6)
CASES_DRV = {"s18": (18, 18, 31, 11, [1, 2, 3, 5, 10], DRV_DOMAIN, (0, 0)),
             "fs18": (18, 18, 33, 11, [1, 2, 3, 5, 10], (16.4e3, 34.4e3, 1.99e6, 2.008e6), (5, 0))}

# Fixed (5) ghosts together with gravity and background fields: the OT build
# with PGRAV0/1 set and nonzero energyb, rhob, b1b, b2b in the .ini.  The
# reference's 2D gravity and energy-coupling kernels also update the two low
# ghost layers (src/centdiff2.cu:587-787), which the fixed boundary keeps.
# name: (nx, ny, seed, NT, steps kept, boundary types, gravity)
CASES_FG = {"fg16": (16, 16, 41, 21, [1, 2, 3, 5, 10, 20], (5, 0), (0.2, -0.1)),
            "fg18y": (18, 12, 42, 21, [1, 2, 3, 5, 10, 20], (0, 5), (-0.1, 0.15))}


def ot_background_state(nx, ny, seed):
    """ot_state plus smooth nonzero background fields with the same total
    state (rho_b, e_b moved out of rho, e)."""
    w, pos = ot_state(nx, ny, seed)
    n1, n0 = w.shape[1:]
    jj, ii = np.meshgrid(np.arange(n1), np.arange(n0), indexing="ij")
    rb = 0.1 * (1 + 0.2 * np.sin(2 * math.pi * ii / n0))
    w[7] = rb
    w[0] = w[0] - rb
    w[8] = 0.05 * np.cos(2 * math.pi * jj / n1)
    w[9] = 0.025
    w[6] = 0.05 + 0.01 * np.cos(2 * math.pi * ii / n0)
    w[3] = w[3] - w[6]
    return w, pos
DRV_PARAMS = {"drv_amp": 200.0, "drv_period": 0.0, "drv_step": 1,
              "drv_x0": (0.0174 * 1.0e6, 1.998046 * 1.0e6), "drv_sigma": (0.001e6, 0.001e6)}


def spicule_state(nx, ny, seed, gamma=GAMMA_REF, domain=DRV_DOMAIN):
    """Orszag-Tang pattern in solar units on `domain`: total density
    2.7e-4 kg/m^3 (2e-4 of it background), flow 1 km/s, gas pressure 1.6e4 Pa
    (1.2e4 of it background, as energyb), field 82 (SAC units); positions
    xmin + i dx including ghosts, as the spicule1 source computes them."""
    x0, x1, y0, y1 = domain
    dx, dy = (x1 - x0) / nx, (y1 - y0) / ny
    X = x0 + np.arange(nx + 4) * dx
    Y = y0 + np.arange(ny + 4) * dy
    Xg, Yg = np.meshgrid(X, Y, indexing="xy")
    xs = 2 * math.pi * (Xg - (x0 - 1.5 * dx)) / (x1 - x0)
    ys = 2 * math.pi * (Yg - (y0 - 1.5 * dy)) / (y1 - y0)
    rng = np.random.default_rng(seed)
    rhob = 2.0e-4
    rho = 0.7e-4 * (1 + 1e-3 * rng.standard_normal(Xg.shape))
    rt = rho + rhob
    b0 = 82.0
    w = np.zeros((10,) + Xg.shape)
    w[0] = rho
    w[1] = -rt * 1.0e3 * np.sin(ys)
    w[2] = rt * 1.0e3 * np.sin(xs)
    w[4] = -b0 * np.sin(ys)
    w[5] = b0 * np.sin(2 * xs)
    w[3] = 0.4e4 / (gamma - 1) + 0.5 * (w[1] ** 2 + w[2] ** 2) / rt + 0.5 * (w[4] ** 2 + w[5] ** 2)
    w[6] = 1.2e4 / (gamma - 1)
    w[7] = rhob
    return w, np.stack([Xg, Yg]), (dx, dy)
CASES3_O6 = {"d3s": ((4, 4, 4), 25, 21, [1, 2, 3, 5, 10, 20], 1)}
O6 = ("USE_DORDER3",)


def tube_state(nx, ny, nz, seed, gamma=GAMMA_REF):
    """Smooth 3D state with nonzero backgrounds on [0, L3]^3: stratified-like
    rho_b, p_b along dim 0, a uniform-plus-sinusoid background field, and
    O(1e-2..1e-1) perturbations; positive pressure everywhere."""
    import smaug_b200.ic as I
    x, _ = I._axis(nx, 0, L3)
    y, _ = I._axis(ny, 0, L3)
    z, _ = I._axis(nz, 0, L3)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    k = 2 * math.pi / L3
    rng = np.random.default_rng(seed)
    w = np.zeros((13,) + X.shape)
    rhob = 1.0 + 0.2 * np.cos(k * X)
    pb = 1.0 + 0.1 * np.cos(k * X)
    bb = [0.3 + 0 * X, 0.05 * np.cos(k * Y), 0.02 * np.sin(k * Z)]
    rho = 0.01 * np.sin(k * X) * np.sin(k * Y) * np.cos(k * Z)
    rho = rho + 1e-3 * rhob * rng.standard_normal(X.shape)
    v = [0.1 * np.sin(k * Y), 0.1 * np.sin(k * Z), 0.1 * np.sin(k * X)]
    b = [0.05 * np.cos(k * Z), 0.05 * np.cos(k * X), 0.05 * np.cos(k * Y)]
    pp = 0.02 * (1.0 + 0.5 * np.sin(k * X + k * Y))
    rt = rho + rhob
    eb = pb / (gamma - 1) + 0.5 * sum(c * c for c in bb)
    et = (pb + pp) / (gamma - 1) + 0.5 * rt * sum(c * c for c in v) + \
        0.5 * sum((bb[d] + b[d]) ** 2 for d in range(3))
    w[0] = rho
    for d in range(3):
        w[1 + d] = rt * v[d]
        w[5 + d] = b[d]
        w[10 + d] = bb[d]
    w[4] = et - eb
    w[8] = eb
    w[9] = rhob
    return w, np.stack([X, Y, Z])


def _build3(name, nx, ny, nz, nt, bt_ref=None, defines=()):
    from oracle import build_ref
    extra = {}
    for d, t in enumerate(bt_ref or ()):
        extra["BCU%d" % d] = str(t)
        extra["BCL%d" % d] = str(t)
    return build_ref.build_ref(name, nx, ny, nt, nk=nz, verbose=False, defines=defines,
                               XMIN="0.0", XMAX=repr(L3), YMIN="0.0", YMAX=repr(L3),
                               ZMIN="0.0", ZMAX=repr(L3), PGRAV0=repr(G3), PGRAV1="0.0",
                               PGRAV2="0.0", **extra)


def _parse_args(argv):
    """command [case,case,...] [--runs DIR]"""
    global RUNS
    args = list(argv)
    if "--runs" in args:
        k = args.index("--runs")
        RUNS = os.path.abspath(args[k + 1])
        del args[k:k + 2]
    return args


ARGS = []


def _selected(table):
    want = ARGS[1].split(",") if len(ARGS) > 1 else None
    return {k: v for k, v in table.items() if want is None or k in want}


def ot_state(nx, ny, seed, noise=1e-3):
    import smaug_b200.ic as I
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
    w[3] = 5 / (12 * math.pi) / (2 / 3) + 0.5 * (w[1] ** 2 + w[2] ** 2) / rho + 0.5 * (w[4] ** 2 + w[5] ** 2)
    return w, np.stack([X, Y])


def prepare():
    from smaug_b200 import formats
    from oracle import build_ref
    os.makedirs(WORK, exist_ok=True)
    for table, defines in ((CASES, ()), (CASES_O6, O6)):
        for name, case in _selected(table).items():
            nx, ny, seed, nt, keep = case[:5]
            w, pos = ot_state(nx, ny, seed)
            formats.write_ini(os.path.join(WORK, name + ".ini"), w, pos)
            build_ref.build_ref(name, nx, ny, nt, verbose=False, defines=defines, **_bc_defines(case))
            print("prepared", name)
    for name, case in _selected(CASES_DRV).items():
        nx, ny, seed, nt, keep, dom, bt = case
        w, pos, _ = spicule_state(nx, ny, seed, domain=dom)
        formats.write_ini(os.path.join(WORK, name + ".ini"), w, pos)
        x0, x1, y0, y1 = dom
        build_ref.build_ref(name, nx, ny, nt, verbose=False, usersource="spicule1",
                            XMIN=repr(x0), XMAX=repr(x1), YMIN=repr(y0), YMAX=repr(y1),
                            **_bc_defines(case[:5] + (bt,)))
        print("prepared", name)
    for name, case in _selected(CASES_FG).items():
        nx, ny, seed, nt, keep, bt, g = case
        w, pos = ot_background_state(nx, ny, seed)
        formats.write_ini(os.path.join(WORK, name + ".ini"), w, pos)
        build_ref.build_ref(name, nx, ny, nt, verbose=False, PGRAV0=repr(g[0]), PGRAV1=repr(g[1]),
                            **_bc_defines(case[:5] + (bt,)))
        print("prepared", name)
    for table, defines in ((CASES3, ()), (CASES3_O6, O6)):
        for name, case in _selected(table).items():
            (nx, ny, nz), seed, nt, keep, runs = case[:5]
            w, pos = tube_state(nx, ny, nz, seed)
            formats.write_ini(os.path.join(WORK, name + ".ini"), w, pos, gamma=GAMMA_REF,
                              g=(G3, 0.0, 0.0))
            _build3(name, nx, ny, nz, nt, case[5] if len(case) > 5 else None, defines)
            print("prepared", name)


def _run_one(name, keep, tag=""):
    from oracle import run_ref
    binp = os.path.join(ROOT, "oracle", "_ref", name, "smaug")
    rundir = os.path.join("/tmp", "gold_" + name + tag)
    rc, times = run_ref.run(binp, os.path.join(WORK, name + ".ini"), rundir,
                            keep=set(keep) | {0})
    dest = os.path.join(RUNS, name + tag)
    os.makedirs(dest, exist_ok=True)
    os.system("cp -r %s/out %s/times.txt %s/stdout_tail.txt %s/" % (rundir, rundir, rundir, dest))
    print(name + tag, "rc", rc, "steps", len(times))
    if rc:
        sys.exit(rc)


def _bc_defines(case):
    if len(case) < 6:
        return {}
    out = {}
    for d, t in enumerate(case[5]):
        out["BCU%d" % d] = str(t)
        out["BCL%d" % d] = str(t)
    return out


def run():
    for name, case in _selected({**CASES, **CASES_O6, **CASES_DRV, **CASES_FG}).items():
        _run_one(name, case[4])
        if name in TWICE:
            _run_one(name, case[4], "_r1")
    for name, case in _selected({**CASES3, **CASES3_O6}).items():
        keep, runs = case[3], case[4]
        for r in range(runs):
            _run_one(name, keep, "" if r == 0 else "_r%d" % r)


def collect():
    from smaug_b200 import formats
    for name, case in _selected({**CASES3, **CASES3_O6}).items():
        (nx, ny, nz), seed, nt, keep, runs = case[:5]
        extra = {"bt": np.array(case[6]), "bt_ref": np.array(case[5])} if len(case) > 6 else {}
        if name in CASES3_O6:
            extra["order"] = 6
        w0, pos0, _ = formats.read_ini(os.path.join(WORK, name + ".ini"), 3)
        states, times = [], []
        for k in keep:
            w, pos, h = formats.read_out(os.path.join(RUNS, name, "out", "ref_%d.out" % k))
            states.append(w)
            times.append(h["t"])
        np.savez_compressed(os.path.join(HERE, name + ".npz"), w0=w0, pos=pos0,
                            steps=np.array(keep), states=np.array(states),
                            hdr_t=np.array(times), gamma=GAMMA_REF,
                            dx=np.array([L3 / nx, L3 / ny, L3 / nz]),
                            g=np.array([G3, 0.0, 0.0]), **extra)
        print("wrote", name)
    for name, case in _selected({**CASES_DRV, **CASES_FG}).items():
        nx, ny, seed, nt, keep = case[:5]
        w0, pos0, _ = formats.read_ini(os.path.join(WORK, name + ".ini"), 2)
        states, times = [], []
        for k in keep:
            w, pos, h = formats.read_out(os.path.join(RUNS, name, "out", "ref_%d.out" % k))
            states.append(w)
            times.append(h["t"])
        if name in CASES_DRV:
            dom, bt = case[5], case[6]
            _, _, dx = spicule_state(nx, ny, seed, domain=dom)
            extra = dict(drv_amp=DRV_PARAMS["drv_amp"], drv_step=DRV_PARAMS["drv_step"],
                         drv_x0=np.array(DRV_PARAMS["drv_x0"]),
                         drv_sigma=np.array(DRV_PARAMS["drv_sigma"]))
        else:
            bt, g = case[5], case[6]
            dx = (2 * math.pi / nx, 2 * math.pi / ny)
            extra = dict(g=np.array(g))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), w0=w0, pos=pos0,
                            steps=np.array(keep), states=np.array(states),
                            hdr_t=np.array(times), gamma=GAMMA_REF, dx=np.array(dx),
                            bt=np.array(bt), **extra)
        print("wrote", name)
    for name, case in _selected({**CASES, **CASES_O6}).items():
        nx, ny, seed, nt, keep = case[:5]
        bt = case[5] if len(case) > 5 else (0, 0)
        w0, pos0, _ = formats.read_ini(os.path.join(WORK, name + ".ini"), 2)
        states, times = [], []
        for k in keep:
            w, pos, h = formats.read_out(os.path.join(RUNS, name, "out", "ref_%d.out" % k))
            states.append(w[:6])
            times.append(h["t"])
        extra = {"order": 6} if name in CASES_O6 else {}
        # the last saved state of a second run of the same binary (name_r1)
        if os.path.isdir(os.path.join(RUNS, name + "_r1")):
            extra["last_r1"] = formats.read_out(
                os.path.join(RUNS, name + "_r1", "out", "ref_%d.out" % keep[-1]))[0][:6]
        np.savez_compressed(os.path.join(HERE, name + ".npz"), w0=w0[:6], pos=pos0,
                            steps=np.array(keep), states=np.array(states),
                            hdr_t=np.array(times), gamma=GAMMA_REF,
                            dx=np.array([2 * math.pi / nx, 2 * math.pi / ny]),
                            bt=np.array(bt), **extra)
        print("wrote", name)


if __name__ == "__main__":
    ARGS = _parse_args(sys.argv[1:])
    {"prepare": prepare, "run": run, "collect": collect}[ARGS[0]]()
