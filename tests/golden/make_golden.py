"""Generate the golden fixtures of tests/golden/ from the reference itself.

The reference (mikeg64/smaug) has no tests and ships no golden outputs, so
these fixtures are produced by running the reference's own GPU binary (built
from its sources by oracle/build_ref.py) on a B200, on inputs written here:

  python tests/golden/make_golden.py prepare   # here: .ini inputs + reference builds
  python tests/golden/make_golden.py run       # on the GPU box: run the binaries
  python tests/golden/make_golden.py collect   # here: .out files -> *.npz fixtures

Cases (Orszag-Tang on [0,2pi]^2, seeded 1e-3 rho noise, the reference OT
model parameters with PGAMMA 1.66666667, courant 0.3, DT 1, moddton on):
  g16      16x16 interior, 20 steps   -- one thread block: race-free
  g18x12   18x12 interior, 20 steps   -- one thread block: race-free
  ot64     64x64 interior, 11 steps   -- multi-block (17 thread blocks)
  ot24x20  24x20 interior, steps 0-5  -- multi-block, consecutive steps for
           one-step parity away from the column the pad race can touch
The reference launches one thread per cell in 512-thread blocks; its
hyperdifvisc1r_parallel stores tmp6 through the wrong index (encode3) into
the padded array while the same launch zeroes it.  Inside one block the
stray store lands last; across blocks the order is not fixed, which can
change nu_r in the last interior column along dim 0.
Each .npz holds the evolved fields (rho m1 m2 e b1 b2, ghosts included) of
the initial state and of the saved steps, the positions, and the header
times of the reference's .out files.
"""
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

WORK = os.path.join(HERE, "_inputs")          # git-ignored; travels to the GPU box
RUNS = os.path.join(ROOT, "gpurun_out", "gold")

# name: (nx, ny, seed, NT, steps kept)
CASES = {
    "g16": (16, 16, 11, 21, [1, 2, 3, 5, 10, 20]),
    "g18x12": (18, 12, 12, 21, [1, 2, 3, 5, 10, 20]),
    "ot64": (64, 64, 1, 12, [1, 11]),
    "ot24x20": (24, 20, 5, 12, [0, 1, 2, 3, 4, 5]),
}
GAMMA_REF = 1.66666667  # models/iosmaugparams.h.ot PGAMMA


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
    for name, (nx, ny, seed, nt, keep) in CASES.items():
        w, pos = ot_state(nx, ny, seed)
        formats.write_ini(os.path.join(WORK, name + ".ini"), w, pos)
        build_ref.build_ref(name, nx, ny, nt, verbose=False)
        print("prepared", name)


def run():
    from oracle import run_ref
    for name, (nx, ny, seed, nt, keep) in CASES.items():
        binp = os.path.join(ROOT, "oracle", "_ref", name, "smaug")
        rundir = os.path.join("/tmp", "gold_" + name)
        rc, times = run_ref.run(binp, os.path.join(WORK, name + ".ini"), rundir, keep=set(keep) | {0})
        dest = os.path.join(RUNS, name)
        os.makedirs(dest, exist_ok=True)
        os.system("cp -r %s/out %s/times.txt %s/" % (rundir, rundir, dest))
        print(name, "rc", rc, "steps", len(times))
        if rc:
            sys.exit(rc)


def collect():
    from smaug_b200 import formats
    for name, (nx, ny, seed, nt, keep) in CASES.items():
        w0, pos0, _ = formats.read_ini(os.path.join(WORK, name + ".ini"), 2)
        states, times = [], []
        for k in keep:
            w, pos, h = formats.read_out(os.path.join(RUNS, name, "out", "ref_%d.out" % k))
            states.append(w[:6])
            times.append(h["t"])
        np.savez_compressed(os.path.join(HERE, name + ".npz"), w0=w0[:6], pos=pos0,
                            steps=np.array(keep), states=np.array(states),
                            hdr_t=np.array(times), gamma=GAMMA_REF,
                            dx=np.array([2 * math.pi / nx, 2 * math.pi / ny]))
        print("wrote", name)


if __name__ == "__main__":
    {"prepare": prepare, "run": run, "collect": collect}[sys.argv[1]]()
