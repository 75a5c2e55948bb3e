"""Loading of the reference golden fixtures (tests/golden/*.npz)."""
import os

import numpy as np

from smaug_b200 import params as P

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
STRICT = ("g16", "g18x12", "ot64")     # full multi-step runs
BOUNDARY = ("f16x", "f18y")            # fixed ghosts along dim 0 / dim 1
ONESTEP = ("ot24x20",)                 # consecutive steps, one-step parity
RACE = ("ot128",)                      # 128^2, 200 steps, two runs of the reference
STRICT3 = ("t3s", "t3a", "t3b", "t3f")  # 3D flux-tube build, contcd4 (t3f: fixed dim 0) ghosts
ORDER6 = ("d16",)                      # 2D, the reference built with -DUSE_DORDER3
ORDER6_3D = ("d3s",)                   # 3D, the same
DRIVER = ("s18",)                      # 2D, the spicule1 model's user source term
# 2D fixed ghosts that the reference updates: gravity and background fields
# (fg16 fixed along dim 0, fg18y along dim 1), the driver (fs18)
FIXED_UPDATES = ("fg16", "fg18y", "fs18")


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    d = {k: z[k] for k in z.files}
    if d["w0"].ndim == 4 or d["w0"].shape[0] == 10:  # all fields (3D; 2D with backgrounds)
        d["w0full"] = d["w0"].copy()
        return d
    w0 = np.zeros((10,) + d["w0"].shape[1:])
    w0[:6] = d["w0"]
    d["w0full"] = w0
    return d


def params(d, **kw):
    kw.setdefault("integrator", P.INT_EULER)
    if "order" in d:
        kw.setdefault("stencil_order", int(d["order"]))
    if d["w0"].ndim == 4:
        nz, ny, nx = d["w0"].shape[1:]
        bt = [int(b) for b in d["bt"]] if "bt" in d else [P.BC_CONTCD4] * 3
        kw.setdefault("boundtype", bt)
        return P.make_params(ndim=3, n=(nx, ny, nz), dx=tuple(d["dx"]),
                             gamma=float(d["gamma"]), courant=0.3, dtmax=1.0, dt=1e-8,
                             g=tuple(d["g"]), **kw)
    ny, nx = d["w0"].shape[1:]
    if "drv_amp" in d:
        kw.setdefault("driver", P.DRIVER_GAUSS_STEP)
        kw.setdefault("drv_amp", float(d["drv_amp"]))
        kw.setdefault("drv_step", int(d["drv_step"]))
        kw.setdefault("drv_x0", tuple(float(v) for v in d["drv_x0"]))
        kw.setdefault("drv_sigma", tuple(float(v) for v in d["drv_sigma"]))
    if "bt" in d:
        kw.setdefault("boundtype", tuple(int(b) for b in d["bt"]))
    if "g" in d:
        kw.setdefault("g", tuple(float(v) for v in d["g"]))
    return P.make_params(ndim=2, n=(nx, ny, 1), dx=tuple(d["dx"]), gamma=float(d["gamma"]),
                         courant=0.3, dtmax=1.0, dt=1e-8, **kw)


def full(w6):
    w = np.zeros((10,) + w6.shape[1:])
    w[:6] = w6
    return w


def race_mask(d):
    """Cells outside the last interior column along dim 0 and its periodic
    image: the only cells the multi-block pad race of the reference reaches in
    one step."""
    n0 = d["w0"].shape[2]
    mask = np.ones(d["w0"].shape[1:], bool)
    mask[:, [1, n0 - 3]] = False
    return mask

