"""Run parameters: ctypes mirror of smaug_params_t (include/smaug_b200.h).

The fields mirror the reference's struct params (include/iotypes.h:85-175)
that the time advance reads, plus the integrator/precision switches of this
engine.  Field and derived-variable numbering follows include/iotypes.h:209-230.
"""
import ctypes
import math

PARAMS_VERSION = 1
MAXVAR = 13

BC_PERIODIC = 0
BC_CONT = 3
BC_CONTCD4 = 4
BC_FIXED = 5
BC_SYMM = 6
BC_ASYMM = 7

INT_EULER = 0
INT_RK4 = 1

PREC_FP64 = 0
PREC_MIXED = 1

PAD_STRAY = 0
PAD_ZERO = 1

DRIVER_NONE = 0
DRIVER_GAUSS = 1
DRIVER_GAUSS_STEP = 2  # the same term in the step whose counter equals drv_step only


class SmaugParams(ctypes.Structure):
    _fields_ = [
        ("version", ctypes.c_int32),
        ("ndim", ctypes.c_int32),
        ("n", ctypes.c_int32 * 3),
        ("moddton", ctypes.c_int32),
        ("hyperdifmom", ctypes.c_int32),
        ("integrator", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("pad_model", ctypes.c_int32),
        ("boundtype", (ctypes.c_int32 * 2) * 3),
        ("driver", ctypes.c_int32),
        ("stencil_order", ctypes.c_int32),
        ("drv_step", ctypes.c_int32),
        ("reserved_i", ctypes.c_int32 * 5),
        ("dx", ctypes.c_double * 3),
        ("dt", ctypes.c_double),
        ("dtmax", ctypes.c_double),
        ("courant", ctypes.c_double),
        ("gamma", ctypes.c_double),
        ("eta", ctypes.c_double),
        ("g", ctypes.c_double * 3),
        ("chyp", ctypes.c_double * MAXVAR),
        ("xmin", ctypes.c_double * 3),
        ("drv_amp", ctypes.c_double),
        ("drv_period", ctypes.c_double),
        ("drv_x0", ctypes.c_double * 3),
        ("drv_sigma", ctypes.c_double * 3),
        ("reserved_d", ctypes.c_double * 8),
    ]

    # ---- convenience -------------------------------------------------
    @property
    def nvar(self):
        return 4 + 3 * self.ndim

    @property
    def ncells(self):
        n = 1
        for d in range(self.ndim):
            n *= self.n[d]
        return n

    @property
    def shape(self):
        """numpy shape of one field, slowest first: (n2, n1, n0) or (n1, n0)."""
        return tuple(self.n[d] for d in reversed(range(self.ndim)))

    def interior_cells(self):
        c = 1
        for d in range(self.ndim):
            c *= self.n[d] - 4
        return c


def field_ids(ndim):
    """Field indices of include/iotypes.h:209-216 for NDIM=ndim."""
    ids = {"rho": 0, "energy": 1 + ndim, "energyb": 2 + 2 * ndim, "rhob": 3 + 2 * ndim}
    for d in range(ndim):
        ids["mom%d" % (d + 1)] = 1 + d
        ids["b%d" % (d + 1)] = 2 + ndim + d
        ids["b%db" % (d + 1)] = 4 + 2 * ndim + d
    return ids


def field_names(ndim):
    ids = field_ids(ndim)
    names = [None] * (4 + 3 * ndim)
    for k, v in ids.items():
        names[v] = k
    return names


def evolved_fields(ndim):
    """rho .. b_last: the fields the time advance updates."""
    return list(range(0, 2 + 2 * ndim))


def make_params(ndim=2, n=(132, 132, 1), dx=None, gamma=5.0 / 3.0, courant=0.3,
                dtmax=1.0, dt=1.0e-8, moddton=1, hyperdifmom=1, chyp=0.2,
                boundtype=None, integrator=INT_EULER, g=(0.0, 0.0, 0.0),
                eta=0.0, xmin=(0.0, 0.0, 0.0), pad_model=PAD_STRAY,
                driver=DRIVER_NONE, drv_amp=0.0, drv_period=0.0, precision=PREC_FP64,
                drv_x0=(0.0, 0.0, 0.0), drv_sigma=(0.0, 0.0, 0.0), stencil_order=4,
                drv_step=0):
    """Build a parameter block.  Defaults: the reference's Orszag-Tang model
    (models/iosmaugparams.h.ot) with a 0.3 Courant number; `chyp` may be a
    scalar (every field) or a sequence indexed by field; stencil_order 6
    selects the 6th-order flux derivative of the reference's USE_DORDER3
    build."""
    p = SmaugParams()
    p.version = PARAMS_VERSION
    p.ndim = ndim
    nn = list(n) + [1] * (3 - len(n))
    if ndim == 2:
        nn[2] = 1
    for d in range(3):
        p.n[d] = nn[d]
    if dx is None:
        dx = [2.0 * math.pi / (nn[d] - 4) if d < ndim else 0.0 for d in range(3)]
    for d in range(3):
        p.dx[d] = dx[d] if d < len(dx) else 0.0
        p.g[d] = g[d] if d < len(g) else 0.0
        p.xmin[d] = xmin[d] if d < len(xmin) else 0.0
        p.drv_x0[d] = drv_x0[d] if d < len(drv_x0) else 0.0
        p.drv_sigma[d] = drv_sigma[d] if d < len(drv_sigma) else 0.0
    p.gamma = gamma
    p.eta = eta
    p.courant = courant
    p.dtmax = dtmax
    p.dt = dt
    p.moddton = moddton
    p.hyperdifmom = hyperdifmom
    p.integrator = integrator
    p.precision = precision
    p.pad_model = pad_model
    if isinstance(chyp, (int, float)):
        for f in range(MAXVAR):
            p.chyp[f] = float(chyp)
    else:
        for f in range(MAXVAR):
            p.chyp[f] = float(chyp[f]) if f < len(chyp) else 0.0
    for d in range(3):
        bt = BC_PERIODIC if boundtype is None else boundtype[d] if d < len(boundtype) else 0
        if isinstance(bt, (tuple, list)):
            p.boundtype[d][0], p.boundtype[d][1] = bt
        else:
            p.boundtype[d][0] = p.boundtype[d][1] = bt
    p.driver = driver
    p.stencil_order = stencil_order
    p.drv_amp = drv_amp
    p.drv_period = drv_period
    p.drv_step = drv_step
    return p
