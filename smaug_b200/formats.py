"""Reference file formats: ASCII VAC .ini input and binary .out output.

.ini  (src/readwrite.c:975-1082 reader, :1084-1316 writer)
  line 1  run name
  line 2  "it t ndim neqpar nw"
  line 3  grid sizes n0 n1 [n2] (ghosts included)
  line 4  equation parameters gamma eta g1 g2 [g3] 0 0
  line 5  variable names
  then one line per cell, x fastest: pos[ndim] w[nvar]
The reference writer prints with %lG (6 digits); `write_ini` defaults to full
round-trip precision so both engines read bit-identical inputs.

.out  (src/readwrite.c:160-366; read layout of python/smaug-read2.py:24-61)
  char[79] name | int32 it | float64 t | int32 ndim, neqpar, nw |
  int32 n[ndim] | float64 eqpar[neqpar] | char[79] varnames |
  (ndim+nvar) fields of n0*n1[*n2] float64, x fastest: pos[ndim] then w | '\\n'
"""
import struct

import numpy as np

VARNAMES_2D = "x y rho mx my e bx by  gamma eta g1 g2"
VARNAMES_3D = "x y z rho mx my mz e bx by bz gamma eta g1 g2 g3"


def write_ini(path, w, pos, gamma=5.0 / 3.0, eta=0.0, g=(0.0, 0.0, 0.0), it=0, t=0.0,
              name="smaug_b200", fmt="%.17E"):
    """Write a reference ASCII .ini. w: (nvar, [n2,] n1, n0); pos: (ndim, ...)."""
    ndim = pos.shape[0]
    nvar = w.shape[0]
    shape = w.shape[1:]
    n = list(reversed(shape))
    cols = np.concatenate([pos.reshape(ndim, -1), w.reshape(nvar, -1)], axis=0).T
    with open(path, "w") as f:
        f.write("%s\n" % name)
        f.write("%d %g %d %d %d\n" % (it, t, ndim, 6 if ndim == 2 else 7, nvar))
        f.write(" ".join("%d" % v for v in n) + "\n")
        gg = " ".join("%.17g" % g[d] for d in range(ndim))
        f.write("%.17g %.17g %s 0 0\n" % (gamma, eta, gg))
        f.write((VARNAMES_2D if ndim == 2 else VARNAMES_3D) + "\n")
        np.savetxt(f, cols, fmt=fmt, delimiter=" ")


def read_ini(path, ndim, n=None):
    """Read a reference .ini; returns (w, pos, header dict).  `n` (n0, n1[, n2])
    defaults to the grid line of the file (the reference takes it from its
    compile-time NI/NJ instead)."""
    with open(path) as f:
        name = f.readline().rstrip("\n")
        l2 = f.readline().split()
        it, t = int(l2[0]), float(l2[1])
        nfile = [int(v) for v in f.readline().split()]
        eq = [float(v) for v in f.readline().split()]
        names = f.readline().rstrip("\n")
        data = np.loadtxt(f, dtype=np.float64)
    if n is None:
        n = nfile
    n = list(n)[:ndim]
    ncell = int(np.prod(n))
    nvar = 4 + 3 * ndim
    if data.ndim == 1:
        data = data[None, :]
    if data.shape[0] < ncell or data.shape[1] != ndim + nvar:
        raise ValueError("ini %s: expected %d rows x %d cols, got %s"
                         % (path, ncell, ndim + nvar, data.shape))
    data = data[:ncell]
    shape = tuple(reversed(n))
    pos = np.ascontiguousarray(data[:, :ndim].T).reshape((ndim,) + shape)
    w = np.ascontiguousarray(data[:, ndim:].T).reshape((nvar,) + shape)
    hdr = {"name": name, "it": it, "t": t, "n": nfile, "eqpar": eq, "varnames": names}
    return w, pos, hdr


def read_out(path):
    """Read a reference binary .out; returns (w, pos, header dict)."""
    with open(path, "rb") as f:
        buf = f.read()
    o = 0
    name = buf[o:o + 79].split(b"\0")[0].decode("latin-1").rstrip()
    o += 79
    it, = struct.unpack_from("<i", buf, o); o += 4
    t, = struct.unpack_from("<d", buf, o); o += 8
    ndim, neqpar, nw = struct.unpack_from("<3i", buf, o); o += 12
    n = list(struct.unpack_from("<%di" % ndim, buf, o)); o += 4 * ndim
    eq = list(struct.unpack_from("<%dd" % neqpar, buf, o)); o += 8 * neqpar
    varnames = buf[o:o + 79]
    o += 79
    ncell = int(np.prod(n))
    nf = ndim + nw
    arr = np.frombuffer(buf, dtype="<f8", count=nf * ncell, offset=o)
    shape = tuple(reversed(n))
    arr = arr.reshape((nf,) + shape)
    pos = arr[:ndim].copy()
    w = arr[ndim:].copy()
    hdr = {"name": name, "it": it, "t": t, "ndim": ndim, "neqpar": neqpar, "nw": nw,
           "n": n, "eqpar": eq, "varnames": varnames,
           "trailer": buf[o + 8 * nf * ncell:]}
    return w, pos, hdr


def write_out(path, w, pos, gamma, eta=0.0, g=(0.0, 0.0, 0.0), it=0, t=0.0,
              name="test1"):
    """Write a reference binary .out (python mirror of smaug_write_out_host)."""
    ndim = pos.shape[0]
    nw = w.shape[0]
    n = list(reversed(w.shape[1:]))
    with open(path, "wb") as f:
        f.write(name.encode("latin-1")[:79].ljust(79, b"\0"))
        f.write(struct.pack("<i", it))
        f.write(struct.pack("<d", t))
        f.write(struct.pack("<3i", ndim, 6 if ndim == 2 else 7, nw))
        f.write(struct.pack("<%di" % ndim, *n))
        if ndim == 2:
            f.write(struct.pack("<6d", gamma, eta, g[0], g[1], 0.0, 0.0))
        else:
            f.write(struct.pack("<7d", gamma, eta, g[0], g[1], g[2], 0.0, 0.0))
        vn = (VARNAMES_2D if ndim == 2 else VARNAMES_3D).encode()
        f.write(vn[:79].ljust(79, b"\0"))
        f.write(np.ascontiguousarray(pos, dtype="<f8").tobytes())
        f.write(np.ascontiguousarray(w, dtype="<f8").tobytes())
        f.write(b"\n")
