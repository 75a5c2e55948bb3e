"""Recipe: build the reference SMAUG GPU binary from its own sources.

TEST INFRASTRUCTURE.  The reference (mikeg64/smaug) has no CPU solver: every
solver routine is a CUDA kernel.  To pin the CPU oracle against the real
reference, this script compiles the reference's unmodified solver sources for
sm_100a and the result runs on the B200 box as a checker.  Nothing of the
reference enters the repository: sources are copied to a scratch directory
under /tmp, the build output goes to oracle/_ref/<name>/ (git-ignored).

The reference's build selects a model by copying models/*.<model> over the
compile-time parameter header and instantiates the shared device helpers by
`sed s/MODID/<id>/` (src/Makefile:79-227); this recipe does the same for the
Orszag-Tang model (`make ot`, 2D) or the flux-tube model (`make fluxtube1`,
3D with -DUSE_SAC_3D)
with the run parameters substituted into include/iosmaugparams.h.  Three workarounds are needed with CUDA 12.9 / GCC 13:
  1. src/init.cu:169 passes an undeclared `w`; it is built with `wmod`
     (the only array in scope; the call is inside `if(p->readini==0)`,
     not taken when an .ini is read).
  2. the library list of src/Makefile:152 precedes the objects; linking is
     done here with nvcc and the objects first.
  3. most cu* wrappers return int but fall off the end without a return
     (e.g. src/computedervfields.cu:1800-1830); GCC 13 compiles that to a
     trap instruction at -O0 (nvcc's host pass), so host code is built with
     -fno-unreachable-traps, which restores a plain return.
Usage:  python oracle/build_ref.py NAME NI NJ NT [key=value ...]
"""
import glob
import os
import re
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference checkout (its smaug/ project directory); SMAUG_REFERENCE overrides
REFROOT = os.environ.get("SMAUG_REFERENCE", "/root/reference/smaug")
OUT = os.path.join(HERE, "_ref")

# sed instantiation table of src/Makefile:163-227: object -> [(template, id)]
MODIDS = {
    "nushk1.cu": [("gradops.cu", "nshk")],
    "hyperdifvisc1.cu": [("gradops.cu", "hdv1")],
    "hyperdifvisc1l.cu": [("gradops.cu", "hdv1l")],
    "hyperdifvisc1r.cu": [("gradops.cu", "hdv1r")],
    "hyperdifrhosource1.cu": [("gradops.cu", "hdr1")],
    "hyperdifesource1.cu": [("gradops.cu", "hde1")],
    "hyperdifbsource1.cu": [("gradops.cu", "hdb1")],
    "hyperdifbsourcene1.cu": [("gradops.cu", "hdbne1")],
    "hyperdifmomsource1.cu": [("gradops.cu", "hdm1")],
    "hyperdifmomsourcene1.cu": [("gradops.cu", "hdmne1")],
    "centdiff1.cu": [("gradops.cu", "cd1"), ("dervfields.cu", "cd1"), ("usersource.cu", "cd1")],
    "centdiff2.cu": [("gradops.cu", "cd2"), ("dervfields.cu", "cd2"), ("usersource.cu", "cd2")],
    "computedervfields.cu": [("gradops.cu", "cdf"), ("dervfields.cu", "cdf")],
    "boundary.cu": [("gradops.cu", "b")],
    "init.cu": [("gradops.cu", "i"), ("init_user.cu", "i")],
    "update.cu": [("gradops.cu", "u")],
    "advance.cu": [("gradops.cu", "adv"), ("dervfields.cu", "adv")],
    "divb.cu": [("gradops.cu", "db"), ("dervfields.cu", "db")],
}
CFILES = ["iosmaug.c", "initialisation.c", "dxroutines.c", "readwrite.c"]
# the flux-tube parameter header (Meta *metad) pairs with the C driver, whose
# USE_SAC_3D branches allocate the z positions with nj entries (src/iosmaug.c:65-68),
# so 3D builds need nk <= nj
CFILES_3D = ["iosmaug.c", "initialisation.c", "dxroutines.c", "readwrite.c"]

DEFAULTS = {
    "XMIN": "0.0", "XMAX": "6.283185307179586", "YMIN": "0.0", "YMAX": "6.283185307179586",
    "DT": "1.0", "PCOURANT": "0.3", "PMODDTON": "1.0", "PCFGSAVEFREQUENCY": "1",
    "PGAMMA": "1.66666667", "CHYP": "0.2", "CFGFILE": '"ref.ini"', "CFGOUT": '"out/ref"',
}


def _set_define(text, name, value):
    pat = re.compile(r"^#define\s+%s\s+.*$" % name, re.M)
    if not pat.search(text):
        raise RuntimeError("define %s not found" % name)
    return pat.sub("#define %s %s" % (name, value), text)


def _configure(tmp, ni, nj, nt, nk, cfg, usersource=None):
    """Copy the reference tree to tmp and select the model and run parameters
    as `make ot` / `make fluxtube1` does; returns (src, inc).  `usersource`
    names a model whose user source term (models/usersource.cu.<model>)
    replaces src/usersource.cu (built with -DUSE_USERSOURCE)."""
    three = nk is not None
    for d in ("src", "include", "models"):
        shutil.copytree(os.path.join(REFROOT, d), os.path.join(tmp, d))
    subprocess.check_call(["chmod", "-R", "u+w", tmp])
    src, inc, mod = (os.path.join(tmp, d) for d in ("src", "include", "models"))
    model = "fluxtube1" if three else "ot"
    # make ot / make fluxtube1 (src/Makefile:32-101)
    shutil.copy(os.path.join(mod, "iosmaugparams.h." + model), os.path.join(inc, "iosmaugparams.h"))
    shutil.copy(os.path.join(mod, "init_user.cu." + model), os.path.join(src, "init_user.cu"))
    shutil.copy(os.path.join(mod, "boundary.cu." + model), os.path.join(src, "boundary.cu"))
    if three:
        shutil.copy(os.path.join(mod, "usersource.cu." + model), os.path.join(src, "usersource.cu"))
        shutil.copy(os.path.join(mod, "initialisation_user.h.default"),
                    os.path.join(inc, "initialisation_user.h"))
    if usersource:
        shutil.copy(os.path.join(mod, "usersource.cu." + usersource), os.path.join(src, "usersource.cu"))
    ph = os.path.join(inc, "iosmaugparams.h")
    text = open(ph).read()
    text = _set_define(text, "NI", str(ni))
    text = _set_define(text, "NJ", str(nj))
    text = _set_define(text, "NT", str(nt))
    keys = ["XMIN", "XMAX", "YMIN", "YMAX", "DT", "PCOURANT", "PMODDTON",
            "PCFGSAVEFREQUENCY", "PGAMMA", "CFGFILE", "CFGOUT"]
    if three:
        text = _set_define(text, "NK", str(nk))
        keys += ["ZMIN", "ZMAX", "PGRAV0", "PGRAV1", "PGRAV2"]
    for k in keys:
        text = _set_define(text, k, cfg[k])
    # boundary types per dimension (BCU*: upper, BCL*: lower), when given
    for k in ("BCU0", "BCL0", "BCU1", "BCL1") + (("BCU2", "BCL2") if three else ()):
        if k in cfg:
            text = _set_define(text, k, cfg[k])
    if not three:  # 2D gravity, when given (models/iosmaugparams.h.ot:17-19)
        for k in ("PGRAV0", "PGRAV1"):
            if k in cfg:
                text = _set_define(text, k, cfg[k])
    for k in ("PCHYP", "PCHYPRHO", "PCHYPENERGY", "PCHYPB0", "PCHYPB1", "PCHYPB2",
              "PCHYPMOM0", "PCHYPMOM1", "PCHYPMOM2"):
        text = _set_define(text, k, cfg.get(k, cfg["CHYP"]))
    open(ph, "w").write(text)
    return src, inc


def _driver_objects(src, three, verbose, defines=()):
    """The reference's host driver (g++, as src/make_inputs:3 selects)."""
    sac = "-DUSE_SAC_3D" if three else "-DUSE_SAC"
    objs = []
    for c in (CFILES_3D if three else CFILES):
        o = os.path.join(src, c.rsplit(".", 1)[0] + ".o")
        cmd = ["g++", "-O0", "-fno-unreachable-traps", sac, "-DD1D", "-w", "-fpermissive"] + \
            ["-D" + d for d in defines] + ["-o", o, "-c", os.path.join(src, c)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd, cwd=src)
        objs.append(o)
    return objs


def _cached(name, stamp):
    dest = os.path.join(OUT, name)
    os.makedirs(dest, exist_ok=True)
    binp = os.path.join(dest, "smaug")
    stampf = os.path.join(dest, "build.txt")
    fresh = os.path.exists(binp) and os.path.exists(stampf) and open(stampf).read() == stamp
    return binp, stampf, fresh


def build_ref(name, ni, nj, nt, arch="sm_100a", verbose=True, nk=None, defines=(), usersource=None,
              **kw):
    """Build the reference's GPU binary for an ni x nj (x nk) grid and nt
    steps; `defines` are extra build macros of the reference (e.g.
    USE_DORDER3, the 6th-order flux derivative), `usersource` a model whose
    user source term is compiled in (models/usersource.cu.<model>, with
    -DUSE_USERSOURCE), kw override iosmaugparams.h."""
    if usersource:
        defines = tuple(defines) + ("USE_USERSOURCE",)
    if not os.path.isdir(REFROOT):
        raise RuntimeError("reference sources not present at %s" % REFROOT)
    cfg = dict(DEFAULTS)
    cfg.update({k.upper(): str(v) for k, v in kw.items()})
    three = nk is not None
    if three and nk > nj:
        raise ValueError("3D reference builds need nk <= nj")
    stamp = "ni=%d nj=%d nk=%s nt=%d %s arch=%s%s%s\n" % (
        ni, nj, nk, nt, sorted(cfg.items()), arch, "".join(" -D" + d for d in defines),
        " usersource=%s" % usersource if usersource else "")
    binp, stampf, fresh = _cached(name, stamp)
    if fresh:
        return binp
    tmp = tempfile.mkdtemp(prefix="smaug_ref_")
    try:
        src, inc = _configure(tmp, ni, nj, nt, nk, cfg, usersource)
        # workaround 1 (see module docstring)
        initcu = os.path.join(src, "init.cu")
        lines = open(initcu).read().split("\n")
        if "init_user_i(w,p,ii)" not in lines[168]:
            raise RuntimeError("unexpected src/init.cu:169: %r" % lines[168])
        lines[168] = lines[168].replace("init_user_i(w,p,ii)", "init_user_i(wmod,p,ii)")
        open(initcu, "w").write("\n".join(lines))
        # MODID instantiation
        for cu, pairs in MODIDS.items():
            for tpl, mid in pairs:
                t = open(os.path.join(src, tpl)).read().replace("MODID", mid)
                base = tpl[:-3]
                open(os.path.join(inc, "%s_%s.cuh" % (base, mid)), "w").write(t)
        objs = []
        sac = "-DUSE_SAC_3D" if three else "-DUSE_SAC"
        for cu in MODIDS:
            o = os.path.join(src, cu[:-3] + ".o")
            cmd = ["nvcc", "-arch=" + arch, "-maxrregcount=32", sac, "-w",
                   "-Xcompiler", "-fno-unreachable-traps"] + ["-D" + d for d in defines] + \
                  ["-o", o, "-c", os.path.join(src, cu)]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.check_call(cmd, cwd=src)
            objs.append(o)
        objs += _driver_objects(src, three, verbose, defines)
        cmd = ["nvcc", "-arch=" + arch, "-o", binp] + objs + ["-lcudart", "-lm"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd, cwd=src)
        with open(stampf, "w") as f:
            f.write(stamp)
        return binp
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def build_compat(name, ni, nj, nt, verbose=True, nk=None, **kw):
    """The reference's unchanged host driver (src/iosmaug.c, readwrite.c,
    initialisation.c, dxroutines.c) linked against this project's wrapper
    shim smaug_b200/libsmaug_compat{2d,3d}.so instead of the reference's .cu
    objects.  Same parameters as build_ref; the binary finds the shim through
    an rpath relative to its own location (oracle/_ref/<name>/smaug)."""
    if not os.path.isdir(REFROOT):
        raise RuntimeError("reference sources not present at %s" % REFROOT)
    cfg = dict(DEFAULTS)
    cfg.update({k.upper(): str(v) for k, v in kw.items()})
    three = nk is not None
    if three and nk > nj:
        raise ValueError("3D reference builds need nk <= nj")
    pkg = os.path.join(os.path.dirname(HERE), "smaug_b200")
    shim = os.path.join(pkg, "libsmaug_compat%s.so" % ("3d" if three else "2d"))
    if not os.path.exists(shim):
        raise RuntimeError("build the package first (smaug_b200/build.py): %s missing" % shim)
    stamp = "compat ni=%d nj=%d nk=%s nt=%d %s shim=%s\n" % (ni, nj, nk, nt, sorted(cfg.items()),
                                                          os.path.getmtime(shim))
    binp, stampf, fresh = _cached(name, stamp)
    if fresh:
        return binp
    tmp = tempfile.mkdtemp(prefix="smaug_compat_")
    try:
        src, inc = _configure(tmp, ni, nj, nt, nk, cfg)
        objs = _driver_objects(src, three, verbose)
        cmd = ["g++", "-o", binp] + objs + [
            "-L", pkg, "-lsmaug_compat%s" % ("3d" if three else "2d"), "-lsmaug_b200",
            "-Wl,-rpath,$ORIGIN/../../../smaug_b200", "-lm"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd, cwd=src)
        with open(stampf, "w") as f:
            f.write(stamp)
        return binp
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


# Binaries used by tests/golden/make_golden.py (single-block grids, every
# step saved) and by bench.py's reference-GPU timing line (1024^2, no
# per-step output).
STANDARD = [
    ("g16", 16, 16, 21, {}),
    ("g18x12", 18, 12, 21, {}),
    ("ot1024t", 1024, 1024, 12, {"PCFGSAVEFREQUENCY": "100000"}),
]


_T3 = {"XMIN": "0.0", "XMAX": "0.1", "YMIN": "0.0", "YMAX": "0.1", "ZMIN": "0.0",
       "ZMAX": "0.1", "PGRAV0": "-0.1", "PGRAV1": "0.0", "PGRAV2": "0.0"}
# The same driver builds linked against the wrapper shim (tests/test_compat.py
# runs them on the golden fixtures' inputs; the 1024^2 one times the unchanged
# driver on the engine beside ot1024t).
COMPAT_STANDARD = [
    ("compat_g16", 16, 16, 21, None, {}),
    ("compat_g18x12", 18, 12, 21, None, {}),
    ("compat_t3s", 4, 4, 21, 4, _T3),
    ("compat_ot1024t", 1024, 1024, 12, None, {"PCFGSAVEFREQUENCY": "100000"}),
]


def build_standard(verbose=False):
    out = {}
    for name, ni, nj, nt, kw in STANDARD:
        out[name] = build_ref(name, ni, nj, nt, verbose=verbose, **kw)
    for name, ni, nj, nt, nk, kw in COMPAT_STANDARD:
        out[name] = build_compat(name, ni, nj, nt, verbose=verbose, nk=nk, **kw)
    return out


if __name__ == "__main__":
    a = sys.argv[1:]
    if len(a) < 4:
        print(__doc__)
        sys.exit(2)
    kw = dict(x.split("=", 1) for x in a[4:])
    print(build_ref(a[0], int(a[1]), int(a[2]), int(a[3]), **kw))
