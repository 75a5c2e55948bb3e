"""The reference-wrapper shim (libsmaug_compat2d/3d.so, include/smaug_compat.h).

CPU: every wrapper the header declares is exported under the C++-mangled
name the reference's driver references; the shim's struct params/state have
the layout of the reference's include/iotypes.h (when the reference sources
are present); the unchanged reference driver links against the shim.
GPU: that driver, run on the golden fixtures' inputs, writes .out files equal
to the reference binary's (the fixtures) at 1e-12.
"""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from golden_util import load

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(ROOT, "include", "smaug_compat.h")
PKG = os.path.join(ROOT, "smaug_b200")
from oracle.build_ref import REFROOT  # noqa: E402  (SMAUG_REFERENCE overrides)

REFINC = os.path.join(REFROOT, "include")
MACROS = {"2d": "-DUSE_SAC", "3d": "-DUSE_SAC_3D"}


def declared_wrappers():
    src = open(HDR).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"//[^\n]*", "", src)
    return sorted(set(re.findall(r"^int\s+(cu[a-z0-9]+|initgrid)\s*\(", src, flags=re.M)))


def _defined(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True,
                         check=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if ln.strip()}


def _mangled_by_header(tmp, macro):
    """Mangled names g++ gives the header's declarations (the names a driver
    compiled by g++ against matching declarations references)."""
    names = declared_wrappers()
    src = os.path.join(tmp, "probe.cpp")
    with open(src, "w") as f:
        f.write('#include "smaug_compat.h"\n')
        f.write("void* probe_table[] = {%s};\n" % ", ".join("(void*)&%s" % n for n in names))
    obj = os.path.join(tmp, "probe.o")
    subprocess.check_call(["g++", "-c", macro, "-I", os.path.join(ROOT, "include"), src, "-o", obj])
    out = subprocess.run(["nm", "-u", obj], capture_output=True, text=True, check=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if ln.strip().startswith("U _Z")}


def test_header_declares_the_driver_wrappers():
    w = declared_wrappers()
    for s in ("cuinit", "initgrid", "cuboundary", "cucomputedervfields", "cucomputec",
              "cucomputemaxc", "cucentdiff1", "cucentdiff2", "cusource", "cuupdate", "cusync",
              "cuhyperdifvisc1r", "cuhyperdifbsourcene1"):
        assert s in w
    assert len(w) == 37


@pytest.mark.parametrize("nd", ["2d", "3d"])
def test_shim_exports_mangled_wrappers(engine_lib, nd):
    lib = os.path.join(PKG, "libsmaug_compat%s.so" % nd)
    assert os.path.exists(lib)
    have = _defined(lib)
    with tempfile.TemporaryDirectory() as tmp:
        want = _mangled_by_header(tmp, MACROS[nd])
    assert len(want) == len(declared_wrappers())
    assert not (want - have), sorted(want - have)
    # one known name, as nvcc mangles the reference's own definition
    assert "_Z11cucentdiff1PP6paramsS1_PP5statePPdS6_S6_S6_iidii" in have
    assert "smaug_compat_set_driver" in have and "smaug_compat_handle" in have


PARAM_FIELDS = ("n ng npgp fullgridini hdmean hdmax pmax pmin pmean emax emin emean xmax xmin "
                "nt it tmax qt boundu boundl cmax maxcourant steeringenabled finishsteering dt "
                "dx gamma mu eta g sodifon rkon moddton divbon divbfix cfgsavefrequency "
                "hyperdifmom mode readini courant maxviscoef dtdiffvisc chyp chyp3 test "
                "boundtype gpid npe noghost").split()
STATE_FIELDS = "it t dt rho m1 m2 m3 e b1 b2 b3".split()


def _layout(tmp, tag, includes, macro, incdir):
    src = os.path.join(tmp, tag + ".cpp")
    with open(src, "w") as f:
        f.write("#include <cstdio>\n#include <cstddef>\n")
        for h in includes:
            f.write('#include "%s"\n' % h)
        f.write("int main() {\n")
        for fld in PARAM_FIELDS:
            f.write('  std::printf("params.%s %%zu\\n", offsetof(struct params, %s));\n' % (fld, fld))
        for fld in STATE_FIELDS:
            f.write('  std::printf("state.%s %%zu\\n", offsetof(struct state, %s));\n' % (fld, fld))
        f.write('  std::printf("sizes %zu %zu %zu\\n", sizeof(struct params), '
                'sizeof(struct state), sizeof(struct bparams));\n  return 0;\n}\n')
    exe = os.path.join(tmp, tag)
    subprocess.check_call(["g++", "-w", "-fpermissive", macro, "-I", incdir, src, "-o", exe])
    return subprocess.run([exe], capture_output=True, text=True, check=True).stdout


@pytest.mark.skipif(not os.path.isdir(REFINC), reason="reference sources not present")
@pytest.mark.parametrize("nd", ["2d", "3d"])
def test_struct_layout_matches_reference(nd):
    with tempfile.TemporaryDirectory() as tmp:
        ours = _layout(tmp, "ours", ["smaug_compat.h"], MACROS[nd], os.path.join(ROOT, "include"))
        ref = _layout(tmp, "ref", ["iotypes.h", "iobparams.h"], MACROS[nd], REFINC)
    assert ours == ref


@pytest.mark.skipif(not os.path.isdir(REFINC), reason="reference sources not present")
def test_reference_driver_links_against_shim(engine_lib):
    from oracle import build_ref
    for name, ni, nj, nt, nk, kw in build_ref.COMPAT_STANDARD[:3]:
        binp = build_ref.build_compat(name, ni, nj, nt, verbose=False, nk=nk, **kw)
        assert os.path.exists(binp)


# --------------------------------------------------------------------------
# GPU: the unchanged driver on the engine vs the reference binary's outputs
# --------------------------------------------------------------------------
GAMMA_REF = 1.66666667


def _run_driver(name, d, env_extra=None, tmpdir=None):
    from oracle import run_ref
    from smaug_b200 import formats
    binp = os.path.join(ROOT, "oracle", "_ref", "compat_" + name, "smaug")
    if not os.path.exists(binp):
        pytest.skip("compat driver %s not built (needs the reference sources)" % name)
    ini = os.path.join(tmpdir, name + ".ini")
    if d["w0full"].ndim == 4:
        formats.write_ini(ini, d["w0full"], d["pos"], gamma=GAMMA_REF, g=tuple(d["g"]))
    else:
        formats.write_ini(ini, d["w0full"], d["pos"])
    rundir = os.path.join(tmpdir, "run")
    old = {}
    for k, v in (env_extra or {}).items():
        old[k] = os.environ.get(k)
        os.environ[k] = v
    try:
        rc, times = run_ref.run(binp, ini, rundir, keep=set(int(s) for s in d["steps"]),
                                timeout=300)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    tail = open(os.path.join(rundir, "stdout_tail.txt")).read()
    assert rc == 0, tail[-2000:]
    return rundir


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["g16", "g18x12", "t3s"])
def test_reference_driver_on_engine_matches_reference(name, tmp_path, engine_lib):
    from smaug_b200 import formats
    d = load(name)
    rundir = _run_driver(name, d, tmpdir=str(tmp_path))
    nevo = 8 if d["w0full"].ndim == 4 else 6
    nd = d["pos"].shape[0]
    pos_grid, _ = engine_lib.grid_metric(nd, list(reversed(d["pos"].shape[1:])), d["pos"])
    for k, step in enumerate(d["steps"]):
        w, pos, h = formats.read_out(os.path.join(rundir, "out", "ref_%d.out" % step))
        ref = d["states"][k]
        for f in range(nevo):
            assert _rel(w[f], ref[f]) <= 1e-12, (name, int(step), f, _rel(w[f], ref[f]))
        assert abs(h["t"] - d["hdr_t"][k]) <= 1e-12 * max(abs(d["hdr_t"][k]), 1e-300)
        # positions as the shim's initgrid rewrote them in the driver's wd
        assert np.array_equal(pos, pos_grid)


@pytest.mark.gpu
def test_reference_driver_on_engine_mixed(tmp_path):
    """SMAUG_COMPAT_PRECISION=mixed runs the same driver on the mixed form."""
    from smaug_b200 import formats
    d = load("g16")
    rundir = _run_driver("g16", d, env_extra={"SMAUG_COMPAT_PRECISION": "mixed"},
                         tmpdir=str(tmp_path))
    k = list(d["steps"]).index(5)
    w, pos, h = formats.read_out(os.path.join(rundir, "out", "ref_5.out"))
    ref = d["states"][k]
    errs = [_rel(w[f], ref[f]) for f in range(6)]
    assert max(errs) <= 1e-4, errs
    assert max(errs) > 0.0  # the float stage buffers were used


SHIM_PROBE = r"""
#include <cstdio>
#include <cstring>
#include <vector>
#include "smaug_compat.h"
int main(int argc, char** argv) {
  params* p = new params();
  std::memset(p, 0, sizeof(params));
  p->n[0] = 12; p->n[1] = 12;
  p->rkon = argv[1][0] == 'r' ? 1 : 0;
  for (int f = 0; f < SMAUG_COMPAT_NVAR; f++)
    for (int d = 0; d < SMAUG_COMPAT_NDIM; d++) p->boundtype[f][d][0] = p->boundtype[f][d][1] = 0;
  if (argv[1][0] == 'b') p->boundtype[0][1][0] = 7;
  state* st = new state();
  bparams* bp = nullptr;
  std::vector<double> wmod(2 * SMAUG_COMPAT_NVAR * 144), wd(19 * 144);
  double *w = wmod.data(), *wdp = wd.data(), *dummy = nullptr;
  params* dp = nullptr; bparams* dbp = nullptr; state* ds = nullptr;
  cuinit(&p, &bp, &w, &dummy, &wdp, &st, &dp, &dbp, &dummy, &dummy, &dummy, &dummy, &ds, &dummy,
         &dummy, &dummy);
  std::printf("cuinit returned\n");
  std::fflush(stdout);
  cuboundary(&p, &bp, &dp, &dbp, &ds, &dummy, 0, 1, 0);
  std::printf("cuboundary returned\n");
  return 0;
}
"""


@pytest.mark.parametrize("mode,expect_rc,needle", [
    ("ok", 0, None),
    ("rk", 3, "rkon=1"),
    ("bc", 3, "boundary type"),
])
def test_shim_refuses_unsupported_driver_use(engine_lib, tmp_path, mode, expect_rc, needle):
    """The reference's driver ignores wrapper return values, so the shim ends
    the process (status 3, message on stderr) on a use it does not support:
    the RK driver, or a boundary type other than 0/4/5.  (No device work is
    reached: the engine is created at the first step.)"""
    src = tmp_path / "probe.cpp"
    src.write_text(SHIM_PROBE)
    exe = tmp_path / "probe"
    subprocess.check_call(["g++", "-DUSE_SAC", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                           str(exe), "-L", PKG, "-lsmaug_compat2d", "-lsmaug_b200",
                           "-Wl,-rpath," + PKG])
    r = subprocess.run([str(exe), mode], capture_output=True, text=True, timeout=60)
    assert r.returncode == expect_rc, (r.returncode, r.stdout, r.stderr)
    if needle:
        assert "smaug_compat:" in r.stderr and needle in r.stderr, r.stderr
    else:
        assert "cuboundary returned" in r.stdout
