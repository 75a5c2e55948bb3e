"""The C-ABI library builds for sm_100a, loads, and exports every entry point
declared in include/smaug_b200.h (no compute calls: CPU-safe)."""
import ctypes
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "smaug_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(smaug_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_core_api():
    syms = declared_symbols()
    for s in ("smaug_create", "smaug_step", "smaug_get_state", "smaug_destroy",
              "smaug_last_error", "smaug_write_out", "smaug_read_ini"):
        assert s in syms


def test_library_exports_all_declared(engine_lib):
    lib = ctypes.CDLL(engine_lib.LIBPATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_exports_are_unmangled(engine_lib):
    out = subprocess.run(["nm", "-D", "--defined-only", engine_lib.LIBPATH],
                         capture_output=True, text=True, check=True).stdout
    names = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    for s in declared_symbols():
        assert s in names, s


def test_python_binding_lists_exports(engine_lib):
    assert set(engine_lib.EXPORTS) == set(declared_symbols())


def test_library_is_sm100a(engine_lib):
    """The shared object carries sm_100a device code (cuobjdump is not used:
    the ELF notes list the targets through the CUDA fatbin header)."""
    from smaug_b200 import build
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)


def test_version_string(engine_lib):
    assert "sm_100a" in engine_lib.version()


def test_params_default_without_gpu(engine_lib):
    from smaug_b200.params import SmaugParams
    p = SmaugParams()
    rc = engine_lib.lib().smaug_params_default(ctypes.byref(p), 2)
    assert rc == 0 and p.ndim == 2 and p.version == 1 and p.n[0] == 132
    rc = engine_lib.lib().smaug_params_default(ctypes.byref(p), 4)
    assert rc == 1 and b"bad" in engine_lib.lib().smaug_last_error()
