"""Build the engine shared library (sm_100a) in-tree: smaug_b200/libsmaug_b200.so,
and the reference-wrapper shims libsmaug_compat2d.so / libsmaug_compat3d.so on
top of it (host C++, one per NDIM as the reference's struct params differs).

The translation units (the 2D and 3D stage kernels, the engine host code and
the file formats) compile to objects in parallel under smaug_b200/_build/,
then nvcc links them.  An object is rebuilt when its source or one of the
headers under csrc/ or include/ is newer than it.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libsmaug_b200.so")
OBJDIR = os.path.join(HERE, "_build")
CSRC = os.path.join(HERE, "csrc")
SRCS = [os.path.join(CSRC, f) for f in ("engine.cu", "stage2d.cu", "stage2d_tma.cu", "stage3d.cu", "batch.cu", "batch16.cu",
                                         "adjoint.cu", "host_io.cpp")]
HEADERS = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith((".h", ".cuh"))] + [
    os.path.join(ROOT, "include", "smaug_b200.h")]
COMPAT_SRC = os.path.join(CSRC, "compat.cpp")
COMPAT_HDR = os.path.join(ROOT, "include", "smaug_compat.h")
# (library, build macro of the reference): USE_SAC = 2D, USE_SAC_3D = 3D
COMPAT = [(os.path.join(HERE, "libsmaug_compat2d.so"), "-DUSE_SAC"),
          (os.path.join(HERE, "libsmaug_compat3d.so"), "-DUSE_SAC_3D")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2"]


def _obj(src):
    return os.path.join(OBJDIR, os.path.basename(src) + ".o")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, extra, verbose):
    cmd = ["nvcc"] + ARCH + FLAGS + list(extra) + ["-c", "-o", _obj(src), src]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def build(force=False, verbose=False, extra=()):
    os.makedirs(OBJDIR, exist_ok=True)
    todo = [s for s in SRCS if force or _stale(_obj(s), [s] + HEADERS)]
    if todo:
        with ThreadPoolExecutor(max_workers=len(todo)) as ex:
            for f in [ex.submit(_compile, s, extra, verbose) for s in todo]:
                f.result()
    objs = [_obj(s) for s in SRCS]
    if force or todo or _stale(LIB, objs):
        cmd = ["nvcc"] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    for lib, macro in COMPAT:
        if force or _stale(lib, [COMPAT_SRC, COMPAT_HDR, os.path.join(ROOT, "include", "smaug_b200.h"),
                                 LIB]):
            cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-Wall", macro,
                   "-I", os.path.join(ROOT, "include"), "-o", lib, COMPAT_SRC,
                   "-L", HERE, "-lsmaug_b200", "-Wl,-rpath,$ORIGIN"]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    extra = [a for a in sys.argv[1:] if a != "--force"]
    print(build(force=True, verbose=True, extra=extra))
