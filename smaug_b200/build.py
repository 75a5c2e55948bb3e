"""Build the engine shared library (sm_100a) in-tree: smaug_b200/libsmaug_b200.so."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libsmaug_b200.so")
SRCS = [os.path.join(HERE, "csrc", f) for f in ("engine.cu", "host_io.cpp")]
DEPS = SRCS + [os.path.join(HERE, "csrc", f) for f in sorted(os.listdir(os.path.join(HERE, "csrc")))
               if f.endswith((".h", ".cuh"))] + [os.path.join(ROOT, "include", "smaug_b200.h")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def build(force=False, verbose=False, extra=()):
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= max(os.path.getmtime(d) for d in DEPS)):
        return LIB
    cmd = (["nvcc"] + ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                              "-Xcompiler", "-O2", "-shared", "-o", LIB] + list(extra) + SRCS
           + ["-lcudart"])
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    extra = [a for a in sys.argv[1:] if a != "--force"]
    print(build(force=True, verbose=True, extra=extra))
