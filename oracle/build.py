"""Build the CPU oracle (test infrastructure) into oracle/_build/liboracle.so.

The oracle is the parity checker for the CUDA engine; it is compiled with
plain gcc, -O2, no FMA contraction, OpenMP over cells.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "liboracle.so")
SRC = os.path.join(HERE, "smaug_oracle.c")


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= os.path.getmtime(SRC)):
        return LIB
    cmd = ["gcc", "-O2", "-std=gnu99", "-fPIC", "-shared", "-fopenmp",
           "-ffp-contract=off", "-Wall", "-Wno-unused-variable",
           "-Wno-unused-but-set-variable", "-o", LIB, SRC, "-lm"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
