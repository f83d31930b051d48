"""Build recipe for the oracle (test infrastructure): compiles
oracle/grn_oracle.cpp into oracle/_build/libgrn_oracle.so with g++.

The reference's own CPU simulator cannot be compiled here: its sources
include Qt5 and Eigen headers, which are not installed, so no oracle/_ref
library is built.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libgrn_oracle.so")
SOURCES = [os.path.join(HERE, "grn_oracle.cpp")]
DEPS = SOURCES + [os.path.join(HERE, "grn_oracle.h"),
                  os.path.join(HERE, "..", "include", "grn_gpu.h")]


def build(force=False, verbose=False):
    os.makedirs(OUT_DIR, exist_ok=True)
    if not force and os.path.exists(LIB):
        t = os.path.getmtime(LIB)
        if all(os.path.getmtime(d) <= t for d in DEPS):
            return LIB
    # -O2 without -ffast-math: the restatement must keep IEEE FP64 semantics.
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-pthread",
           "-fno-fast-math", "-ffp-contract=off", "-o", LIB] + SOURCES
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
