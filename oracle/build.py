"""Build recipe for the oracle (test infrastructure only).

Compiles oracle/oracle_capi.cpp into oracle/_build/liborc.so with g++ (OpenMP,
-ffp-contract=off so that the float instance performs exactly the IEEE operations
the source spells out; the intersection KAT relies on this).
The reference itself cannot be compiled here (bazel + clang-15/libc++ + enoki +
OptiX SDK are required), so there is no oracle/_ref build.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liborc.so")
SRCS = [os.path.join(HERE, "oracle_capi.cpp")]
DEPS = SRCS + [os.path.join(HERE, "psdr_oracle.hpp")]


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    if not force and os.path.exists(LIB):
        mt = os.path.getmtime(LIB)
        if all(os.path.getmtime(d) <= mt for d in DEPS):
            return LIB
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
           "-fno-fast-math", "-o", LIB] + SRCS
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
