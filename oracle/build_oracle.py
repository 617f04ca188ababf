"""Build recipe for the CPU oracle (test infrastructure only).

Compiles oracle/*.cpp into oracle/_build/liboracle.so with
-O2 -ffp-contract=off (no FMA contraction, no reassociation: the arithmetic
model of gfortran -O2 on x86-64) and OpenMP over the outer k loops.

The reference itself (Fortran 90 + MPI) cannot be built on this machine: there
is no Fortran compiler and no MPI.  oracle/_ref/ is therefore never produced.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "liboracle.so")
SOURCES = ["oracle_geom.cpp", "oracle_step.cpp", "oracle_ic.cpp", "oracle_post.cpp", "oracle_api.cpp"]
FLAGS = ["-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared", "-std=c++17",
         "-Wall", "-Wno-unused-variable"]


def build(force: bool = False) -> str:
    srcs = [os.path.join(HERE, s) for s in SOURCES]
    deps = srcs + [os.path.join(HERE, "oracle.hpp"), os.path.join(HERE, "..", "include", "rg_pow.h")]
    if not force and os.path.exists(LIB):
        t = os.path.getmtime(LIB)
        if all(os.path.getmtime(d) <= t for d in deps):
            return LIB
    os.makedirs(BUILD, exist_ok=True)
    tmp = LIB + ".tmp%d" % os.getpid()
    cmd = ["g++"] + FLAGS + srcs + ["-o", tmp]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
