"""Build the in-tree CUDA library raishinsource_b200/libraishin_gpu.so.

nvcc compiles the sm_100a kernels (-gencode arch=compute_100a,code=sm_100a)
and the host side of the C ABI into one shared library with plain extern "C"
entry points (include/raishin_gpu.h).  Multiply-adds are contracted into FMA
(the arithmetic the parity tests hold to 1e-12 per step against the oracle);
RG_FMAD=0 builds the uncontracted variant whose operation sequence equals the
reference's (gfortran -O2 on x86-64 emits no FMA).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libraishin_gpu.so")
SOURCES = ["rg_kernels.cu", "rg_capi.cu", "rg_geometry.cpp"]
HEADERS = ["rg_device.cuh", "rg_recon.cuh", "rg_kernels.cuh", "rg_batch.cuh", "rg_types.h", "rg_host.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def build(force: bool = False, verbose: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(HERE, "..", "include", "raishin_gpu.h"), os.path.abspath(__file__)]
    if not force and os.path.exists(LIB):
        t = os.path.getmtime(LIB)
        if all(os.path.getmtime(d) <= t for d in deps):
            return LIB
    tmp = LIB + ".tmp%d" % os.getpid()
    fmad = "false" if os.environ.get("RG_FMAD", "1") == "0" else "true"
    cmd = [nvcc(), "-O3", "-std=c++17", *ARCH, "-lineinfo", f"--fmad={fmad}", "-shared",
           "-Xcompiler", "-fPIC,-ffp-contract=off,-O2,-fopenmp", "-o", tmp, *srcs, "-lgomp"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
