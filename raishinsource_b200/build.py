"""Build the in-tree CUDA libraries.

nvcc compiles the sm_100a kernels (-gencode arch=compute_100a,code=sm_100a)
and the host side of the C ABI into shared libraries with plain extern "C"
entry points (include/raishin_gpu.h).  Two variants of the same sources:

* libraishin_gpu.so (the product): multiply-adds contracted into FMA, and
  x**gam for gam = 4/3 or 5/3 evaluated through cbrt.  The parity tests hold
  it to 1e-12 of the oracle per step.
* libraishin_gpu_exact.so: no FMA contraction (--fmad=false) and every power
  of the step through the library's own rg_pow (include/rg_pow.h, IEEE basic
  operations only), so that the operation sequence is the reference's
  (gfortran -O2 on x86-64 emits no FMA) and a host restatement that uses
  rg_pow as well reproduces it bit for bit, step after step.  It exists for
  long-horizon parity (1000 steps), where MP5's limiter switches amplify any
  last-bit difference.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libraishin_gpu.so")
EXACT_LIB = os.path.join(HERE, "libraishin_gpu_exact.so")
VARIANTS = {
    "fast": (LIB, ["--fmad=true"]),
    "exact": (EXACT_LIB, ["--fmad=false", "-DRG_EXACT_ARITH"]),
}
SOURCES = ["rg_kernels.cu", "rg_ic.cu", "rg_capi.cu", "rg_geometry.cpp"]
HEADERS = ["rg_device.cuh", "rg_recon.cuh", "rg_kernels.cuh", "rg_batch.cuh", "rg_types.h", "rg_host.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _command(variant: str, out: str, verbose: bool) -> list:
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    cmd = [nvcc(), "-O3", "-std=c++17", *ARCH, "-lineinfo", *VARIANTS[variant][1], "-shared",
           "-Xcompiler", "-fPIC,-ffp-contract=off,-O2,-fopenmp", "-o", out, *srcs, "-lgomp"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    return cmd


def _stale(path: str) -> bool:
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [
        os.path.join(HERE, "..", "include", "raishin_gpu.h"), os.path.join(HERE, "..", "include", "rg_pow.h"),
        os.path.abspath(__file__)]
    if not os.path.exists(path):
        return True
    t = os.path.getmtime(path)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, variants=("fast",)) -> str:
    """Compile the named variants (concurrently) if stale; returns the path
    of the first."""
    jobs = []
    for v in variants:
        path = VARIANTS[v][0]
        if force or _stale(path):
            tmp = path + ".tmp%d" % os.getpid()
            jobs.append((subprocess.Popen(_command(v, tmp, verbose)), tmp, path))
    failed = []
    for proc, tmp, path in jobs:
        if proc.wait() != 0:
            failed.append(path)
        else:
            os.replace(tmp, path)
    if failed:
        raise RuntimeError("nvcc failed for " + ", ".join(failed))
    return VARIANTS[variants[0]][0]


def build_all(force: bool = False) -> None:
    build(force=force, variants=tuple(VARIANTS))


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv,
                variants=tuple(VARIANTS) if "--all" in sys.argv else ("fast",)))
