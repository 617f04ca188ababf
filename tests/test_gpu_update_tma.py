"""GPU: the TMA-staged stage update (k_update_tma) against the generic one
(k_update).

For runs stored in full the stage update stages the rows its RK combine
reads -- the three face-flux arrays, the flux-CT components and U^n
(rkt.f90:2-180 with ct.f90:98-109; in the FP32 region of a mixed run the
FP32 fluxes) -- in shared memory by TMA tile loads.  It
reads the same values and performs the same operations as the generic
kernel.  In the uncontracted build (libraishin_gpu_exact.so) a context with
it (the default) and one without it (RAISHIN_UPDATE_TMA=0, read when the
context is created) therefore give the same state bit for bit, over many
steps and with the boxes clipped at every edge of the grid.  In the FMA build
the compiler contracts each kernel on its own, so the two agree to rounding.
"""
import json
import os
import subprocess
import sys

import pytest

from conftest import has_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="no CUDA device")]

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CASES = {
    # imax not a multiple of the block's 32 cells, jmax not a multiple of its 4 rows
    "mp5_40x26x16": dict(nr=40, nth=16, nph=26, irec=6),
    "ppm_48x24x20": dict(nr=48, nth=20, nph=24, irec=5),
    "mc_ict2_36x20x18": dict(nr=36, nth=18, nph=20, irec=1, ict=2),
    # imax = 2 (mod 4): the update is staged, the faces are not (their TMA wants imax a multiple of 4)
    "mp5_42x20x16": dict(nr=42, nth=16, nph=20, irec=6),
    # a mixed run: FP64 update inside 2 r_H, the staged FP32-region kernel (FP32 fluxes, FP64 U^n) beyond
    "mixed_mp5_40x24x16": dict(nr=40, nth=16, nph=24, irec=6, precision="mixed"),
}

CHILD = r"""
import json, os, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from oracle import Oracle
from raishinsource_b200 import Context, config

cases, nsteps = json.loads(sys.argv[2]), int(sys.argv[3])
res = {}
for name, kw in cases.items():
    p = dict(config.torus(**kw), guard=1)
    o = Oracle(p); o.ic_torus(seed=77); o.init_cons()
    q0 = o.prims()
    out = {}
    for flag in ("1", "0"):
        os.environ["RAISHIN_UPDATE_TMA"] = flag
        with Context(0) as ctx:
            r = ctx.admit(p); r.upload_prims(q0)
            st = r.step(nsteps, stats=True, strict=False)
            out[flag] = (r.prims(), [st["recov_fail"], st["recov_carry"]])
            r.release()
    a, b = out["1"][0], out["0"][0]
    scale = np.abs(b).reshape(-1, 9).max(axis=0).clip(1e-300)
    res[name] = dict(equal=bool(np.array_equal(a, b, equal_nan=True)), finite=bool(np.isfinite(a).all()),
                     rel=float((np.abs(a - b).reshape(-1, 9).max(axis=0) / scale).max()),
                     counts=[out["1"][1], out["0"][1]])
maps = open("/proc/self/maps").read()
res["libs"] = sorted({l.split()[-1] for l in maps.splitlines() if "libraishin_gpu" in l})
print(json.dumps(res))
"""


def run_child(lib, nsteps):
    env = dict(os.environ)
    if lib:
        env["RAISHIN_GPU_LIB"] = lib
    else:
        env.pop("RAISHIN_GPU_LIB", None)
    out = subprocess.run([sys.executable, "-c", CHILD, ROOT, json.dumps(CASES), str(nsteps)], env=env, cwd=ROOT,
                         capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, out.stderr[-3000:]
    res = json.loads(out.stdout.strip().splitlines()[-1])
    return res.pop("libs"), res


def test_staged_update_equals_generic_bit_for_bit_uncontracted():
    libs, res = run_child("exact", 40)
    assert [os.path.basename(x) for x in libs] == ["libraishin_gpu_exact.so"], libs
    for case, r in res.items():
        assert r["equal"] and r["finite"], (case, r)
        assert r["counts"][0] == r["counts"][1], (case, r)


def test_staged_update_agrees_with_generic_fma_build():
    libs, res = run_child(None, 1)
    assert [os.path.basename(x) for x in libs] == ["libraishin_gpu.so"], libs
    for case, r in res.items():
        assert r["finite"] and r["rel"] < 1e-13, (case, r)
