"""GPU: the uncontracted-arithmetic build (libraishin_gpu_exact.so: no FMA
contraction, every power through pow()) against the oracle.

Its operation sequence is the oracle's (the C++ restatement is compiled with
-ffp-contract=off, as gfortran -O2 on x86-64 emits no FMA), so after one RK3
step the only differences left are last-bit differences between CUDA's and
glibc's pow/exp/log/sin/cos: the L1 difference of every field is a few units
of 1e-16 or less, against up to 1e-13 for the FMA build.  The library is
process-global, so the check runs in a child process, which also reports
which library file it mapped.
"""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from oracle import Oracle
from raishinsource_b200 import Context, config
res = {}
with Context(0) as ctx:
    for irec, guard in ((6, 1), (6, 3), (5, 0), (7, 1)):
        p = dict(config.torus(nr=64, nth=64, irec=irec), guard=guard)
        o = Oracle(p); o.ic_torus(seed=4); o.init_cons()
        r = ctx.admit(p); r.upload_prims(o.prims())
        o.step(1); r.step(1)
        a, b = r.prims(), o.prims(); r.release()
        n = o.nm1
        sl = (slice(n, -n),) * 3
        l1 = np.abs(a[sl] - b[sl]).sum(axis=(0, 1, 2)) / np.abs(b[sl]).sum(axis=(0, 1, 2)).clip(1e-300)
        res["%d_%d" % (irec, guard)] = [float(x) for x in l1]
maps = open("/proc/self/maps").read()
res["libs"] = sorted({l.split()[-1] for l in maps.splitlines() if "libraishin_gpu" in l})
print(json.dumps(res))
"""


def test_exact_build_one_step_agrees_to_last_bits():
    env = dict(os.environ, RAISHIN_GPU_LIB="exact")
    out = subprocess.run([sys.executable, "-c", CHILD, ROOT], env=env, cwd=ROOT, capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    res = json.loads(out.stdout.strip().splitlines()[-1])
    libs = res.pop("libs")
    assert [os.path.basename(x) for x in libs] == ["libraishin_gpu_exact.so"], libs
    for case, l1 in res.items():
        worst = max(l1[v] for v in (0, 1, 2, 3, 4, 6, 7, 8))
        assert worst < 2e-15, (case, l1)
