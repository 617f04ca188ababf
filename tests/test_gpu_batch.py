"""GPU: 1D Riemann tubes (transverse directions stored as one plane) against
the oracle, and batched steps (rg_step_batch) against the same runs stepped
alone.

A run with a slab direction steps through the batched kernels alone (as a
batch of one) and in any batch, and the tuner changes only which block takes
which tile, so its result in a batch equals its result alone bit for bit; the
tests assert exact equality.  Tube parity with the oracle uses the per-step
bound of the FP64 path (1e-12 of each field's maximum).
"""
import numpy as np
import pytest

from conftest import field_err
from oracle import Oracle
from raishinsource_b200 import config

pytestmark = pytest.mark.gpu

TOL = 1e-12


def test_tube_ic_matches_oracle(gpu_ctx):
    p = config.tube(n=120)
    o = Oracle(p)
    o.ic_tube(seed=7, tube=3)
    r = gpu_ctx.admit(p)
    r.ic_tube(seed=7, tube=3)
    got = r.prims()
    r.release()
    assert np.array_equal(got, o.prims())


@pytest.mark.parametrize("tube", [0, 1, 2, 5])
def test_tube_steps_match_oracle(gpu_ctx, tube):
    """Seeded tubes (some hit the b^2/rho and b^2/p ceilings of pminmax2b):
    five steps, each restarted from the oracle's state."""
    p = config.tube(n=160)
    o = Oracle(p)
    o.ic_tube(seed=2012, tube=tube)
    o.init_cons()
    r = gpu_ctx.admit(p)
    r.ic_tube(seed=2012, tube=tube)
    errs = []
    for _ in range(5):
        o.step(1)
        r.step(1)
        errs.append(field_err(r.prims(), o.prims()).max())
        r.upload_prims(o.prims(), t0=o.time)
    r.release()
    assert max(errs) < TOL, errs


def test_tube_runs_to_tmax(gpu_ctx):
    """The loop-top time check (main.f90:617-632): a run stops once time > tmax."""
    p = config.tube(n=100, tmax=0.05)
    r = gpu_ctx.admit(p)
    r.ic_tube(seed=1, tube=0)
    st = r.step(100000, stats=True)
    r.release()
    assert st["time"] > 0.05
    assert st["time"] - st["dt"] <= 0.05 + 1e-15
    assert 0 < st["steps"] < 100000


def _alone_vs_batch(gpu_ctx, params, ics, steps, info=True):
    alone, batch = [], []
    for p, ic in zip(params, ics):
        a = gpu_ctx.admit(p)
        b = gpu_ctx.admit(p)
        ic(a)
        ic(b)
        alone.append(a)
        batch.append(b)
    for a in alone:
        a.step(steps)
    st = gpu_ctx.step_batch(batch, steps, stats=True)
    # one batch per class (precision etc.); report the tuned shape of the first run's class
    if info:
        same = [b for b, p in zip(batch, params) if p.get("precision", "fp64") == params[0].get("precision", "fp64")]
        info = gpu_ctx.batch_info(same)
    out = []
    for a, b, s in zip(alone, batch, st):
        sa = a.stats()
        out.append((a.prims(), b.prims(), sa, s))
        a.release()
        b.release()
    return out, info


def test_batch_tubes_equal_alone(gpu_ctx):
    """70 steps in one call: the batch starts with the default shape, is tuned
    after its 32nd step (block width, cells per tile, persistent grid) and
    continues with the chosen shape; every tube still equals itself alone."""
    lengths = [400, 517, 1203, 64, 900]
    params = [config.tube(n=n, tmax=0.4) for n in lengths]
    ics = [lambda r, t=t: r.ic_tube(seed=2012, tube=t) for t in range(len(lengths))]
    out, info = _alone_vs_batch(gpu_ctx, params, ics, 70)
    for a, b, sa, sb in out:
        assert np.array_equal(a, b)
        assert sa["time"] == sb["time"] and sa["steps"] == sb["steps"] == 70
    assert info["launches_per_step"] > 0 and info["tuned_ms_per_step"] > 0
    assert info["width"] in (64, 128) and info["tile_cells"] in (64, 128, 256, 512)


def test_batch_tori_fp64_and_mixed_equal_alone(gpu_ctx):
    """2D phi-slab tori of different sizes and spins, FP64 and mixed
    precision in one call (two batch classes)."""
    params = [
        dict(config.torus(nr=64, nth=64, akm=0.5), guard=1),
        dict(config.torus(nr=96, nth=64, akm=0.9375), guard=1),
        dict(config.torus(nr=64, nth=96, akm=0.9375, precision="mixed"), guard=1),
        dict(config.torus(nr=80, nth=80, akm=0.7, precision="mixed"), guard=1),
    ]
    ics = [lambda r, s=s: r.ic_torus(seed=100 + s) for s in range(len(params))]
    out, _ = _alone_vs_batch(gpu_ctx, params, ics, 10)
    for a, b, sa, sb in out:
        assert np.isfinite(b).all()
        assert np.array_equal(a, b)
        assert sa["time"] == sb["time"]


def test_batch_with_3d_and_unbatched_schemes_equals_alone(gpu_ctx):
    """Runs without a slab direction (3D tori, which fill the GPU alone) and
    runs whose schemes have no batched kernels (upwind flux-CT, recov2) join a
    batch and take each step with their own launches, after the tubes' batched
    step: every run, the tubes included, equals itself stepped alone (rg_step)
    bit for bit."""
    params = [
        dict(config.torus(nr=40, nth=24, nph=16), guard=1),                 # 3D, MP5, staged kernels
        dict(config.torus(nr=36, nth=20, nph=18, irec=5), guard=1),         # 3D PPM
        dict(config.torus(nr=48, nth=40, ict=3), guard=1),                  # 2D slab, upwind flux-CT
        dict(config.torus(nr=40, nth=28, nph=12), guard=1, iwvec=2),        # 3D recov2
        config.tube(n=300, tmax=0.4),
        config.tube(n=517, tmax=0.4),
    ]
    ics = [lambda r: r.ic_torus(seed=31), lambda r: r.ic_torus(seed=32), lambda r: r.ic_torus(seed=33),
           lambda r: r.ic_torus(seed=34), lambda r: r.ic_tube(seed=2012, tube=1),
           lambda r: r.ic_tube(seed=2012, tube=2)]
    out, _ = _alone_vs_batch(gpu_ctx, params, ics, 6, info=False)
    for n, (a, b, sa, sb) in enumerate(out):
        assert np.isfinite(b).all(), n
        assert np.array_equal(a, b), n
        assert sa["time"] == sb["time"] and sa["steps"] == sb["steps"] == 6, n


def test_batch_membership_change_and_release(gpu_ctx):
    """A run released after a batched step leaves the other runs' batches usable."""
    rs = [gpu_ctx.admit(config.tube(n=200)) for _ in range(3)]
    for t, r in enumerate(rs):
        r.ic_tube(seed=5, tube=t)
    gpu_ctx.step_batch(rs, 3)
    rs[1].release()
    keep = [rs[0], rs[2]]
    gpu_ctx.step_batch(keep, 3)
    solo = gpu_ctx.admit(config.tube(n=200))
    solo.ic_tube(seed=5, tube=2)
    solo.step(6)
    assert np.array_equal(solo.prims(), rs[2].prims())
    for r in (rs[0], rs[2], solo):
        r.release()


def test_tube_mixed_tracks_fp64(gpu_ctx):
    """FP32-mixed tubes (Minkowski: no FP64 region) stay close to FP64 over 40 steps."""
    ps = [dict(config.tube(n=300), guard=1), dict(config.tube(n=300, precision="mixed"), guard=1)]
    rs = [gpu_ctx.admit(p) for p in ps]
    for r in rs:
        r.ic_tube(seed=2012, tube=4)
    for r in rs:
        r.step(40)
    a, b = rs[1].stored_prims()[:, 0, 0, :], rs[0].stored_prims()[:, 0, 0, :]
    for r in rs:
        r.release()
    l1 = np.abs(a - b).sum(axis=1) / np.abs(b).sum(axis=1).clip(1e-300)
    assert np.isfinite(a).all()
    assert l1[0] < 1e-4, l1
