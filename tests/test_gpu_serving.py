"""GPU: continuous batching of a request stream (raishinsource_b200.serving).

Requests arrive while others are on the GPU, are admitted as slots and
memory free up, and step together with the resident runs.  Each result must
equal the same run stepped alone: the stated tolerance is exact equality,
because a slab run goes through the same compiled kernels alone and in any
batch.
"""
import numpy as np
import pytest

from raishinsource_b200 import config, serving
from raishinsource_b200.capi import footprint

pytestmark = pytest.mark.gpu


def test_stream_results_equal_alone(gpu_ctx):
    reqs = serving.poisson_stream(8, rate=200.0, seed=9, steps=40, grids=(48, 64, 72))
    big = max(footprint(r.params) for r in reqs)
    # a budget of about two runs: later arrivals wait for memory to free up
    srv = serving.Server(gpu_ctx, mem_budget=int(2.2 * big), max_runs=4, tick_steps=10, keep_prims=True)
    out = srv.serve(reqs)
    srv.close()
    assert out["requests"] == len(reqs)
    assert out["p50_latency_s"] <= out["p99_latency_s"]
    assert out["zone_updates"] == sum(config.interior_cells(r.params) * r.steps for r in reqs)
    assert any(d.admitted > d.arrival for d in out["done"])
    by_id = {d.rid: d for d in out["done"]}
    for r in reqs:
        run = gpu_ctx.admit(r.params)
        run.ic_torus(**r.ic)
        run.step(r.steps)
        alone = run.prims()
        run.release()
        got = by_id[r.rid].prims
        assert np.isfinite(got).all()
        assert np.array_equal(got, alone), r.rid


def test_admission_respects_budget(gpu_ctx):
    reqs = serving.poisson_stream(5, rate=1000.0, seed=3, steps=20, grids=(48,))
    fps = [footprint(r.params) for r in reqs]
    budget = int(1.02 * max(fps))
    assert budget < 2 * min(fps)  # room for exactly one run
    srv = serving.Server(gpu_ctx, mem_budget=budget, max_runs=8, tick_steps=20)
    out = srv.serve(reqs)
    srv.close()
    done = sorted(out["done"], key=lambda d: d.admitted)
    # with room for one run at a time, every run is admitted after the previous one finished
    for a, b in zip(done, done[1:]):
        assert b.admitted >= a.finished
    assert out["ticks"] == len(reqs)


def test_stream_marks(gpu_ctx):
    """rg_ctx_mark / rg_ctx_wait_mark: a mark after queued steps completes,
    an unused slot reports completion, an out-of-range slot is refused."""
    from raishinsource_b200.capi import RgError
    p = config.torus(nr=64, nth=64)
    r = gpu_ctx.admit(p)
    r.ic_torus(seed=5)
    gpu_ctx.step_batch([r], 20)
    gpu_ctx.mark(3)
    assert gpu_ctx.wait_mark(3) is True
    assert gpu_ctx.wait_mark(3, block=False) is True
    assert gpu_ctx.wait_mark(5, block=False) is True
    with pytest.raises(RgError):
        gpu_ctx.mark(8)
    r.release()
