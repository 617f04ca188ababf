"""The allocation-free flux entry point (rg_calflx_static).

A host program whose device memory comes only from its own pool or arena
cannot let the library call cudaMalloc behind its back (the allocation would
synchronise the device and take memory the pool does not know about).  Such a
caller passes its own device buffers and gets the same fluxes as rg_calflx,
with flux-CT's intermediate held in the library's static device array.  This
file is collected last so that a run stopping at the first failure has already
run every other test; it also passes alone in a fresh process.
"""
import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.mark.skipif(not has_gpu(), reason="no CUDA device")
def test_calflx_static_matches_calflx_two_calls():
    import torch

    from oracle import Oracle
    from raishinsource_b200 import Context, config

    p = dict(config.torus(nr=48, nth=40, nph=12), guard=1)
    N = p["imax"] * p["jmax"] * p["kmax"]
    nm0, _ = config.ghost_widths(p["irec"], p.get("ict", 1))
    reg = (slice(nm0, -nm0),) * 3  # inside the hll range (1-based nm0..n-nm0)
    states = []
    for seed in (21, 22):
        o = Oracle(p)
        o.ic_torus(seed=seed)
        states.append(o.prims())
    with Context(0) as ctx:
        run = ctx.admit(p)
        d_prims = torch.empty((9, N), dtype=torch.float64, device="cuda")
        d_ww = torch.empty((3, 9, N), dtype=torch.float64, device="cuda")
        free_after = []
        for u in states:
            want = run.calflx(u)  # (kmax, jmax, imax, 9, 3) through the allocating entry point
            d_prims.copy_(torch.from_numpy(np.ascontiguousarray(u.reshape(N, 9).T)))
            d_ww.fill_(np.nan)
            torch.cuda.synchronize()
            run.calflx_static(d_prims.data_ptr(), d_ww.data_ptr())
            free_after.append(torch.cuda.mem_get_info()[0])
            got = d_ww.cpu().numpy().reshape(3, 9, p["kmax"], p["jmax"], p["imax"])
            got = np.moveaxis(got, (0, 1), (4, 3))  # -> (kmax, jmax, imax, 9, 3)
            a, b = got[reg], want[reg]
            scale = np.maximum(np.abs(b).max(axis=(0, 1, 2)), 1e-300)
            err = np.abs(a - b).max(axis=(0, 1, 2)) / scale
            assert np.isfinite(a).all()
            assert err.max() < TOL, err
        run.release()
    # the second call allocated nothing
    assert free_after[0] == free_after[1]


@pytest.mark.skipif(not has_gpu(), reason="no CUDA device")
def test_calflx_static_rejects_grids_beyond_its_scratch():
    import torch

    from raishinsource_b200 import Context, RgError, config

    p = config.torus(nr=96, nth=96, nph=32)  # 294912 cells > 262144
    N = p["imax"] * p["jmax"] * p["kmax"]
    with Context(0) as ctx:
        run = ctx.admit(p)
        d_prims = torch.zeros((9, N), dtype=torch.float64, device="cuda")
        d_ww = torch.zeros((3, 9, N), dtype=torch.float64, device="cuda")
        with pytest.raises(RgError) as e:
            run.calflx_static(d_prims.data_ptr(), d_ww.data_ptr())
        assert e.value.code == 1 and "262144" in str(e.value)
        run.release()
