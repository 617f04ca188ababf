"""GPU parity: the sm_100a path (through the C ABI) against the oracle.

Tolerance: the FP64 kernels keep the reference's evaluation order; the
product build contracts multiply-adds into FMA and evaluates x**(4/3) and
x**(5/3) through cbrt, so results differ from the oracle in the last bits.
Per-routine results must agree to 1e-12 of each field's maximum (relative
L-infinity per variable); one full RK3 step likewise (the parity bound of
1e-12 per step).
"""
import numpy as np
import pytest

from conftest import field_err
from oracle import Oracle
from raishinsource_b200 import config

pytestmark = pytest.mark.gpu

TOL = 1e-12


def flux_err(a, b):
    """max |a-b| per (variable, direction) relative to the variable's largest
    flux over all three directions (a direction whose flux vanishes in exact
    arithmetic may carry round-off residue of the others' size)."""
    fin = np.isfinite(b)
    scale = np.abs(np.where(fin, b, 0)).max(axis=(0, 1, 2, 4))[:, None]
    diff = np.abs(np.where(fin, a - b, 0)).max(axis=(0, 1, 2))
    return diff / np.maximum(scale, 1e-300)


def _pair(gpu_ctx, p, seed=2012):
    o = Oracle(p)
    o.ic_torus(seed=seed)
    r = gpu_ctx.admit(p)
    r.upload_prims(o.prims())
    return o, r


@pytest.fixture(scope="module")
def torus2d(gpu_ctx):
    p = config.torus(nr=64, nth=64)
    p["guard"] = 1
    o, r = _pair(gpu_ctx, p)
    yield p, o, r
    r.release()


@pytest.fixture(scope="module")
def torus3d(gpu_ctx):
    p = config.torus(nr=40, nth=24, nph=16)
    p["guard"] = 1
    o, r = _pair(gpu_ctx, p, seed=99)
    yield p, o, r
    r.release()


def test_ic_torus_matches_oracle(gpu_ctx):
    p = config.torus(nr=64, nth=48, nph=12)
    o = Oracle(p)
    o.ic_torus(seed=123, amp=0.04)
    r = gpu_ctx.admit(p)
    r.ic_torus(seed=123, amp=0.04)
    err = field_err(r.prims(), o.prims())
    r.release()
    assert err.max() < 1e-13, err


@pytest.mark.parametrize("irec,ict,nph", [(config.IREC_MC, 1, None), (config.IREC_PPM, 1, None),
                                          (config.IREC_MP5, 2, None), (config.IREC_MC, 0, 12)])
def test_ic_torus_ghost_widths(gpu_ctx, irec, ict, nph):
    """Device-side torus initial data for every ghost width nm1 = nm0 + ict: 2D
    phi slabs (stored as one plane, jmax = 2*nm1+1) and a 3D run."""
    p = config.torus(nr=48, nth=40, nph=nph, irec=irec, ict=ict)
    o = Oracle(p)
    o.ic_torus(seed=61)
    r = gpu_ctx.admit(p)
    r.ic_torus(seed=61)
    err = field_err(r.prims(), o.prims())
    r.release()
    assert err.max() < 1e-13, err


@pytest.mark.parametrize("case", ["mks3d", "slab_mc_ict0", "slab_ppm", "ks303", "mixed3d", "full_slab"])
def test_ic_torus_device(gpu_ctx, case):
    """Torus initial data computed on the device (rg_run_ic_torus_device)
    against the oracle's construction and the host one: the same torus cells,
    every primitive within a few units in the last place (CUDA's exp, log and
    pow in the per-cell terms), on MKS and Kerr-Schild grids, phi slabs
    stored as one plane or in full, every ghost width and the FP32-mixed
    layout."""
    p = {
        "mks3d": lambda: config.torus(nr=64, nth=48, nph=12),
        "slab_mc_ict0": lambda: config.torus(nr=48, nth=40, irec=config.IREC_MC, ict=0),
        "slab_ppm": lambda: config.torus(nr=64, nth=64, irec=config.IREC_PPM),
        "ks303": lambda: dict(config.torus(nr=48, nth=40, nph=12), metric=303, ix1=1, ix3=1, xmax=30.0),
        "mixed3d": lambda: config.torus(nr=48, nth=32, nph=12, precision="mixed"),
        "full_slab": lambda: dict(config.torus(nr=48, nth=40), flags=config.FLAG_FULL),
    }[case]()
    o = Oracle(p)
    o.ic_torus(seed=17, amp=0.04, beta=50.0)
    rh = gpu_ctx.admit(p)
    rd = gpu_ctx.admit(p)
    try:
        rh.ic_torus(seed=17, amp=0.04, beta=50.0)
        rd.ic_torus_device(seed=17, amp=0.04, beta=50.0)
        ref, host, dev = o.prims(), rh.prims(), rd.prims()
    finally:
        rh.release()
        rd.release()
    assert field_err(host, ref).max() < 1e-13
    torus = ref[..., 1:4].any(axis=-1)
    assert torus.sum() > 100
    assert np.array_equal(dev[..., 1:4].any(axis=-1), torus)
    err = field_err(dev, ref)
    assert err.max() < 1e-12, err


def test_caluu1(torus2d):
    _, o, r = torus2d
    u = o.prims()
    err = field_err(r.caluu1(u), o.caluu1(u))
    assert err.max() < TOL, err


@pytest.mark.parametrize("irec", [config.IREC_MP5, config.IREC_WENO5, config.IREC_PPM, config.IREC_MC,
                                  config.IREC_MINMOD, config.IREC_WENOZ, config.IREC_MUSCL, config.IREC_LIMO3,
                                  config.IREC_MVL, config.IREC_KOREN, config.IREC_WENOM, config.IREC_MPWENO,
                                  config.IREC_CENO])
def test_calflx_guarded(gpu_ctx, irec):
    p = config.torus(nr=48, nth=40, nph=12, irec=irec)
    p["guard"] = 1
    o, r = _pair(gpu_ctx, p, seed=5)
    u = o.prims()
    wg, wo = r.calflx(u), o.fluxes(u)
    r.release()
    n = o.nm1 - 1  # inside the hll range nm0 .. n-nm0 (1-based)
    reg = (slice(n, -n), slice(n, -n), slice(n, -n))
    err = flux_err(wg[reg], wo[reg])
    assert err.max() < TOL, np.unravel_index(err.argmax(), err.shape)


def test_calflx_reference_semantics_nan_pattern(gpu_ctx):
    """guard = 0: both paths produce the same non-finite entropy fluxes and
    agree everywhere else."""
    p = config.torus(nr=48, nth=40, nph=10)
    o, r = _pair(gpu_ctx, p, seed=5)
    u = o.prims()
    wg, wo = r.calflx(u), o.fluxes(u)
    r.release()
    n = o.nm1 - 1
    reg = (slice(n, -n), slice(n, -n), slice(n, -n))
    a, b = wg[reg], wo[reg]
    assert np.array_equal(np.isfinite(a), np.isfinite(b))
    assert (~np.isfinite(b)).any()
    err = flux_err(a, b)
    assert err.max() < TOL, np.unravel_index(err.argmax(), err.shape)


def test_recov(torus3d):
    p, o, r = torus3d
    u = o.prims()
    rng = np.random.default_rng(0)
    uu = o.caluu1(u)
    n = o.nm1
    pert = uu.copy()
    pert[n:-n, n:-n, n:-n, :5] *= 1 + 1e-3 * rng.standard_normal(pert[n:-n, n:-n, n:-n, :5].shape)
    _, want = o.recov(pert, u)
    got = r.recov(pert, u)
    err = field_err(got, want, (slice(n, -n), slice(n, -n), slice(n, -n)))
    assert err[[0, 1, 2, 3, 4, 6, 7, 8]].max() < TOL, err


def test_calsf(torus3d):
    """caltenr + calsf on every cell (ghosts included, the reference's loop
    range), relative to the largest source component: S_t and S_phi vanish in
    exact arithmetic for a stationary axisymmetric metric, so both sides hold
    cancellation residue there and are compared at the scale of S_r."""
    _, o, r = torus3d
    u = o.prims()
    got, want = r.calsf(u), o.calsf(u)
    assert np.isfinite(got).all()
    err = np.abs(got - want).max(axis=(0, 1, 2)) / np.abs(want).max()
    assert err.max() < TOL, err


@pytest.mark.parametrize("stage", [1, 2, 3])
def test_rkt(torus3d, stage):
    """One RK3 stage of rkt.f90 from the oracle's own fluxes and sources:
    interior cells against the oracle, the other cells untouched."""
    _, o, r = torus3d
    u = o.prims()
    rng = np.random.default_rng(stage)
    ww = o.fluxes(u)
    sf = o.calsf(u)
    ucur = o.caluu1(u)
    uo = ucur * (1 + 1e-3 * rng.standard_normal(ucur.shape)) if stage > 1 else None
    unew = rng.standard_normal(ucur.shape)
    dt = 0.4 * o.cdtcfl(u)
    got = r.rkt(stage, dt, ww, uo, ucur, sf, unew)
    want = o.rkt(stage, dt, ww, uo, ucur, sf, unew)
    n = o.nm1
    inner = (slice(n, -n), slice(n, -n), slice(n, -n))
    err = field_err(got, want, inner)
    assert err.max() < TOL, err
    outside = np.ones(got.shape[:3], dtype=bool)
    outside[inner] = False
    assert np.array_equal(got[outside], unew[outside])


def _derived_err(got, want):
    assert np.array_equal(np.isfinite(got), np.isfinite(want))
    fin = np.isfinite(want)
    scale = np.abs(np.where(fin, want, 0)).reshape(-1, 7).max(axis=0)
    diff = np.abs(np.where(fin, got - want, 0)).reshape(-1, 7).max(axis=0)
    return diff / np.maximum(scale, 1e-300)


@pytest.mark.parametrize("case", ["torus3d", "torus2d"])
def test_derived_matches_oracle(case, request):
    """The converter's derived quantities on the device (every cell and the
    meridional cut) against the oracle; NaN (static observer inside the
    ergosphere) at the same cells.  The 2D run stores its phi slab as one
    plane and answers for every phi index."""
    p, o, r = request.getfixturevalue(case)
    u = o.prims()
    r.upload_prims(u)
    got, want = r.derived(), o.derived(u)
    err = _derived_err(got, want)
    assert err.max() < TOL, err
    j = p["jmax"] // 2 + 1
    assert np.array_equal(r.derived(jslice=j), got[:, j - 1], equal_nan=True)


def test_cdtcfl(torus3d):
    _, o, r = torus3d
    u = o.prims()
    assert r.cdtcfl(u) == pytest.approx(o.cdtcfl(u), rel=TOL)


def test_bnd_floor(torus3d):
    _, o, r = torus3d
    u = o.prims()
    rng = np.random.default_rng(1)
    v = u * (1 + 1e-2 * rng.standard_normal(u.shape))
    v[..., 0] = np.abs(v[..., 0])
    err = field_err(r.bnd_floor(v, u), o.bnd_floor(v, u))
    assert err.max() < TOL, err


def _step_err(gpu_ctx, p, steps, seed):
    o = Oracle(p)
    o.ic_torus(seed=seed)
    r = gpu_ctx.admit(p)
    r.upload_prims(o.prims())
    o.init_cons()
    errs = []
    for _ in range(steps):
        o.step(1)
        st = r.step(1, stats=True)
        errs.append(field_err(r.prims(), o.prims()).max())
        r.upload_prims(o.prims(), t0=o.time)  # per-step bound: restart both from the oracle state
    r.release()
    return np.array(errs), st


def test_step_2d_mp5(gpu_ctx):
    p = dict(config.torus(nr=64, nth=64), guard=1)
    errs, _ = _step_err(gpu_ctx, p, 3, seed=2012)
    assert errs.max() < TOL, errs


def test_step_3d_mp5(gpu_ctx):
    p = dict(config.torus(nr=40, nth=24, nph=16), guard=1)
    errs, _ = _step_err(gpu_ctx, p, 2, seed=77)
    assert errs.max() < TOL, errs


def test_step_benchmark_grids(gpu_ctx):
    """One step on the benchmark's own grids, MP5 with the positivity
    fallback: the 3D torus 256x128x128 (the headline, 3.57 M interior cells)
    and the 2D torus 256x256 (phi slab), within 1e-12 of each field's
    maximum."""
    for p in (dict(config.torus(nr=256, nth=128, nph=128), guard=1), dict(config.torus(nr=256, nth=256), guard=1)):
        errs, st = _step_err(gpu_ctx, p, 1, seed=2012)
        assert errs.max() < TOL, (p["imax"], p["jmax"], p["kmax"], errs)
        assert st["steps"] == 1


def test_step_3d_weno5(gpu_ctx):
    p = dict(config.torus(nr=40, nth=24, nph=16, irec=config.IREC_WENO5), guard=1)
    errs, _ = _step_err(gpu_ctx, p, 2, seed=78)
    assert errs.max() < TOL, errs


def _vector_scaled_err(a, b):
    """Per-variable max |a-b| relative to the largest value of its quantity:
    the three velocity components share one scale, as do the three field
    components (a small component such as u^theta carries round-off of the
    size of the momentum fluxes that produce it)."""
    a = a.reshape(-1, 9)
    b = b.reshape(-1, 9)
    mx = np.abs(b).max(axis=0)
    scale = mx.copy()
    scale[1:4] = mx[1:4].max()
    scale[6:9] = mx[6:9].max()
    return np.abs(a - b).max(axis=0) / np.maximum(scale, 1e-300)


@pytest.mark.parametrize("irec", [config.IREC_MC, config.IREC_MINMOD, config.IREC_WENOZ, config.IREC_MUSCL,
                                  config.IREC_LIMO3, config.IREC_MVL, config.IREC_KOREN, config.IREC_WENOM,
                                  config.IREC_MPWENO, config.IREC_CENO])
def test_step_3d_limiters_and_wenoz(gpu_ctx, irec):
    """MC, minmod, MUSCL, LimO3, MVL, Koren (rec.f90:145-739, 4037-4697),
    WENO-Z (rec.f90:3161-3436) and WENO-M (rec.f90:3439-3793): one full step
    per comparison, 3D torus, 1e-12 of each quantity's scale."""
    p = dict(config.torus(nr=40, nth=24, nph=16, irec=irec), guard=1)
    o = Oracle(p)
    o.ic_torus(seed=80 + irec)
    r = gpu_ctx.admit(p)
    r.upload_prims(o.prims())
    o.init_cons()
    for _ in range(2):
        o.step(1)
        r.step(1)
        err = _vector_scaled_err(r.prims(), o.prims())
        assert err.max() < TOL, err
        r.upload_prims(o.prims(), t0=o.time)
    r.release()


def test_multistep_drift(gpu_ctx):
    """20 steps without re-synchronisation stay within a loose bound (round-off growth)."""
    p = dict(config.torus(nr=48, nth=48), guard=3)
    o = Oracle(p)
    o.ic_torus(seed=4)
    r = gpu_ctx.admit(p)
    r.upload_prims(o.prims())
    o.init_cons()
    o.step(20)
    st = r.step(20, stats=True)
    got = r.prims()
    r.release()
    assert st["steps"] == 20 and st["time"] == pytest.approx(o.time, rel=1e-12)
    n = o.nm1
    l1 = np.abs(got - o.prims())[n:-n, n:-n, n:-n].sum(axis=(0, 1, 2)) / np.abs(o.prims()[n:-n, n:-n, n:-n]).sum(axis=(0, 1, 2)).clip(1e-300)
    assert l1[[0, 4, 6, 8]].max() < 1e-10, l1


def test_step_3d_ppm_reference_semantics(gpu_ctx):
    """PPM needs no guard: reference semantics (guard = 0) stay finite."""
    p = config.torus(nr=40, nth=24, nph=16, irec=config.IREC_PPM)
    errs, st = _step_err(gpu_ctx, p, 2, seed=79)
    assert errs.max() < TOL, errs


def _l1(a, b, n):
    a, b = a[n:-n, n:-n, n:-n], b[n:-n, n:-n, n:-n]
    return np.abs(a - b).sum(axis=(0, 1, 2)) / np.abs(b).sum(axis=(0, 1, 2)).clip(1e-300)


@pytest.mark.parametrize("irec", [config.IREC_MP5, config.IREC_PPM])
def test_mixed_precision_tracks_fp64(gpu_ctx, irec):
    """FP32 reconstruction/fluxes/CT/RK combine (compensated) with FP64
    recovery and near-horizon metric: L1 density error vs the FP64 GPU run
    stays below the 1e-5 bound of the mixed path after 100 steps."""
    p = dict(config.torus(nr=48, nth=32, nph=16, irec=irec), guard=1)
    r64 = gpu_ctx.admit(p)
    r32 = gpu_ctx.admit(dict(p, precision="mixed"))
    r64.ic_torus(seed=31)
    r32.ic_torus(seed=31)
    s64 = r64.step(100, stats=True)
    s32 = r32.step(100, stats=True)
    a, b = r32.prims(), r64.prims()
    r64.release()
    r32.release()
    assert np.isfinite(a).all()
    assert s32["time"] == pytest.approx(s64["time"], rel=1e-5)
    l1 = _l1(a, b, config.ghost_widths(irec)[1])
    assert l1[0] < 1e-5, l1
    assert l1[[4, 6, 8]].max() < 1e-4, l1


def test_slab_2d_equals_full_compute(gpu_ctx):
    """The 2D phi slab (jmax = 2*nm1+1) is stored as one plane; stepping it
    gives the primitives of computing all jmax planes (RG_FLAG_FULL) to the
    per-step bound (the two are separately compiled kernels, so FMA
    contraction may differ in the last bit)."""
    p = dict(config.torus(nr=64, nth=48), guard=1)
    rs = gpu_ctx.admit(p)
    rf = gpu_ctx.admit(dict(p, flags=config.FLAG_FULL))
    rs.ic_torus(seed=11)
    rf.ic_torus(seed=11)
    ss = rs.step(5, stats=True)
    sf = rf.step(5, stats=True)
    a, b = rs.prims(), rf.prims()
    rs.release()
    rf.release()
    assert ss["time"] == pytest.approx(sf["time"], rel=1e-13)
    err = field_err(a, b)
    assert err.max() < 1e-12, err
    # every phi plane of the download is the stored plane
    assert (a == a[:, 4:5]).all()


def test_slab_rejects_nonuniform_upload(gpu_ctx):
    from raishinsource_b200.capi import RgError
    p = dict(config.torus(nr=40, nth=40), guard=1)
    o = Oracle(p)
    o.ic_torus(seed=3)
    u = o.prims()
    r = gpu_ctx.admit(p)
    r.upload_prims(u)  # uniform along phi: accepted
    u2 = u.copy()
    u2[:, 0, :, 0] *= 1.01  # one phi ghost plane differs
    with pytest.raises(RgError) as e:
        r.upload_prims(u2)
    r.release()
    assert e.value.code == 1


@pytest.mark.parametrize("irec", [config.IREC_PPM, config.IREC_WENO5, config.IREC_MC, config.IREC_WENOZ,
                                  config.IREC_KOREN, config.IREC_MPWENO])
def test_step_2d_slab_schemes(gpu_ctx, irec):
    """2D phi slab (stored as one plane; jmax = 2*nm1+1: 11 for PPM, 7 for MC)
    against the oracle, which computes every phi cell."""
    p = dict(config.torus(nr=56, nth=48, irec=irec), guard=1)
    errs, _ = _step_err(gpu_ctx, p, 2, seed=21)
    assert errs.max() < TOL, errs


def test_admission_refuses_oversize_footprint(gpu_ctx):
    """A run whose device footprint exceeds free memory is refused before any
    allocation (RG_ENOMEM_ADMIT)."""
    from raishinsource_b200.capi import RgError, footprint
    import torch
    free, _ = torch.cuda.mem_get_info()
    p = config.torus(nr=1536, nth=1024, nph=1024)
    assert footprint(p) > free
    with pytest.raises(RgError) as e:
        gpu_ctx.admit(p)
    assert e.value.code == 2


def test_thousand_steps_l1_ppm(gpu_ctx):
    """1000 steps without re-synchronisation (PPM, reference semantics, 2D
    torus 64x64): L1 of rho, p and B against the oracle stays below 1e-10."""
    p = config.torus(nr=64, nth=64, irec=config.IREC_PPM)
    o = Oracle(p)
    o.ic_torus(seed=4)
    o.init_cons()
    r = gpu_ctx.admit(p)
    r.upload_prims(o.prims())
    o.step(1000)
    st = r.step(1000, stats=True)
    got, want = r.prims(), o.prims()
    r.release()
    assert st["steps"] == 1000
    l1 = _l1(got, want, o.nm1)
    assert l1[[0, 4, 6, 7, 8]].max() < 1e-10, l1


def test_thousand_steps_l1_mp5_3d(gpu_ctx):
    """1000 steps of the product (FMA-contracted) build on the 40x24x16 3D
    torus, MP5 with the positivity fallback (the benchmark's scheme): L1 of
    rho, the internal energy (p) and B against the oracle stays below 1e-10.
    (The uncontracted build is bit-identical to the oracle over the same run,
    tests/test_gpu_exact.py.)"""
    p = dict(config.torus(nr=40, nth=24, nph=16), guard=1)
    o = Oracle(p)
    o.ic_torus(seed=2012)
    o.init_cons()
    r = gpu_ctx.admit(p)
    r.upload_prims(o.prims())
    o.step(1000)
    st = r.step(1000, stats=True)
    got, want = r.prims(), o.prims()
    r.release()
    assert st["steps"] == 1000
    l1 = _l1(got, want, o.nm1)
    assert l1[[0, 4, 6, 7, 8]].max() < 1e-10, l1


def test_per_routine_calls_leave_the_run_alone(gpu_ctx):
    """The reference-interface entry points compute on their own scratch
    state: calling them between steps of a run changes neither its result,
    its time, nor its statistics."""
    p = dict(config.torus(nr=40, nth=24, nph=16), guard=1)
    o = Oracle(p)
    o.ic_torus(seed=31)
    u = o.prims()
    a, b = gpu_ctx.admit(p), gpu_ctx.admit(p)
    a.upload_prims(u)
    b.upload_prims(u)
    a.step(1)
    b.step(1)
    cur = b.prims()
    b.calflx(cur)
    b.cdtcfl(cur)
    b.recov(b.caluu1(cur), cur)
    b.bnd_floor(cur, cur)
    b.calsf(cur)
    b.horizon_flux()
    b.derived()
    sa, sb = a.step(2, stats=True), b.step(2, stats=True)
    assert sa == sb
    assert np.array_equal(a.prims(), b.prims())
    a.release()
    b.release()


@pytest.mark.parametrize("ict", [0, 2, 3])
def test_constrained_transport_variants(gpu_ctx, ict):
    """ict = 0 (no CT), ict = 2 (mflct, ct.f90:121-233) and ict = 3 (upflct,
    ct.f90:236-445): fluxes through the C ABI and one full step per comparison
    against the oracle, 3D torus; ghost width nm1 = nm0 + ict."""
    p = dict(config.torus(nr=40, nth=28, nph=20, ict=ict), guard=1)
    o, r = _pair(gpu_ctx, p, seed=40 + ict)
    assert o.nm1 == 3 + ict
    u = o.prims()
    wg, wo = r.calflx(u), o.fluxes(u)
    n = o.nm1 - 1
    reg = (slice(n, -n), slice(n, -n), slice(n, -n))
    assert flux_err(wg[reg], wo[reg]).max() < TOL
    o.init_cons()
    for _ in range(2):
        o.step(1)
        r.step(1)
        err = _vector_scaled_err(r.prims(), o.prims())
        assert err.max() < TOL, err
        r.upload_prims(o.prims(), t0=o.time)
    r.release()


@pytest.mark.parametrize("ict", [2, 3])
def test_ct_variants_2d_slab(gpu_ctx, ict):
    """mflct and upflct on a 2D phi slab stored as one plane (mflct through the
    batched kernels, upflct through the single-run launches) against the
    oracle computing every phi cell."""
    p = dict(config.torus(nr=48, nth=40, ict=ict), guard=1)
    errs, _ = _step_err(gpu_ctx, p, 2, seed=23)
    assert errs.max() < TOL, errs


def test_kerr_schild_metric(gpu_ctx):
    """Metric 303 (Kerr-Schild on uniform r and theta grids): initial data,
    two steps against the oracle (including the cells whose W rescale loop
    hits its cap, counted alike in the first step) and the converter's derived
    quantities."""
    p = dict(config.torus(nr=48, nth=40, nph=12), metric=303, ix1=1, ix3=1, guard=1, xmax=30.0)
    o = Oracle(p)
    o.ic_torus(seed=3)
    r = gpu_ctx.admit(p)
    r.ic_torus(seed=3)
    assert field_err(r.prims(), o.prims()).max() < 1e-13
    o.init_cons()
    for n in range(2):
        o.step(1)
        st = r.step(1, stats=True, strict=False)
        if n == 0:
            ost = o.stats()
            assert (st["recov_cap"], st["recov_nr2"]) == (ost["recov_cap"], ost["recov_nr2"])
        err = _vector_scaled_err(r.prims(), o.prims())
        assert err.max() < TOL, err
        r.upload_prims(o.prims(), t0=o.time)
    u = o.prims()
    err = _derived_err(r.derived(), o.derived(u))
    assert err.max() < TOL, err
    r.release()


@pytest.mark.parametrize("nph", [16, None])
def test_recov2(gpu_ctx, nph):
    """recov2 (iwvec 2, recov.f90:1919-2456): two full steps (the reference's
    stage sequence: fluxes with CT, caluu1, calsf, rkt, recov2) per comparison
    on a 3D torus and on a 2D phi slab stored as one plane, with the oracle's
    count of cells that keep their primitives; then rg_recov on perturbed
    conserved variables (after the steps: the oracle's recov leaves its result
    in the oracle's state)."""
    p = dict(config.torus(nr=40, nth=28, nph=nph), guard=1, iwvec=2)
    o, r = _pair(gpu_ctx, p, seed=77)
    o.init_cons()
    for _ in range(2):
        o.step(1)
        st = r.step(1, stats=True, strict=False)
        err = _vector_scaled_err(r.prims(), o.prims())
        assert err.max() < TOL, err
        r.upload_prims(o.prims(), t0=o.time)
    assert st["recov_fail"] == o.stats()["recov_fail"]  # both counted over the two steps
    u = o.prims()
    n = o.nm1
    reg = (slice(n, -n), slice(n, -n), slice(n, -n))
    uu = o.caluu1(u)
    pert = uu.copy()
    rng = np.random.default_rng(1)
    pert[n:-n, n:-n, n:-n, :5] *= 1 + 1e-3 * rng.standard_normal(pert[n:-n, n:-n, n:-n, :5].shape)
    got = r.recov(pert, u)
    _, want = o.recov(pert, u)
    err = field_err(got, want, reg)
    assert err[[0, 1, 2, 3, 4, 6, 7, 8]].max() < TOL, err
    r.release()


def _hll_region(o):
    """Slices (k, j, i) of the hll range nm0..n-nm0 (1-based) in every direction."""
    m = o.nm1 - o.params.get("ict", 1) - 1  # nm0 - 1
    return (slice(m, -(m + 1)),) * 3


def _rel(a, b, axis):
    """max |a-b| relative to the largest |b| of the same variable over all six
    face arrays (a component that vanishes in exact arithmetic on one face
    carries the round-off residue of the others' size)."""
    axis = (0,) + tuple(axis)
    scale = np.maximum(np.abs(b).max(axis=axis), 1e-300)
    return (np.abs(a - b).max(axis=axis) / scale).max()


@pytest.mark.parametrize("irec,guard", [(config.IREC_MP5, 1), (config.IREC_MP5, 3), (config.IREC_PPM, 0),
                                        (config.IREC_WENO5, 1), (config.IREC_MC, 1)])
def test_rec2_calcha_hll_ct_one_at_a_time(gpu_ctx, irec, guard):
    """rg_rec2, rg_calcha, rg_hll and rg_ct, each fed the oracle's inputs,
    against the oracle's rec2 (with caluu3/calflx3), calcha, hll and ct on the
    hll range; chained on the device they give rg_calflx's fluxes."""
    p = dict(config.torus(nr=48, nth=40, nph=12, irec=irec), guard=guard)
    o, r = _pair(gpu_ctx, p, seed=19)
    u = o.prims()
    reg = (slice(None),) + _hll_region(o)
    fo = o.rec2_full(u)
    fd = r.rec2(u)
    for a, b in zip(fd, fo):  # face primitives, conserved variables, fluxes
        assert _rel(a[reg], b[reg], (1, 2, 3)) < TOL
    cho = o.calcha(fo[0])
    chd = r.calcha(fo[0])
    assert _rel(chd[reg], cho[reg], (1, 2, 3)) < TOL
    ww0 = np.random.default_rng(3).standard_normal(u.shape + (3,))
    wo = o.hll(fo[1], fo[2], cho, ww0)
    wd = r.hll(fo[1], fo[2], cho, ww0)
    assert flux_err(wd, wo).max() < TOL
    co, cd = o.ct(u, wo), r.ct(u, wo)
    assert flux_err(cd, co).max() < TOL
    # the device chain equals the fused call
    chain = r.ct(u, r.hll(fd[1], fd[2], r.calcha(fd[0]), ww0))
    fused = r.calflx(u)
    n = o.nm1 - 1
    sl = (slice(n, -n),) * 3
    assert flux_err(chain[sl], fused[sl]).max() < TOL
    r.release()


def test_per_routine_entry_points_take_device_arrays(gpu_ctx):
    """The reference-interface entry points accept device pointers in place
    of host arrays (cudaMemcpyDefault): a driver that keeps its arrays on the
    GPU gets the same results without host copies."""
    import torch

    from raishinsource_b200.capi import _check
    p = dict(config.torus(nr=40, nth=32, nph=12), guard=1)
    o, r = _pair(gpu_ctx, p, seed=23)
    u = o.prims()
    lib, h, rid = r.lib, gpu_ctx.h, r.id
    du = torch.from_numpy(u).cuda()

    def dev(shape):
        return torch.zeros(shape, dtype=torch.float64, device="cuda")

    uu = dev(u.shape)
    _check(lib, lib.rg_caluu1(h, rid, ctypes_ptr(du), ctypes_ptr(uu)))
    assert np.array_equal(uu.cpu().numpy(), r.caluu1(u))
    ww = dev(u.shape + (3,))
    _check(lib, lib.rg_calflx(h, rid, ctypes_ptr(du), ctypes_ptr(ww)))
    assert np.array_equal(ww.cpu().numpy(), r.calflx(u))
    fp = dev((6,) + u.shape)
    _check(lib, lib.rg_rec2(h, rid, du.data_ptr(), fp.data_ptr(), None, None))
    assert np.array_equal(fp.cpu().numpy(), r.rec2(u, cons=False)[0])
    sf = dev(u.shape[:3] + (4,))
    _check(lib, lib.rg_calsf(h, rid, ctypes_ptr(du), ctypes_ptr(sf)))
    assert np.array_equal(sf.cpu().numpy(), r.calsf(u))
    r.release()


def ctypes_ptr(t):
    import ctypes
    return ctypes.cast(t.data_ptr(), ctypes.POINTER(ctypes.c_double))


@pytest.mark.parametrize("which", ["bnd4", "infchk", "atmosphere1a", "pminmax2b"])
def test_bnd4_and_floors_one_at_a_time(torus3d, which):
    """bnd4, infchk, atmosphere1a and pminmax2b as separate calls (main.f90:860-878)
    on a perturbed state that triggers the floors, against the oracle's routines."""
    _, o, r = torus3d
    u = o.prims()
    rng = np.random.default_rng(11)
    pert = u.copy()
    pert[..., 0] *= np.exp(rng.uniform(-4.0, 0.5, pert.shape[:3]))  # densities below the floor, some
    pert[..., 1:4] *= 1 + 3 * rng.standard_normal(pert.shape[:3] + (3,))
    urio = u
    got = r.bnd_part(which, pert, urio)
    want = o.bnd_part(which, pert, urio if which == "bnd4" else None)
    assert np.isfinite(got).all()
    err = field_err(got, want)
    assert err[[0, 1, 2, 3, 4, 6, 7, 8]].max() < TOL, err
    assert not np.array_equal(want, pert) or which == "infchk"
