"""CPU checks of the oracle (the C++ restatement of the reference).

The reference ships no golden vectors, so the oracle is checked against
properties the reference's own formulas imply: the LU inverse of the metric,
exact prim -> conserved -> prim round trips through recov1a, flux-CT keeping
the corner-centred divergence of B at round-off, the positivity guard being a
no-op where no face state is negative, and thread-count independence.
"""
import numpy as np
import pytest

from conftest import field_err
from oracle import Oracle
from raishinsource_b200 import config


@pytest.fixture(scope="module")
def torus_small():
    p = config.torus(nr=48, nth=48, irec=config.IREC_MP5)
    p["guard"] = 1
    o = Oracle(p)
    o.ic_torus(seed=7)
    return p, o


def test_metric_inverse_and_detg(torus_small):
    _, o = torus_small
    for loc in ("", "i", "k"):
        g = o.array("gcov" + loc).reshape(-1, 4, 4)
        gc = o.array("gcon" + loc).reshape(-1, 4, 4)
        err = np.abs(np.einsum("qab,qbc->qac", g, gc) - np.eye(4)).max()
        assert err < 1e-13, loc
        detg = o.array("detg" + loc)
        assert np.all(detg > 0)
        assert np.allclose(detg, np.sqrt(-np.linalg.det(g)), rtol=1e-12)


def test_grid_matches_reference_formulas(torus_small):
    p, o = torus_small
    x1 = o.array("x1")
    assert x1[0] == pytest.approx(p["xmin"], rel=1e-14)
    # grid.f90:37 scales by the single-precision 1./float(imax-1): r_out misses xmax at 1e-7
    assert x1[-1] == pytest.approx(p["xmax"], rel=1e-6) and x1[-1] != p["xmax"]
    x1b = o.array("x1b")
    assert np.allclose(np.diff(x1b), np.diff(x1b)[0], rtol=1e-6)  # uniform in log r (MKS)
    x3b = o.array("x3b")
    assert x3b[0] == pytest.approx(0.02, rel=1e-14)
    assert x3b[-1] == pytest.approx(np.pi - 0.02, rel=1e-12)


def test_torus_ic_physical(torus_small):
    p, o = torus_small
    u = o.prims()
    assert np.isfinite(u).all()
    assert u[..., 0].max() == pytest.approx(1.0, rel=0.05)
    assert (u[..., 0] > 0).all() and (u[..., 4] > 0).all()
    assert np.abs(u[..., 6:]).max() > 0


def test_recov_round_trip_is_exact(torus_small):
    _, o = torus_small
    u = o.prims()
    uu = o.caluu1(u)
    _, u2 = o.recov(uu, u)
    n = o.nm1
    err = field_err(u2, u, (slice(n, -n), slice(n, -n), slice(n, -n)))
    assert err[[0, 1, 2, 4, 6, 7, 8]].max() < 1e-12, err
    assert o.stats()["recov_nr2"] == 0


def corner_divb(u, o):
    """Toth's corner-centred div(sqrt(-g) B) in the (r, theta) plane (2D, j-invariant)."""
    detg = o.array("detg").reshape(o.params["kmax"], o.params["imax"])
    dx1 = o.array("dx1b")[1]
    dx3 = o.array("dx3b")[1]
    j = o.params["jmax"] // 2
    b1 = detg * u[:, j, :, 6]
    b3 = detg * u[:, j, :, 8]
    d1 = (b1[1:, 1:] + b1[:-1, 1:] - b1[1:, :-1] - b1[:-1, :-1]) / (2 * dx1)
    d3 = (b3[1:, 1:] + b3[1:, :-1] - b3[:-1, 1:] - b3[:-1, :-1]) / (2 * dx3)
    return d1 + d3


def _divb_drift(guard):
    p = config.torus(nr=40, nth=40)
    o = Oracle(dict(p, guard=guard))
    o.ic_torus(seed=3, amp=0.0)  # phi-uniform data: the 2D corner divergence is the full one
    o.init_cons()
    n = o.nm1
    d0 = corner_divb(o.prims(), o)[n:-n, n:-n]
    o.step(3)
    d1 = corner_divb(o.prims(), o)[n:-n, n:-n]
    bscale = np.abs(o.prims()[..., 6:]).max() / o.array("dx1b")[1]
    return np.abs(d1 - d0).max() / bscale


def test_fluxct_preserves_divb_with_zero_normal_flux():
    """Toth's flux-CT (ct.f90:30-118) keeps the corner divergence at round-off
    once the normal-component flux is zero (guard bit 2)."""
    assert _divb_drift(guard=3) < 1e-11


def test_reference_llf_normal_flux_breaks_divb():
    """Reference semantics: hll.f90 leaves the LLF diffusion of B^d in ww(d,6+d),
    which ct does not replace, so the divergence drifts at O(1e-1)."""
    assert _divb_drift(guard=1) > 1e-3


def test_guard_is_noop_for_ppm():
    p = config.torus(nr=32, nth=32, irec=config.IREC_PPM)
    outs = []
    for g in (0, 1):
        q = dict(p, guard=g)
        o = Oracle(q)
        o.ic_torus(seed=11)
        o.init_cons()
        o.step(2)
        outs.append(o.prims())
    assert np.array_equal(outs[0], outs[1])


def test_mp5_faithful_reference_goes_nonfinite_guarded_does_not():
    """Reference semantics: MP5's absolute switch leaves floor-level density
    unlimited, face rho < 0, and de**gam turns the entropy flux NaN."""
    p = config.torus(nr=40, nth=40)
    o = Oracle(dict(p, guard=0))
    o.ic_torus(seed=5)
    ww = o.fluxes(o.prims())
    assert not np.isfinite(ww[..., 5, :]).all()
    og = Oracle(dict(p, guard=1))
    og.ic_torus(seed=5)
    og.init_cons()
    og.step(5)
    assert np.isfinite(og.prims()).all()


def test_thread_count_independence(monkeypatch):
    """OpenMP over k does not change a single bit (recov's loop-order carry included)."""
    import subprocess
    import sys
    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "import numpy as np\n"
        "from oracle import Oracle\n"
        "from raishinsource_b200 import config\n"
        "p = config.torus(nr=32, nth=32); p['guard'] = 1\n"
        "o = Oracle(p); o.ic_torus(seed=9); o.init_cons(); o.step(2)\n"
        "sys.stdout.buffer.write(o.prims().tobytes())\n"
    )
    from conftest import ROOT
    outs = []
    for nt in ("1", "4"):
        env = dict(__import__("os").environ, OMP_NUM_THREADS=nt)
        r = subprocess.run([sys.executable, "-c", code % ROOT], capture_output=True, env=env, check=True)
        outs.append(r.stdout)
    assert outs[0] == outs[1]


def test_periodic_transverse_corners_stay_stale():
    """With periodic boundaries in both transverse directions of a 1D tube,
    the single-rank periodic fill (bnd.f90:50-70, 160-180, 272-292) covers
    only columns whose transverse indices are interior, so the cells that are
    ghosts in both directions keep their old values; with copy boundaries
    (the tube setup used here) every transverse cell equals the interior one."""
    from raishinsource_b200 import config as cfg
    p = cfg.tube(n=60)
    per = dict(p, ibc=[[5] * 9, [5] * 9, [1] * 9, [1] * 9, [1] * 9, [1] * 9])
    for params, uniform in ((per, False), (p, True)):
        o = Oracle(params)
        o.ic_tube(seed=3, tube=1)
        ic = o.prims()
        o.init_cons()
        o.step(2)
        u = o.prims()  # (k, j, i, v)
        line = u[4, 4]
        same = all(np.array_equal(u[k, j], line) for k in range(9) for j in range(9))
        assert same == uniform
        if not uniform:
            # a corner ghost (j and k both ghosts) still holds the initial data
            assert np.array_equal(u[0, 0], ic[0, 0]) and not np.array_equal(line, ic[4, 4])


def test_rkt_stage_combinations_and_literals(torus_small):
    """rkt.f90 with zero fluxes and sources: stage 1 returns uu, stage 2
    (3 uo + uh)/4, stage 3 (uo + 2 us) times the single-precision (1./3.)
    (rkt.f90:169); cells outside the interior keep unew."""
    _, o = torus_small
    rng = np.random.default_rng(3)
    shape = o.prims().shape
    ww = np.zeros(shape + (3,))
    sf = np.zeros(shape[:3] + (4,))
    uo, uc, unew = (rng.standard_normal(shape) for _ in range(3))
    n = o.nm1
    inner = (slice(n, -n), slice(n, -n), slice(n, -n))
    third = float(np.float32(1.0) / np.float32(3.0))
    want = {1: uc, 2: (3.0 * uo + uc) * 0.25, 3: (uo + 2.0 * uc) * third}
    for stage in (1, 2, 3):
        got = o.rkt(stage, 0.1, ww, uo, uc, sf, unew)
        assert np.array_equal(got[inner], want[stage][inner])
        outside = np.ones(shape[:3], dtype=bool)
        outside[inner] = False
        assert np.array_equal(got[outside], unew[outside])


def test_calsf_covers_every_cell(torus_small):
    """caltenr + calsf run over the reference's whole loop range (calsf.f90:121-123):
    the ghost cells get finite, nonzero sources too."""
    _, o = torus_small
    sf = o.calsf(o.prims())
    assert np.isfinite(sf).all()
    n = o.nm1
    ghosts = np.ones(sf.shape[:3], dtype=bool)
    ghosts[n:-n, n:-n, n:-n] = False
    assert (np.abs(sf[ghosts]).max(axis=1) > 0).mean() > 0.5


def _face_check(o, u, faces, expect, lo):
    """Compare the six face-state arrays of rec2 with expect(d, m) (the exact
    face value of direction d at stored index m, broadcast over the grid):
    left states at m in lo+1..n-lo, right states at m in lo..n-lo-1 (1-based),
    over the cells the reconstruction loop covers in the other directions."""
    worst = 0.0
    for d in range(3):
        ax = 2 - d  # numpy axis of direction d in (k, j, i, v)
        for side, shift in ((0, 1), (1, 0)):
            got = np.moveaxis(faces[2 * d + side], ax, 0)
            want = np.moveaxis(expect(d), ax, 0)
            sl = [slice(lo, -lo)] * 3
            sl[0] = slice(lo - 1 + shift, got.shape[0] - lo - 1 + shift)
            g, w = got[tuple(sl)], want[tuple(sl)]
            worst = max(worst, float(np.abs(g - w).max() / np.abs(w).max()))
    return worst


@pytest.mark.parametrize("irec", [config.IREC_MC, config.IREC_MINMOD, config.IREC_LIMO3, config.IREC_MVL,
                                  config.IREC_KOREN])
def test_slope_limiters_reproduce_linear_data(irec):
    """The second-order limiters (rec.f90:208-739, 4037-4697) return the face
    value of increasing data linear in the reconstruction coordinate (MKS x?b,
    faces at x?ab) up to the 1e-12 regulariser of the spacing."""
    p = config.torus(nr=24, nth=20, nph=14, irec=irec)
    o = Oracle(p)
    xb = [o.array("x1b"), o.array("x2b"), o.array("x3b")]
    xab = [o.array("x1ab"), o.array("x2ab"), o.array("x3ab")]
    coef = [0.5, 0.25, 0.125]

    def field(xs):
        k, j, i = np.meshgrid(xs[2], xs[1], xs[0], indexing="ij")
        return 1.0 + coef[0] * i + coef[1] * j + coef[2] * k

    u = np.repeat(field(xb)[..., None], 9, axis=3) * (1.0 + 0.1 * np.arange(9))
    faces = o.rec2(u)

    def expect(d):
        xs = list(xb)
        xs[d] = xab[d]
        return np.repeat(field(xs)[..., None], 9, axis=3) * (1.0 + 0.1 * np.arange(9))

    assert _face_check(o, u, faces, expect, lo=1) < 1e-9


@pytest.mark.parametrize("irec", [config.IREC_WENO5, config.IREC_WENOZ, config.IREC_WENOM, config.IREC_MPWENO])
def test_weno_reproduces_linear_data(irec):
    """WENO5, WENO-Z, WENO-M and MP-WENO are exact for data linear in the cell
    index (every candidate stencil is, the weights sum to one, and MP5's bounds
    hold the linear value)."""
    p = config.torus(nr=24, nth=20, nph=14, irec=irec)
    o = Oracle(p)
    shape = o.prims().shape
    k, j, i = np.meshgrid(*(np.arange(1, n + 1, dtype=float) for n in shape[:3]), indexing="ij")
    lin = 1.0 + 0.01 * i + 0.02 * j + 0.03 * k
    u = np.repeat(lin[..., None], 9, axis=3)
    faces = o.rec2(u)
    step = [0.01, 0.02, 0.03]

    def expect(d):
        return np.repeat((lin + 0.5 * step[d])[..., None], 9, axis=3)

    assert _face_check(o, u, faces, expect, lo=2) < 1e-13


def test_derived_quantities_sane_and_slice_consistent(torus_small):
    """The converter's derived quantities: the ZAMO Lorentz factor >= 1 and
    b^2 >= 0 everywhere; the static-observer factor u^t sqrt(-g_tt) is NaN
    exactly where no static observer exists (inside the ergosphere, g_tt > 0
    in Boyer-Lindquist coordinates), as in the converter; the phi-plane cut
    equals that plane of the full array."""
    p, o = torus_small
    u = o.prims()
    full = o.derived(u)
    fields = [0, 2, 3, 4, 5, 6]
    assert np.isfinite(full[..., fields]).all()
    assert (full[..., 0] >= 1.0 - 1e-12).all()
    assert (full[..., 2] >= 0.0).all()
    r = o.array("x1b")
    th = o.array("x3b")
    th = th + 0.5 * (1.0 - p["hslope"]) * np.sin(2.0 * th)
    rr = p["R0"] + np.exp(r)
    a = p["akm"]
    sig = rr[None, :] ** 2 + (a * np.cos(th)[:, None]) ** 2
    ergo = (sig - 2.0 * rr[None, :]) < 0  # (k, i): g_tt > 0
    rh = 1.0 + np.sqrt(1.0 - a * a)
    ergo &= rr[None, :] > rh
    nan = ~np.isfinite(full[..., 1])
    assert np.array_equal(nan, np.broadcast_to(ergo[:, None, :], nan.shape))
    j = p["jmax"] // 2 + 1
    np.testing.assert_array_equal(o.derived(u, jslice=j), full[:, j - 1])


def test_limo3_drops_the_slope_sign():
    """lim03a's dk2fi/dk2bi are max(0, ...) without the sign factor tmp2i that
    every other limiter applies (rec.f90:4122-4134), so a decreasing linear
    profile gets its left face value on the increasing side: u + |s| h."""
    p = config.torus(nr=24, nth=20, nph=14, irec=config.IREC_LIMO3)
    o = Oracle(p)
    shape = o.prims().shape
    x1b, x1ab = o.array("x1b"), o.array("x1ab")
    u = np.repeat((5.0 - 0.5 * x1b)[None, None, :, None], 9, axis=3) * np.ones(shape)
    uil = o.rec2(u)[0]
    i = np.arange(2, shape[2] - 1)  # 1-based cells 3..n-1 -> zero-based 2..n-2
    got = uil[5, 5, i, 0]
    slope = 0.5 * (x1b[i + 1] - x1b[i]) / (x1b[i + 1] - x1b[i] + 1e-12)
    want = u[5, 5, i, 0] + slope * (x1ab[i] - x1b[i])
    np.testing.assert_allclose(got, want, rtol=1e-12)


def test_muscl_reproduces_linear_data():
    """MUSCL (rec.f90:145-205) is exact for data linear in the cell index; both
    face states are stored at the face's left cell m = 2..n-2."""
    p = config.torus(nr=24, nth=20, nph=14, irec=config.IREC_MUSCL)
    o = Oracle(p)
    shape = o.prims().shape
    k, j, i = np.meshgrid(*(np.arange(1, n + 1, dtype=float) for n in shape[:3]), indexing="ij")
    step = [0.01, 0.02, 0.03]
    lin = 1.0 + step[0] * i + step[1] * j + step[2] * k
    faces = o.rec2(np.repeat(lin[..., None], 9, axis=3))
    reg = (slice(1, -2),) * 3
    for d in range(3):
        want = (lin + 0.5 * step[d])[reg]
        for side in range(2):
            got = faces[2 * d + side][reg][..., 0]
            assert np.abs(got - want).max() < 1e-14 * np.abs(want).max()


def test_mpweno_radial_right_state_reads_i_minus_11():
    """mpweno5's radial right state takes beta_1 from uri(n,i-11,j,k)
    (rec.f90:2757): changing only that far cell (and nothing within the
    5-point stencil) changes the right states that read it, and no others."""
    p = config.torus(nr=32, nth=20, nph=14, irec=config.IREC_MPWENO)
    o = Oracle(p)
    shape = o.prims().shape
    k, j, i = np.meshgrid(*(np.arange(1, n + 1, dtype=float) for n in shape[:3]), indexing="ij")
    smooth = 1.0 + 0.1 * np.sin(0.4 * i) + 0.05 * np.cos(0.3 * j) + 0.02 * np.sin(0.2 * k)
    u = np.repeat(smooth[..., None], 9, axis=3)  # smooth: MP5's bounds leave the WENO value
    base = o.rec2(u)
    v = u.copy()
    v[6, 6, 4, 0] += 0.5          # cell (i=5, j=7, k=7), 1-based
    changed = np.argwhere(o.rec2(v)[1][..., 0] != base[1][..., 0])
    # uriir(i-1) of cells i = 16 (5 + 11) in the same row: stored at i = 15,
    # plus the ordinary stencil neighbours of cell 5 (stored at i = 2..6)
    rows = {tuple(c[:2]) for c in changed}
    assert rows == {(6, 6)}, rows
    assert 14 in set(changed[:, 2])  # zero-based i of stored index 15



def test_christoffel_table_is_symmetric_in_its_lower_indices(torus_small):
    """Gamma^l_{mn} is stored at l + 4m + 16n; the geometry builds it from a
    symmetric metric, so the table is symmetric in (m, n) bit for bit, which
    the device's source term relies on to load each pair once."""
    _, o = torus_small
    c = o.array("christ").reshape(-1, 4, 4, 4)  # [point][n][m][l]
    assert np.array_equal(c, np.swapaxes(c, 1, 2))


def _ct_case(ict, seed=5):
    p = config.torus(nr=24, nth=20, nph=18, ict=ict)
    o = Oracle(p)
    rng = np.random.default_rng(seed)
    return p, o, rng


def test_ct_variants_agree_on_uniform_fluxes():
    """Face fluxes constant in space: flux-CT, mflct and upflct all give
    ww(2,7) = (fyx - fxy)/2 and its five companions on their ranges (every
    EMF difference of the upwind scheme vanishes, whatever the velocity)."""
    out = {}
    for ict in (1, 2, 3):
        p, o, rng = _ct_case(ict)
        f = np.random.default_rng(1).uniform(-1, 1, 6)
        ww = np.zeros(o.shape + (3,))
        for (d, n), v in zip([(2, 7), (3, 7), (1, 8), (3, 8), (1, 9), (2, 9)], f):
            ww[..., n - 1, d - 1] = v
        uri = rng.uniform(-1, 1, o.shape)  # velocities of both signs
        w = o.ct(uri, ww)
        n = o.nm1  # 1-based range nm1..n-nm1
        reg = w[n - 1:-n, n - 1:-n, n - 1:-n]
        fyx, fzx, fxy, fzy, fxz, fyz = f
        want = {(2, 7): (fyx - fxy) / 2, (3, 7): (fzx - fxz) / 2, (1, 8): (fxy - fyx) / 2,
                (3, 8): (fzy - fyz) / 2, (1, 9): (fxz - fzx) / 2, (2, 9): (fyz - fzy) / 2}
        for (d, m), v in want.items():
            assert np.allclose(reg[..., m - 1, d - 1], v, rtol=0, atol=1e-15), (ict, d, m)
        out[ict] = reg
    assert out[1].shape != out[3].shape  # nm1 = nm0 + ict


def test_upflct_upwinding_falls_back_on_the_radial_velocity():
    """upflct's else-if branches after the first EMF test uri(2) (ct.f90:357-387):
    with u^r = 0 a negative u^phi or u^theta selects the same averaged
    branch as a zero one, while a positive one selects the upwind value."""
    p, o, rng = _ct_case(3)
    ww = rng.uniform(-1, 1, o.shape + (3,))
    base = np.zeros(o.shape)
    base[..., 0] = 1.0
    def run(u2, u3):
        uri = base.copy()
        uri[..., 2] = u2
        uri[..., 3] = u3
        return o.ct(uri, ww.copy())
    zero, neg, pos = run(0.0, 0.0), run(-1.0, -1.0), run(1.0, 1.0)
    n = o.nm1
    reg = (slice(n - 1, -n), slice(n - 1, -n), slice(n - 1, -n))
    assert np.array_equal(zero[reg], neg[reg])
    assert not np.allclose(zero[reg], pos[reg])


def test_recov2_recovers_the_primitives_of_their_conserved_variables():
    """recov2 (iwvec 2, recov.f90:1919-2456) applied to caluu1 of a torus state,
    starting from perturbed guesses, returns that state wherever its
    one-variable Newton-Raphson converges (W' to 1e-8), as recov1a does."""
    p = dict(config.torus(nr=48, nth=40), iwvec=2)
    o = Oracle(p)
    o.ic_torus(seed=8)
    q = o.prims()
    u = o.caluu1(q)
    guess = q.copy()
    rng = np.random.default_rng(3)
    guess[..., 1:5] *= 1.0 + 0.01 * rng.uniform(-1, 1, guess[..., 1:5].shape)
    _, got = o.recov(u, guess)
    n = o.nm1
    reg = (slice(n, -n), slice(n, -n), slice(n, -n))
    st = o.stats()
    assert st["recov_fail"] == 0 and st["recov_cap"] == 0
    rel = np.abs(got[reg] - q[reg])[..., [0, 4]] / np.abs(q[reg])[..., [0, 4]]
    assert np.median(rel) < 1e-10 and rel.max() < 1e-5, (np.median(rel), rel.max())
    o1 = Oracle(dict(p, iwvec=1))
    _, got1 = o1.recov(u, guess)
    assert not np.array_equal(got1[reg], got[reg])  # a different inversion ran
    assert np.abs(got1[reg] - got[reg])[..., [0, 4]].max() / np.abs(q[reg])[..., [0, 4]].min() < 1e-3


def _read_records(path):
    import struct
    with open(path, "rb") as f:
        data = f.read()
    recs, off = [], 0
    while off < len(data):
        (n,) = struct.unpack_from("<i", data, off)
        (m,) = struct.unpack_from("<i", data, off + 4 + n)
        assert m == n
        recs.append(data[off + 4: off + 4 + n])
        off += n + 8
    return recs


def test_output1_layout(tmp_path):
    """output1's snapshot file (restar.f90:91-185) from the oracle: header
    records (time, myrank, npe) and (is, ie, js, je, ks, ke), then one record
    of 13 doubles per cell with k fastest, then j, then i: the MKS coordinates
    x1b, x2b, x3b (metric 403), the nine primitives and sqrt(-g)."""
    import struct
    p = config.torus(nr=20, nth=16, nph=10)
    o = Oracle(p)
    o.ic_torus(seed=3)
    path = str(tmp_path / "structr0000-0001.outdat")
    o.output1(path, myrank=0, npe=1)
    recs = _read_records(path)
    imax, jmax, kmax = p["imax"], p["jmax"], p["kmax"]
    assert len(recs) == 2 + imax * jmax * kmax
    t, rank, npe = struct.unpack("<dii", recs[0])
    assert (t, rank, npe) == (o.time, 0, 1)
    assert struct.unpack("<6i", recs[1]) == (1, imax, 1, jmax, 1, kmax)
    body = np.frombuffer(b"".join(recs[2:]), dtype="<f8").reshape(imax, jmax, kmax, 13)
    u = o.prims()  # (kmax, jmax, imax, 9)
    assert np.array_equal(body[..., 3:12], np.transpose(u, (2, 1, 0, 3)))
    assert np.array_equal(body[:, 0, 0, 0], o.array("x1b"))
    assert np.array_equal(body[0, :, 0, 1], o.array("x2b"))
    assert np.array_equal(body[0, 0, :, 2], o.array("x3b"))
    detg = o.array("detg").reshape(kmax, imax)
    assert np.array_equal(body[:, 3, :, 12], detg.T)
    assert len(open(path, "rb").read()) == 24 + 32 + imax * jmax * kmax * 112
