"""Numerical spacetime: the device boosted-KS grid generator, fisheye +
trilinear + time interpolation and the dyst RHS against the CPU oracle."""
import numpy as np
import pytest

import oracle as O
from gray_b200 import api

BOX = 40.0


def oracle_grid(n, t, a=0.7, v=0.3, axis=1):
    return O.boosted_ks_grid(n, -BOX, BOX, t, a=a, v=v, axis=axis)


def test_oracle_grid_generator_matches_reference_points():
    """The oracle's grid sampler agrees with its pinned point sampler and
    places nodes on the fisheye map of tools/generate_data.py:49-58."""
    xs = O.fisheye_nodes(-BOX, BOX, 10)
    assert xs[0] == pytest.approx(-BOX, rel=1e-12) and xs[-1] == pytest.approx(BOX, rel=1e-12)
    g = oracle_grid(10, 0.0)
    q = np.array([0.0, xs[3], xs[7], xs[1]])
    ref = O.boosted_ks(1.0, 0.7, 0.3, 1, q)
    assert np.allclose(g[1, 7, 3, :50], ref.astype(np.float32), rtol=0, atol=0)


def test_oracle_dyst_rhs_tracks_ks_rhs():
    """On a grid sampled from unboosted KS the interpolated dyst RHS
    approaches the analytic KS geodesic equation (rescaled from affine to
    coordinate-time parametrisation) as the grid is refined."""
    a = 0.5
    q = np.array([0.0, 7.3, -4.1, 5.2])
    u = np.array([1.0, -0.3, 0.5, 0.2])
    u[1:] *= 1.0 / np.linalg.norm(u[1:])
    k = O.ks_rhs(a, np.r_[q, u])[4:]
    ref = k - k[0] * u  # coordinate-time form: a^mu - a^t u^mu
    errs = []
    for n in (33, 65):
        g = O.Grid([O.boosted_ks_grid(n, -BOX, BOX, 0.0, a=a, v=0.0)], [0, -BOX, -BOX, -BOX, 0, BOX, BOX, BOX])
        ds = O.dyst_rhs(g, np.r_[q, u])
        errs.append(np.max(np.abs(ds[4:] - ref)) / np.max(np.abs(ref)))
    assert errs[1] < errs[0] and errs[1] < 0.05


@pytest.mark.gpu
@pytest.mark.parametrize("axis", [1, 3])
def test_device_generator_matches_oracle(ctx, axis):
    """gray_make_boosted_ks (a kernel) against the oracle's restatement of
    tools/boosted_ks.py, field by field in FP32."""
    n = 12
    grid = api.make_grid(n, -BOX, BOX, 5.0, 5.0)
    ctx.make_boosted_ks(grid, 0.7, 0.3, axis, 5.0, 0)
    got = ctx.read_spacetime(grid, 0)
    ref = oracle_grid(n, 5.0, axis=axis)
    fin = np.isfinite(ref)
    assert np.array_equal(fin, np.isfinite(got))
    scale = np.max(np.abs(ref[fin]))
    diff = np.abs(got[fin].astype(np.float64) - ref[fin])
    rel = diff / np.maximum(np.abs(ref[fin]), 1e-6 * scale)
    print("generator: identical %.4f, max rel %.2e" % (np.mean(diff == 0), rel.max()))
    assert rel.max() <= 1e-5


def close_with_nans(g, o, tol):
    """Equal NaN/Inf patterns (rays that fell into the singular region
    compute the same garbage on both sides) and relative agreement on the
    finite rays."""
    fin = np.all(np.isfinite(o), axis=1)
    assert np.array_equal(fin, np.all(np.isfinite(g), axis=1))
    if not fin.any():
        return 1.0, 0.0
    gg, oo = g[fin], o[fin]
    err = np.max(np.abs(gg - oo) / np.abs(oo).max(axis=1, keepdims=True))
    assert err <= tol, err
    return np.mean(np.all(gg == oo, axis=1)), err


def small_grid(ctx, n, t1, t2, physics, bug_gzz=False):
    lv = [oracle_grid(n, t1), oracle_grid(n, t2)]
    box = [t1, -BOX, -BOX, -BOX, t2, BOX, BOX, BOX]
    grid = api.make_grid(n, -BOX, BOX, t1, t2, physics=physics, bug_gzz=bug_gzz)
    ctx.load_spacetime(grid, lv[0], 0)
    ctx.load_spacetime(grid, lv[1], 1)
    return O.Grid(lv, box, physics=physics, bug_gzz=bug_gzz)


def run_dyst(ctx, cfg, precision):
    r = ctx.render(dict(cfg, spacetime=api.ST_NUMERICAL, precision=precision))
    try:
        r.run()
        data, info = r.state(api.LAYOUT_AOS)
        return data, info, r.steps()
    finally:
        r.close()


@pytest.mark.gpu
@pytest.mark.parametrize("physics", [False, True])
def test_fp64_dyst_matches_oracle(ctx, physics):
    n = 24
    og = small_grid(ctx, n, -10.0, 0.0, physics)
    # reference semantics: camera inside the box, |dt| within the levels;
    # physics mode: camera outside the box (flat there)
    cfg = dict(a_spin=0.0, r_obs=(30.0 if not physics else 60.0), i_obs=50.0, j_obs=20.0,
               w_img=30.0, h_img=30.0, n_width=8, n_height=6, dt_dump=-2.0,
               n_dump=3 if not physics else 30, n_sub=100)
    g, ginfo, gsteps = run_dyst(ctx, cfg, api.PREC_FP64)
    o, oinfo, osteps = O.dyst_trace(cfg, og, np.arange(48))
    assert gsteps == osteps.sum()
    exact, err = close_with_nans(g, o, 1e-10)
    print("dyst fp64 physics=%s: bit-identical %.3f, max rel %.3e" % (physics, exact, err))
    fin = np.isfinite(oinfo)
    assert np.max(np.abs(ginfo[fin] - oinfo[fin])) <= 1e-10 * max(1.0, np.max(np.abs(oinfo[fin])))


@pytest.mark.gpu
def test_gzz_bug_compatibility(ctx):
    """dyst.cl:78 reads g_zz from the g_yz image; the flag reproduces it."""
    n = 16
    cfg = dict(a_spin=0.0, r_obs=25.0, i_obs=40.0, w_img=10.0, h_img=10.0, n_width=4,
               n_height=4, dt_dump=-1.0, n_dump=1, n_sub=100)
    infos = []
    for bug in (False, True):
        og = small_grid(ctx, n, -10.0, 0.0, False, bug_gzz=bug)
        r = ctx.render(dict(cfg, spacetime=api.ST_NUMERICAL, precision=api.PREC_FP64))
        r.icond()
        _, info = r.state()
        r.close()
        _, oinfo, _ = O.dyst_trace(dict(cfg, n_dump=0), og, np.arange(16))
        assert np.allclose(info, oinfo, rtol=1e-12, atol=1e-14)
        infos.append(info)
    assert np.max(np.abs(infos[0] - infos[1])) > 1e-6


@pytest.mark.gpu
def test_mixed_dyst_close_to_fp64(ctx):
    n = 32
    small_grid(ctx, n, 0.0, 10.0, True)
    cfg = dict(a_spin=0.0, r_obs=80.0, i_obs=45.0, w_img=40.0, h_img=40.0, n_width=32,
               n_height=32, dt_dump=-10.0, n_dump=16, n_sub=100)
    g64, _, s64 = run_dyst(ctx, cfg, api.PREC_FP64)
    gmx, _, smx = run_dyst(ctx, cfg, api.PREC_MIXED)
    ok = np.all(np.isfinite(g64), axis=1) & np.all(np.isfinite(gmx), axis=1)
    assert ok.mean() > 0.9
    pos = np.linalg.norm(gmx[ok, 1:4] - g64[ok, 1:4]) / np.linalg.norm(g64[ok, 1:4])
    mom = np.linalg.norm(gmx[ok, 4:8] - g64[ok, 4:8]) / np.linalg.norm(g64[ok, 4:8])
    print("mixed vs fp64 dyst: pos %.3e mom %.3e, steps %d vs %d" % (pos, mom, smx, s64))
    assert pos <= 1e-4 and mom <= 1e-3


@pytest.mark.gpu
def test_numerical_batch_follows_grid_changes(ctx):
    """A batch replays a captured graph; after the grid's levels change
    (here gray_swap_levels) its next run must read the levels as they are
    now, like renders run alone."""
    small_grid(ctx, 16, 0.0, 5.0, False)
    base = dict(a_spin=0.0, r_obs=25.0, i_obs=50.0, j_obs=20.0, w_img=20.0, h_img=20.0,
                n_width=6, n_height=5, dt_dump=-2.0, n_dump=3, n_sub=50,
                spacetime=api.ST_NUMERICAL, precision=api.PREC_MIXED)
    cfgs = [base, dict(base, i_obs=70.0, n_width=4)]

    def alone():
        out = []
        for c in cfgs:
            r = ctx.render(c)
            try:
                r.run()
                out.append(r.state(api.LAYOUT_AOS)[0])
            finally:
                r.close()
        return out

    rs = [ctx.render(c) for c in cfgs]
    b = ctx.batch(rs)
    try:
        before = alone()
        for _ in range(2):  # capture, then replay
            b.run()
            for r, d in zip(rs, before):
                close_with_nans(r.state(api.LAYOUT_AOS)[0], d, 1e-10)
        ctx.swap_levels()  # same buffers, exchanged: a different spacetime
        after = alone()
        assert any(np.nanmax(np.abs(a - d)) > 1e-6 for a, d in zip(after, before))
        for _ in range(2):
            b.run()
            for r, d in zip(rs, after):
                close_with_nans(r.state(api.LAYOUT_AOS)[0], d, 1e-10)
    finally:
        ctx.swap_levels()
        b.close()
        for r in rs:
            r.close()
