"""Edge cases of the numerical-spacetime path against the CPU oracle: an
anisotropic grid over an asymmetric box, a single time level, linear time
extrapolation far outside [t1, t2] (reference semantics), forward tracing
(dt_dump > 0, out past t2 and the box edge), and the thermal
transfer with the g_zz flag.  FP64 geodesics bit-identical; the transfer
within the 1e-10 parity bar; mixed end positions within 1e-3 (L2) of FP64
on the rays that leave the box (physics mode)."""
import numpy as np
import pytest

import oracle as O
from gray_b200 import api

N3 = (12, 16, 20)
LO = (-30.0, -40.0, -50.0)
HI = (35.0, 40.0, 45.0)

CAM = dict(a_spin=0.0, i_obs=55.0, j_obs=25.0, w_img=24.0, h_img=18.0, n_width=8,
           n_height=6, n_sub=100)

CASES = {
    # (t1, t2, physics, bug_gzz, render overrides)
    "anisotropic_physics": (0.0, 5.0, True, False, dict(r_obs=80.0, dt_dump=-10.0, n_dump=24)),
    "single_level": (3.0, 3.0, False, False, dict(r_obs=25.0, dt_dump=-2.0, n_dump=3)),
    "time_extrapolation": (0.0, 2.0, False, False, dict(r_obs=25.0, dt_dump=-3.0, n_dump=4)),
    "forward": (0.0, 5.0, False, False, dict(r_obs=25.0, dt_dump=2.0, n_dump=3)),
    "thermal_gzz": (0.0, 5.0, True, True, dict(r_obs=80.0, dt_dump=-10.0, n_dump=24,
                                                nu=(1e10, 3e11), flow_te=10.0, flow_b=1e3)),
}


def levels(t1, t2):
    return [O.boosted_ks_grid(N3, LO, HI, t, a=0.6, v=0.2, axis=2) for t in (t1, t2)]


def setup(ctx, name):
    t1, t2, physics, bug, over = CASES[name]
    lv = levels(t1, t2)
    grid = api.make_grid(N3, LO, HI, t1, t2, physics=physics, bug_gzz=bug)
    ctx.load_spacetime(grid, lv[0], 0)
    ctx.load_spacetime(grid, lv[1], 1)
    box = [t1, LO[0], LO[1], LO[2], t2, HI[0], HI[1], HI[2]]
    og = O.Grid(lv, box, physics=physics, bug_gzz=bug)
    cfg = dict(CAM, spacetime=api.ST_NUMERICAL, **over)
    return cfg, og, physics


def gpu(ctx, cfg, prec):
    r = ctx.render(dict(cfg, precision=prec))
    try:
        r.run()
        d, info = r.state(api.LAYOUT_AOS)
        return d, info, r.steps()
    finally:
        r.close()


def test_anisotropic_grid_nodes_follow_the_fisheye_map():
    g = O.boosted_ks_grid(N3, LO, HI, 0.0, a=0.6, v=0.2, axis=2)
    assert g.shape == (N3[2], N3[1], N3[0], 51)
    for c in range(3):
        xs = O.fisheye_nodes(LO[c], HI[c], N3[c])
        assert xs[0] == pytest.approx(LO[c], rel=1e-12) and xs[-1] == pytest.approx(HI[c], rel=1e-12)
        assert np.all(np.diff(xs) > 0)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_fp64_dyst_edge_case_matches_oracle(ctx, name):
    cfg, og, _ = setup(ctx, name)
    n = cfg["n_width"] * cfg["n_height"]
    g, ginfo, gsteps = gpu(ctx, cfg, api.PREC_FP64)
    o, oinfo, osteps = O.dyst_trace(cfg, og, np.arange(n))
    assert gsteps == osteps.sum()
    fin = np.all(np.isfinite(o), axis=1)
    assert np.array_equal(fin, np.all(np.isfinite(g), axis=1)) and fin.any()
    assert np.array_equal(g[fin, :8], o[fin, :8]), name
    if o.shape[1] > 8:
        scale = np.maximum(np.abs(o[fin, 8:]).max(axis=0), 1e-300)
        assert np.max(np.abs(g[fin, 8:] - o[fin, 8:]) / scale) <= 1e-10
    ok = fin & np.isfinite(oinfo)
    assert np.allclose(ginfo[ok], oinfo[ok], rtol=1e-12, atol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["anisotropic_physics", "thermal_gzz"])
def test_mixed_dyst_edge_case_close_to_fp64(ctx, name):
    cfg, _, _ = setup(ctx, name)
    g64, _, _ = gpu(ctx, cfg, api.PREC_FP64)
    gmx, _, _ = gpu(ctx, cfg, api.PREC_MIXED)
    fin = np.all(np.isfinite(g64), axis=1) & np.all(np.isfinite(gmx), axis=1)
    lo, hi = np.array(LO), np.array(HI)
    out = fin & np.any((g64[:, 1:4] < lo) | (g64[:, 1:4] > hi), axis=1)
    assert out.mean() > 0.5
    pos = np.linalg.norm(gmx[out, 1:4] - g64[out, 1:4]) / np.linalg.norm(g64[out, 1:4])
    assert pos <= 1e-3, pos
    for i in range(len(cfg.get("nu", ()))):
        ref = g64[out, 8 + i]
        assert np.linalg.norm(gmx[out, 8 + i] - ref) / np.linalg.norm(ref) <= 1e-4
