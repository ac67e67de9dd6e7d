"""Thermal radiative transfer on numerical spacetimes (rt.cl:28-198 with the
template flow of flow.cl:36-58).

CPU: the oracle's emissivities against closed forms -- the Planck law, the
Bessel function K_2 (scipy), the Gaunt-factor branches of rt.cl:95-120 --
and the structure of its RHS.  GPU: the FP64 kernels against the oracle
(geodesic bit-identical, transfer within 1e-10 relative: the device exp,
log and cbrt are not glibc's), mixed against FP64 within 1e-4 of the image.
"""
import math
import os
import sys

import numpy as np
import pytest

import oracle as O
from gray_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
C_c, C_h, C_kB, C_me = 2.99792458e+10, 6.62606957e-27, 1.38064881e-16, 9.10938291e-28
C_Ry = 2.17987197e-11
BOX = 40.0
NU = [1e10, 2.3e11, 5e12]


def planck(nu, theta):
    """B_nu for the dimensionless temperature theta = kT / (m_e c^2)."""
    kT = theta * C_me * C_c * C_c
    return 2 * C_h * nu ** 3 / C_c ** 2 / math.expm1(C_h * nu / kT)


@pytest.mark.parametrize("nu,theta", [(1e9, 1.0), (2.3e11, 10.0), (1e14, 0.5),
                                      (5e12, 1e12), (1e10, 1e-3)])
def test_B_Planck_is_the_planck_law(nu, theta):
    """Both branches of rt.cl:80-93 (the exponential and the series for
    h nu / kT < 1e-5) give the Planck law."""
    B = O.emissivities()["B_Planck"](nu, theta)
    assert B == pytest.approx(planck(nu, theta), rel=1e-9)


def test_log_K2_table_matches_scipy():
    """The log K_2(1/te) table (rt.cl:38-68 grid) is the Bessel function at
    the nodes to the table's 1e-10 rounding, and the linear interpolation
    of rt.cl:70-78 stays within its second-order error between them."""
    from scipy.special import kve
    f = O.emissivities()["log_K2it"]
    nodes = 0.1 * 1000.0 ** (np.arange(61) / 60.0)
    exact = lambda te: math.log(kve(2, 1.0 / te)) - 1.0 / te
    for te in nodes[:-1]:
        assert f(te) == pytest.approx(exact(te), abs=1e-10)
    mid = np.sqrt(nodes[:-1] * nodes[1:])
    err = max(abs(f(te) - exact(te)) for te in mid)
    assert err < 2e-2
    assert f(100.0) == pytest.approx(exact(100.0), abs=1e-10)  # last node, in bounds


def test_log_K2_header_is_regenerated_by_its_script():
    sys.path.insert(0, os.path.join(ROOT, "gray_b200", "csrc"))
    try:
        import make_logk2
    finally:
        sys.path.pop(0)
    text = open(os.path.join(ROOT, "gray_b200", "csrc", "logk2_table.h")).read()
    assert make_logk2.render() == text


def test_gaunt_branches():
    """rt.cl:95-120, branch by branch."""
    G = O.emissivities()["Gaunt"]
    g2 = math.sqrt(3) / math.pi
    assert G(4.0, 9.0) == pytest.approx(math.sqrt(3 / math.pi) / 3.0, rel=1e-15)
    assert G(4.0, 0.5) == pytest.approx(g2 * (math.log(4 / 1.78107241799) - math.log(0.5)),
                                        rel=1e-14)
    assert G(0.25, 16.0) == pytest.approx(math.sqrt(12) / (0.5 * 4.0), rel=1e-15)
    assert G(0.25, 0.6) == 1.0
    x, y = 0.25, 0.1
    ref = g2 * (math.log(4 / 1.78107241799 ** 2.5) + math.log(math.sqrt(x) / y))
    assert G(x, y) == pytest.approx(ref, rel=1e-14)
    assert G(0.25, 1e-300) > 0  # floor at EPSILON: never negative


def test_emissivity_limits():
    E = O.emissivities()
    # no synchrotron below T_MIN, along the field, or without a field
    assert E["L_j_syn"](4.3e6, 1e11, 0.05, 1.0, 1e3, 0.3) == 0.0
    assert E["L_j_syn"](4.3e6, 1e11, 10.0, 1.0, 1e3, 1.0) == 0.0
    assert E["L_j_syn"](4.3e6, 1e11, 10.0, 1.0, 0.0, 0.0) == 0.0
    s1 = E["L_j_syn"](4.3e6, 1e11, 10.0, 1.0, 1e3, 0.3)
    s2 = E["L_j_syn"](4.3e6, 1e11, 10.0, 2.0, 1e3, 0.3)
    assert s1 > 0 and s2 == pytest.approx(2 * s1, rel=1e-15)  # linear in n_e
    f1 = E["L_j_ff"](4.3e6, 1e11, 10.0, 1.0)
    f2 = E["L_j_ff"](4.3e6, 1e11, 10.0, 3.0)
    assert f1 > 0 and f2 == pytest.approx(9 * f1, rel=1e-14)  # n_e^2
    assert E["L_j_ff"](8.6e6, 1e11, 10.0, 1.0) == pytest.approx(2 * f1, rel=1e-15)  # M_ADM
    # above T_MAX the analytic log K_2 takes over (rt.cl:166-167)
    assert E["L_j_syn"](4.3e6, 1e11, 1e3, 1.0, 1e3, 0.3) > 0


def oracle_grid(n, t, a=0.7, v=0.3, axis=1):
    return O.boosted_ks_grid(n, -BOX, BOX, t, a=a, v=v, axis=axis)


def cpu_grid(n, t1, t2, physics):
    lv = [oracle_grid(n, t1), oracle_grid(n, t2)]
    return O.Grid(lv, [t1, -BOX, -BOX, -BOX, t2, BOX, BOX, BOX], physics=physics), lv


def test_oracle_rt_rhs_structure():
    """The geodesic part of the thermal RHS is the plain dyst RHS; the
    transfer is -j e^-tau / shift^2 and -j shift / B_nu with shift = -k_t,
    k = down(q, u) and n_e the interpolated rho; no flow, no transfer;
    outside the box in physics mode n_e = 0."""
    g, _ = cpu_grid(16, -10.0, 0.0, True)
    cfg = dict(nu=NU, flow_te=10.0, flow_b=1e3)
    s = np.r_[-4.0, 7.3, -4.1, 5.2, 1.0, -0.3, 0.5, 0.2, [0.0] * 3, [0.3, 0.0, 1.0]]
    ds = O.dyst_rhs_rt(cfg, g, s)
    assert np.array_equal(ds[:8], O.dyst_rhs(g, s[:8]))
    assert np.all(ds[8:11] < 0) and np.all(ds[11:] < 0)
    ratio = ds[8:11] / np.exp(-s[11:])
    assert np.all(np.isfinite(ratio))
    # I' e^tau is independent of tau
    s2 = s.copy(); s2[11:] = 0.0
    assert np.allclose(O.dyst_rhs_rt(cfg, g, s2)[8:11], ratio, rtol=1e-14)
    assert np.all(O.dyst_rhs_rt(dict(cfg, flow=O.FLOW_NONE), g, s)[8:] == 0)
    far = s.copy(); far[1] = 60.0
    assert np.all(O.dyst_rhs_rt(cfg, g, far)[8:] == 0)


# ------------------------------------------------------------------ GPU

def load_grid(ctx, n, t1, t2, physics):
    og, lv = cpu_grid(n, t1, t2, physics)
    grid = api.make_grid(n, -BOX, BOX, t1, t2, physics=physics)
    ctx.load_spacetime(grid, lv[0], 0)
    ctx.load_spacetime(grid, lv[1], 1)
    return og


def run(ctx, cfg, precision):
    r = ctx.render(dict(cfg, spacetime=api.ST_NUMERICAL, precision=precision))
    try:
        r.run()
        data, info = r.state(api.LAYOUT_AOS)
        return data, info, r.steps()
    finally:
        r.close()


@pytest.mark.gpu
@pytest.mark.parametrize("te,b", [(1e12, 0.0), (10.0, 1e3)])
def test_fp64_thermal_matches_oracle(ctx, te, b):
    """te = 1e12, b = 0 is flow.cl's template (free-free only, analytic
    log K_2); te = 10 with a field exercises synchrotron and the K_2 table."""
    og = load_grid(ctx, 24, -10.0, 0.0, True)
    cfg = dict(a_spin=0.0, r_obs=60.0, i_obs=50.0, j_obs=20.0, w_img=30.0, h_img=30.0,
               n_width=8, n_height=6, dt_dump=-2.0, n_dump=30, n_sub=100, nu=NU,
               flow_te=te, flow_b=b)
    g, ginfo, gsteps = run(ctx, cfg, api.PREC_FP64)
    o, oinfo, osteps = O.dyst_trace(cfg, og, np.arange(48))
    assert gsteps == osteps.sum()
    fin = np.all(np.isfinite(o), axis=1)
    assert np.array_equal(fin, np.all(np.isfinite(g), axis=1)) and fin.mean() > 0.5
    assert np.array_equal(g[fin, :8], o[fin, :8])  # geodesic: bit-identical
    I, tau = o[fin, 8:11], o[fin, 11:14]
    assert np.all(I[np.abs(I).max(axis=1) > 0] > 0)
    for sl in (slice(8, 11), slice(11, 14)):
        ref = o[fin, sl]
        scale = np.abs(ref).max(axis=0)
        assert np.all(scale > 0)
        err = np.max(np.abs(g[fin, sl] - ref) / scale)
        print("thermal fp64 te=%g b=%g cols %s: max rel %.3e" % (te, b, sl, err))
        assert err <= 1e-10


@pytest.mark.gpu
def test_mixed_thermal_close_to_fp64(ctx):
    load_grid(ctx, 32, 0.0, 10.0, True)
    cfg = dict(a_spin=0.0, r_obs=80.0, i_obs=45.0, w_img=40.0, h_img=40.0, n_width=32,
               n_height=32, dt_dump=-10.0, n_dump=16, n_sub=100, nu=NU, flow_te=10.0,
               flow_b=1e3)
    g64, _, s64 = run(ctx, cfg, api.PREC_FP64)
    gmx, _, smx = run(ctx, cfg, api.PREC_MIXED)
    ok = np.all(np.isfinite(g64), axis=1) & np.all(np.isfinite(gmx), axis=1)
    # the image: rays that left the box, not those caught by the hole
    img = ok & (np.max(np.abs(g64[:, 1:4]), axis=1) > BOX)
    assert img.mean() > 0.5
    for f in range(3):
        ref, got = g64[img, 8 + f], gmx[img, 8 + f]
        l2 = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        mx = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
        print("mixed vs fp64 thermal nu=%g: image L2 err %.3e, max %.3e (steps %d vs %d)"
              % (NU[f], l2, mx, smx, s64))
        assert l2 <= 1e-4


@pytest.mark.gpu
def test_transfer_models_belong_to_their_spacetime(ctx):
    for bad in (dict(nu=NU, flow=api.FLOW_THERMAL),  # thermal needs the grid's rho
                dict(nu=NU, flow=api.FLOW_TORUS, spacetime=api.ST_NUMERICAL),
                dict(nu=NU, spacetime=api.ST_NUMERICAL, flow_te=0.0)):
        with pytest.raises(api.GrayError) as e:
            ctx.render(dict(dict(n_width=4, n_height=4), **bad))
        assert e.value.status == api.EINVAL
