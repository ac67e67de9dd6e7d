"""Pins the CPU oracle (oracle/gray_oracle.c) before it is trusted.

The reference has no golden vectors for the geodesic path, so the oracle is
checked (1) against fixtures produced by the reference's own Python
spacetime code, tools/boosted_ks.py (tests/golden/make_golden.py), and
(2) against physics invariants of the formulas it restates.
"""
import json
import os

import numpy as np
import pytest

import oracle as O
from gray_b200 import configs

GOLD = os.path.join(os.path.dirname(__file__), "golden")
IDX_G = [(i, j, k) for i in range(4) for j in range(4) for k in range(j, 4)]


def load(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


def sym(g10):
    M = np.zeros((4, 4))
    n = 0
    for i in range(4):
        for j in range(i, 4):
            M[i, j] = M[j, i] = g10[n]
            n += 1
    return M


def test_boosted_ks_matches_reference_tool():
    """orc_boosted_ks restates boosted_ks.py metric() + Christoffel()."""
    for c in load("boosted_ks_points.json")["cases"]:
        out = O.boosted_ks(c["m"], c["a"], c["v"], c["axis"], np.array(c["q"]))
        ref = np.array(c["gamma"] + c["g"])
        scale = np.max(np.abs(ref))
        assert np.max(np.abs(out - ref)) <= 1e-12 * scale, c["q"]


def test_ks_rhs_matches_christoffels():
    """KS.cl gr_rhs (Chan et al. form) equals -Gamma^mu_ab u^a u^b of the
    reference tool at boost 0, and down() equals g_mu_nu u^nu."""
    rng = np.random.default_rng(7)
    n = 0
    for c in load("boosted_ks_points.json")["cases"]:
        if c["v"] != 0.0:
            continue
        q = np.array(c["q"])
        u = np.r_[1.0, rng.normal(size=3)]
        ds = O.ks_rhs(c["a"], np.r_[q, u])
        acc = np.zeros(4)
        for m, (i, j, k) in enumerate(IDX_G):
            acc[i] -= (1 if j == k else 2) * c["gamma"][m] * u[j] * u[k]
        assert np.allclose(ds[:4], u, rtol=0, atol=0)
        assert np.max(np.abs(ds[4:] - acc)) <= 1e-12 * np.max(np.abs(acc))
        k = O.down(c["a"], q, u)
        ref = sym(c["g"]) @ u
        assert np.max(np.abs(k - ref)) <= 1e-13 * np.max(np.abs(ref))
        n += 1
    assert n >= 30


def test_rk4_matches_reference_tool_integration():
    """RK4.cl integrate() on the KS RHS reproduces classical RK4 driven by
    the reference tool's Christoffel symbols."""
    for r in load("ks_rk4_rays.json")["rays"]:
        s = np.array(r["s0"])
        for _ in range(r["n"]):
            s = O.integrate({"a_spin": r["a"]}, s, r["h"])
        ref = np.array(r["s"])
        assert np.max(np.abs(s - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_icond_is_null():
    """KS.cl:207-229 rescales the camera direction so that g(u,u) = 0."""
    cfg = configs.scaled(configs.KERR_SMALL_64, 16)
    st = O.icond(cfg, range(256))
    uu = np.array([O.getuu(cfg["a_spin"], s) for s in st])
    assert np.max(np.abs(uu)) < 1e-12
    assert np.all(st[:, 4] == 1.0)


def test_conserved_quantities_along_rays():
    """Kerr-Schild is stationary and axisymmetric: E = -k_t and
    L_z = x k_y - y k_x are conserved; g(u,u) stays ~ 0."""
    cfg = dict(configs.scaled(configs.KERR_SMALL_64, 16), n_dump=8)
    rays = np.arange(0, 256, 17)
    st0 = O.icond(cfg, rays)
    st1, info, steps = O.trace(cfg, rays, nthreads=2)
    a = cfg["a_spin"]
    for s0, s1 in zip(st0, st1):
        k0 = O.down(a, s0[:4], s0[4:8])
        k1 = O.down(a, s1[:4], s1[4:8])
        assert abs(k1[0] - k0[0]) <= 1e-9 * abs(k0[0])
        L0 = s0[1] * k0[2] - s0[2] * k0[1]
        L1 = s1[1] * k1[2] - s1[2] * k1[1]
        assert abs(L1 - L0) <= 1e-8 * max(1.0, abs(L0))
    assert np.max(np.abs(info)) < 1e-8
    assert np.all(steps == 8 * 1000)


def test_schwarzschild_capture_threshold():
    """a = 0: rays with impact parameter below 3 sqrt(3) M are captured."""
    base = dict(a_spin=0.0, w_img=0.0, h_img=0.0, r_obs=1000.0, i_obs=90.0,
                n_width=1, n_height=1, dt_dump=-31.25, n_sub=1000, n_dump=40)
    bc = 3.0 * np.sqrt(3.0)
    for b, captured in [(bc - 0.15, True), (bc + 0.15, False)]:
        # one pixel at alpha = b: w_img = 2b and n_width = 1 puts the pixel
        # centre at alpha = (0.5 - 0.5) * 2b ... so use a 2-pixel row instead
        cfg = dict(base, w_img=4 * b, n_width=2)  # pixel 1: alpha = +b
        st, info, steps = O.trace(cfg, np.array([1]), nthreads=1)
        r = np.sqrt(O.getrr(0.0, st[0, :4]))
        assert (r < 2.1) == captured, (b, r)


def far_field_deviation(r_obs):
    """Rays of a camera at r_obs over 1000 M of affine parameter: the
    relative departure of q from the straight line q0 + u0 dl, and of u from
    u0 (maxima over 16 rays)."""
    cfg = dict(a_spin=0.9, w_img=0.2 * r_obs, h_img=0.2 * r_obs, r_obs=r_obs, i_obs=60.0,
               j_obs=0.0, n_width=4, n_height=4, t_init=0.0, dt_dump=-250.0, n_sub=1000,
               n_dump=4, nu=())
    rays = np.arange(16)
    s0 = O.icond(cfg, rays)
    s1, _, steps = O.trace(cfg, rays, nthreads=1)
    dl = cfg["n_dump"] * cfg["dt_dump"]
    line = s0[:, :4] + s0[:, 4:8] * dl
    dq = np.linalg.norm(s1[:, :4] - line, axis=1) / np.linalg.norm(s0[:, 4:8] * dl, axis=1)
    du = np.linalg.norm(s1[:, 4:8] - s0[:, 4:8], axis=1) / np.linalg.norm(s0[:, 4:8], axis=1)
    assert np.all(steps == 4 * 1000)
    return dq.max(), du.max()


def test_large_r_straight_line_limit():
    """Far from the hole the Christoffel symbols fall off as M / r^2: rays
    are straight lines, and their departure from one scales as r^-2."""
    q4, u4 = far_field_deviation(1e4)
    q5, u5 = far_field_deviation(1e5)
    assert q5 < 1e-6 and u5 < 1e-6
    assert 70.0 < q4 / q5 < 140.0, (q4, q5)
    assert 70.0 < u4 / u5 < 140.0, (u4, u5)


def test_getdt_rule():
    """phys.cl:48-64: stop below eps 0.01; else min(|dt|, 0.01 eps^2)."""
    cfg = dict(a_spin=0.9)
    rp = O.rplus(0.9)
    assert O.getdt(cfg, np.array([0, rp + 0.005, 0, 0]), -0.03) == 0.0
    e = 1.0
    q = np.array([0.0, 0.0, 0.0, 0.0])
    # on the axis r = |z| exactly (a^2 z^2 term), pick z = r_+ + e
    q[3] = rp + e
    r = np.sqrt(O.getrr(0.9, q))
    eps = r - rp
    assert O.getdt(cfg, q, -1.0) == pytest.approx(-0.01 * eps * eps, rel=1e-15)
    assert O.getdt(cfg, q, -1e-4) == -1e-4


def test_isco_and_horizon():
    assert O.risco(0.0) == pytest.approx(6.0, abs=1e-12)
    assert O.rplus(0.0) == 2.0
    assert O.risco(0.998) == pytest.approx(1.2370, abs=1e-3)


def test_torus_transfer_kappa_pin():
    """The frozen kappa puts tau(nu=1) = 1 on the central ray; tau scales as
    nu^-2 and I grows monotonically along the backward ray."""
    cfg = dict(configs.TORUS_RT_1024)
    st, info, steps = O.trace(cfg, np.array([512 * 1024 + 512]), nthreads=1)
    tau = st[0, 12:16]
    assert tau[0] == pytest.approx(1.0, abs=1e-4)
    assert np.allclose(tau[1:] / tau[0], [0.25, 0.0625, 0.015625], rtol=1e-6)
    assert np.all(st[0, 8:12] > 0)


def test_dump_intervals_compose():
    """Evolving dump by dump equals the all-dump trace (same tick loop)."""
    cfg = dict(configs.scaled(configs.KERR_SMALL_64, 8), n_dump=4)
    rays = np.array([0, 9, 27, 63])
    full, _, _ = O.trace(cfg, rays, nthreads=1)
    st = O.icond(cfg, rays)
    L = O.lib()
    d = O.make_desc(cfg)
    import ctypes
    for k in range(len(rays)):
        s = np.ascontiguousarray(st[k])
        for i in range(4):
            t = cfg["t_init"] + i * cfg["dt_dump"]
            tg = cfg["t_init"] + (i + 1) * cfg["dt_dump"]
            L.orc_evolve_ray(ctypes.byref(d), O._p(s), tg - t, cfg["n_sub"])
        assert np.array_equal(s, full[k])
