"""The CPU oracle against the reference's own kernel sources.

oracle/_ref holds the reference's sim-org OpenCL programs compiled for the
CPU from its own .cl files (oracle/ref_shim supplies OpenCL's vector types,
built-ins and images, and the build-time definitions of sim-org/build.c):
the analytic Kerr-Schild program (KS.cl with phys.cl, RK4.cl, driver.cl)
and the numerical-spacetime program (interp.cl, dyst.cl, flow.cl, rt.cl,
phys.cl, RK4.cl, driver.cl).  These tests pin the restatement to them,
beyond the reference's Python spacetime code:
 - KS.cl's getrr, geteps, down and gr_rhs at random events;
 - whole traces of the reference's icond_drv and evolve_drv (camera, the
   integer-tick loop, getdt, the RK4 macro form) against the oracle's;
 - the fisheye map, clamp-to-edge and linear-filter interpolation, the
   time interpolation and extrapolation, the dyst RHS, flow.cl's template
   flow and rt.cl's thermal emissivities, including the g_zz typo of
   dyst.cl:78 that the oracle reproduces under its bug_gzz flag.
The two sides group their floating-point operations differently (OpenCL
vector expressions against explicit fma()), so they agree to rounding, not
bit for bit; rays near the photon ring amplify that over ~10^4 steps.

The libraries exist only where the reference tree was present at build
time; without them these tests skip.
"""
import numpy as np
import pytest

import oracle as O
from gray_b200 import configs

pytestmark = pytest.mark.skipif(not O.ref_available(),
                                reason="oracle/_ref not built (no reference tree at build time)")


def test_ks_functions_are_the_references():
    rng = np.random.default_rng(7)
    worst = {"getrr": 0.0, "geteps": 0.0, "down": 0.0, "rhs": 0.0}
    for _ in range(500):
        a = rng.uniform(-0.998, 0.998)
        q = np.r_[rng.uniform(-5, 5), rng.uniform(-40, 40, 3)]
        u = np.r_[1.0, rng.uniform(-1, 1, 3)]
        if O.geteps(a, q) < 0.05:
            continue
        for f in ("getrr", "geteps"):
            ref = O.ref_ks_func(f, a, q)
            got = O.getrr(a, q) if f == "getrr" else O.geteps(a, q)
            worst[f] = max(worst[f], abs(got - ref) / abs(ref))
        k = O.ref_ks_func("down", a, q, u)
        worst["down"] = max(worst["down"], np.max(np.abs(O.down(a, q, u) - k)) / np.max(np.abs(k)))
        ds = O.ref_ks_rhs(a, np.r_[q, u])
        worst["rhs"] = max(worst["rhs"], np.max(np.abs(O.ks_rhs(a, np.r_[q, u]) - ds)) /
                           np.max(np.abs(ds)))
    print("oracle vs KS.cl, max rel: %s" % {k: "%.1e" % v for k, v in worst.items()})
    assert max(worst.values()) <= 1e-14


def test_ks_traces_are_the_references():
    """kerr_small_64's camera and step control through the reference's own
    driver kernels, on 64 rays spread over the image."""
    cfg = configs.KERR_SMALL_64
    rays = (np.arange(64, dtype=np.int64) * 61) % (64 * 64)
    ref, rinfo = O.ref_ks_trace(cfg, rays)
    got, ginfo, _ = O.trace(cfg, rays)
    rel = np.max(np.abs(got - ref) / np.abs(ref).max(axis=1, keepdims=True), axis=1)
    print("kerr_small_64 traces, oracle vs sim-org program: median %.1e, max %.1e"
          % (np.median(rel), rel.max()))
    assert np.median(rel) <= 1e-14
    assert rel.max() <= 1e-9
    norm = np.sum(ref[:, 4:8] ** 2, axis=1)
    assert np.max(np.abs(ginfo - rinfo) / norm) <= 1e-14


def test_reference_loop_steps_and_threads():
    """The reference's driver loop counts the same accepted RK4 steps per ray
    as the oracle (kerr_small_64, and the first rays of the torus_rt_1024
    CPU sample), and its multi-threaded run equals the single-threaded one."""
    cfg = configs.KERR_SMALL_64
    rays = (np.arange(64, dtype=np.int64) * 61) % (64 * 64)
    one, info1 = O.ref_ks_trace(cfg, rays)
    many, info_m, steps = O.ref_ks_trace(cfg, rays, nthreads=4, with_steps=True)
    assert np.array_equal(one, many) and np.array_equal(info1, info_m)
    _, _, osteps = O.trace(cfg, rays)
    assert np.array_equal(steps, osteps)
    cfg = configs.TORUS_RT_1024
    rays = (np.arange(24, dtype=np.int64) * 7919) % (1024 * 1024)
    ref, _, steps = O.ref_ks_trace(cfg, rays, nthreads=0, with_steps=True)
    got, _, osteps = O.trace(cfg, rays)
    assert np.array_equal(steps, osteps)
    assert np.max(np.abs(got[:, :8] - ref) / np.abs(ref).max(axis=1, keepdims=True)) <= 1e-8


def test_ks_trace_a_zero_spin_and_forward():
    """a = 0 and a forward (dt > 0) trace, two dumps."""
    cfg = dict(configs.scaled(configs.KERR_SMALL_64, 6), a_spin=0.0, r_obs=60.0, i_obs=80.0,
               j_obs=30.0, dt_dump=4.0, n_dump=2, n_sub=64)
    rays = np.arange(36, dtype=np.int64)
    ref, _ = O.ref_ks_trace(cfg, rays)
    got, _, _ = O.trace(cfg, rays)
    assert np.max(np.abs(got - ref) / np.abs(ref).max(axis=1, keepdims=True)) <= 1e-12


BOX = 40.0


def grid(n, t1, t2):
    lv = [O.boosted_ks_grid(n, -BOX, BOX, t, a=0.7, v=0.3, axis=1).astype(np.float32)
          for t in (t1, t2)]
    return lv, [t1, -BOX, -BOX, -BOX, t2, BOX, BOX, BOX]


def compare_dyst(cfg, lv, box, rays, bug_gzz=True):
    ref, rinfo = O.ref_dyst_trace(cfg, lv, box, rays)
    got, ginfo, _ = O.dyst_trace(cfg, O.Grid(lv, box, bug_gzz=bug_gzz), rays)
    fin = np.all(np.isfinite(ref), axis=1)
    assert np.array_equal(fin, np.all(np.isfinite(got), axis=1))
    out = {}
    for name, cols in (("geodesic", slice(0, 8)), ("I", slice(8, 9)), ("tau", slice(9, 10))):
        a, b = got[fin, cols], ref[fin, cols]
        out[name] = float(np.max(np.abs(a - b) / np.maximum(np.abs(b).max(axis=1, keepdims=True),
                                                           1e-300)))
    out["info"] = float(np.max(np.abs(ginfo[fin] - rinfo[fin]) / np.abs(rinfo[fin])))
    return out


def test_dyst_program_with_thermal_transfer_is_the_references():
    """An in-box camera on a two-level boosted-KS grid, one frequency of
    thermal transfer: interp.cl, dyst.cl, flow.cl and rt.cl as written,
    including the g_zz typo (dyst.cl:78) the oracle reproduces with
    bug_gzz; without the flag the null-constraint diagnostic differs."""
    lv, box = grid(20, -10.0, 0.0)
    cfg = dict(a_spin=0.0, r_obs=30.0, i_obs=50.0, j_obs=20.0, w_img=30.0, h_img=30.0,
               n_width=6, n_height=4, dt_dump=-2.0, n_dump=3, n_sub=100, nu=(2.3e11,),
               m_adm=4.3e6, flow_te=1e12, flow_b=0.0)
    rays = np.arange(24, dtype=np.int64)
    err = compare_dyst(cfg, lv, box, rays)
    print("dyst program, oracle vs sim-org: %s" % {k: "%.1e" % v for k, v in err.items()})
    assert max(err.values()) <= 1e-13
    assert compare_dyst(cfg, lv, box, rays, bug_gzz=False)["info"] > 1e-6


def test_dyst_clamp_to_edge_and_time_extrapolation_are_the_references():
    """A camera outside the box (clamp-to-edge fields, interp.cl:69-75) and
    dump times past the first level (unclamped linear extrapolation in time,
    interp.cl:204)."""
    lv, box = grid(16, -4.0, 0.0)
    cfg = dict(a_spin=0.0, r_obs=55.0, i_obs=35.0, j_obs=0.0, w_img=40.0, h_img=40.0,
               n_width=4, n_height=4, dt_dump=-3.0, n_dump=4, n_sub=50, nu=(1e12,),
               m_adm=4.3e6, flow_te=1e12, flow_b=0.0)
    err = compare_dyst(cfg, lv, box, np.arange(16, dtype=np.int64))
    print("dyst outside the box and past t1: %s" % {k: "%.1e" % v for k, v in err.items()})
    assert max(err.values()) <= 1e-12
