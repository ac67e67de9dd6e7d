"""Continuous-batching server: each request's result is the same alone and
in the mix; admission under the HBM budget; cancellation; validation.

Stated tolerance for "the same alone and in the mix": the server advances
renders a few dump intervals per launch and re-loads the FP64 state between
launches; the (hi, lo) FP32 pair of the compensated state survives that
round trip exactly except at rounding ties, so results are bit-identical
for nearly every ray and, at worst, within 1e-6 relative per component
(image relative L2 error <= 1e-7)."""
import time

import numpy as np
import pytest

from gray_b200 import api, configs

pytestmark = pytest.mark.gpu

BOX = 40.0


def kerr_requests():
    cfgs = configs.survey(n=5, side_lo=12, side_hi=36, seed=7)
    for c in cfgs:
        c["n_dump"] = 12
    return cfgs


def numerical_requests():
    base = dict(a_spin=0.0, r_obs=80.0, w_img=30.0, h_img=30.0, dt_dump=-10.0, n_dump=8,
                n_sub=100, nu=(), spacetime=api.ST_NUMERICAL)
    return [dict(base, i_obs=30.0, n_width=16, n_height=12),
            dict(base, i_obs=70.0, j_obs=40.0, n_width=10, n_height=10),
            # thermal transfer at two frequencies: its own table and launch
            dict(base, i_obs=50.0, n_width=8, n_height=8, nu=(1e10, 2.3e11), flow_te=10.0,
                 flow_b=1e3)]


def alone(ctx, cfg):
    r = ctx.render(dict(cfg, precision=api.PREC_MIXED))
    try:
        r.run()
        return r.state(api.LAYOUT_SOA)
    finally:
        r.close()


def wait(ctx, ids, timeout=300.0):
    t0 = time.time()
    while True:
        st = [ctx.poll(i).state for i in ids]
        if all(s >= api.REQ_DONE for s in st):
            return st
        assert time.time() - t0 < timeout, st
        time.sleep(0.01)


@pytest.fixture
def grid(ctx):
    g = api.make_grid(24, -BOX, BOX, 0.0, 0.0, physics=True)
    ctx.make_boosted_ks(g, 0.7, 0.3, 1, 0.0, 0)
    return g


def test_results_same_alone_and_in_the_mix(ctx, grid):
    reqs = kerr_requests() + numerical_requests()
    ref = [alone(ctx, c) for c in reqs]
    ctx.serve_start(max_inflight=64, dumps_per_iter=3)
    try:
        ids = []
        for k, c in enumerate(reqs):
            ids.append(ctx.submit(c))
            if k == 2:
                time.sleep(0.05)  # later requests arrive while the first run
        states = wait(ctx, ids)
        assert all(s == api.REQ_DONE for s in states)
        stats, st = ctx.serve_stats()
        assert st == api.OK and stats.completed == len(reqs) and stats.ray_steps[0] > 0
        assert stats.ray_steps[1] > 0
        exact = 0
        for rid, c, (d, info) in zip(ids, reqs, ref):
            s = ctx.poll(rid)
            assert s.t_submit <= s.t_admit <= s.t_done
            got, ginfo = ctx.result(rid, d.shape[0], d.shape[1])
            fin = np.all(np.isfinite(d), axis=0)
            assert np.array_equal(fin, np.all(np.isfinite(got), axis=0))
            scale = np.abs(d[:, fin]).max(axis=1, keepdims=True)
            err = np.max(np.abs(got[:, fin] - d[:, fin]) / np.maximum(scale, 1e-300))
            assert err <= 1e-6, err
            if c.get("nu"):
                for i in range(len(c["nu"])):
                    e = np.linalg.norm(got[8 + i] - d[8 + i]) / np.linalg.norm(d[8 + i])
                    assert e <= 1e-7
            exact += int(np.array_equal(got[:, fin], d[:, fin]))
        print("served results bit-identical to alone: %d of %d" % (exact, len(reqs)))
    finally:
        assert ctx.serve_stop() == api.OK


def test_admission_waits_for_memory(ctx):
    reqs = kerr_requests()[:3]
    sizes = [c["n_width"] * c["n_height"] * (8 + 2 * len(c["nu"]) + 1) * 8 for c in reqs]
    budget = max(sizes) + min(sizes) // 2  # never two of the larger ones at once
    ctx.serve_start(hbm_budget=budget, dumps_per_iter=4)
    try:
        big = dict(kerr_requests()[0], n_width=200, n_height=200)
        bad = ctx.submit(big)  # can never fit: fails at once
        assert ctx.poll(bad).state == api.REQ_FAILED and ctx.poll(bad).status == api.EBUDGET
        ids = [ctx.submit(c) for c in reqs]
        wait(ctx, ids)
        st = [ctx.poll(i) for i in ids]
        assert all(s.state == api.REQ_DONE for s in st)
        # any two requests resident at the same time fit the budget together
        spans = [(s.t_admit, s.t_done, sz) for s, sz in zip(st, sizes)]
        for i, a in enumerate(spans):
            for j, b in enumerate(spans):
                if i < j and b[0] < a[1] and a[0] < b[1]:
                    assert a[2] + b[2] <= budget
        for i in ids + [bad]:
            ctx.release(i)
    finally:
        ctx.serve_stop()


def test_cancel_and_validation(ctx):
    ctx.serve_start(dumps_per_iter=1)
    try:
        long = dict(configs.scaled(configs.TORUS_RT_1024, 64))
        rid = ctx.submit(long)
        ctx.cancel(rid)
        wait(ctx, [rid])
        assert ctx.poll(rid).state == api.REQ_CANCELLED
        ok = ctx.submit(dict(kerr_requests()[1]))
        wait(ctx, [ok])
        assert ctx.poll(ok).state == api.REQ_DONE
        with pytest.raises(api.GrayError) as e:
            ctx.submit(dict(kerr_requests()[1], precision=api.PREC_FP64))
        assert e.value.status == api.EINVAL
        with pytest.raises(api.GrayError) as e:
            ctx.submit(dict(kerr_requests()[1], a_spin=1.5))
        assert e.value.status == api.EINVAL
        with pytest.raises(api.GrayError) as e:
            ctx.poll(987654321)
        assert e.value.status == api.ENOTFOUND
        ctx.release(rid)
        ctx.release(ok)
    finally:
        ctx.serve_stop()
    with pytest.raises(api.GrayError) as e:
        ctx.submit(dict(kerr_requests()[1]))
    assert e.value.status == api.ESTATE


def test_stop_without_drain_drops_pending(ctx):
    ctx.serve_start(max_inflight=1, dumps_per_iter=1)
    ids = [ctx.submit(dict(configs.scaled(configs.TORUS_RT_1024, 48))) for _ in range(3)]
    assert ctx.serve_stop(drain=False) == api.OK
    del ids


def test_windows_sized_by_time_and_empty_requests(ctx):
    """A large render and several small ones together: an iteration lasts
    dumps_per_iter of the large render's (estimated) intervals, at least
    50 ms; the small ones get windows of that length and finish in an
    iteration or two, with the same results as alone; a request with no dump
    intervals returns its camera state."""
    big = dict(configs.scaled(configs.TORUS_RT_1024, 512), n_dump=24)
    small = [dict(configs.scaled(configs.TORUS_RT_1024, 8), n_dump=24, i_obs=float(10 + 20 * k))
             for k in range(3)]
    empty = dict(configs.scaled(configs.TORUS_RT_1024, 8), n_dump=0)
    reqs = [big] + small + [empty]
    ref = [alone(ctx, c) for c in reqs]
    ctx.serve_start(max_inflight=16, dumps_per_iter=2)
    try:
        ids = [ctx.submit(c) for c in reqs]
        assert all(s == api.REQ_DONE for s in wait(ctx, ids))
        stats, _ = ctx.serve_stats()
        done = [ctx.poll(i).t_done for i in ids]
        for rid, c, (d, info) in zip(ids, reqs, ref):
            got, ginfo = ctx.result(rid, 8 + 2 * len(c["nu"]), c["n_width"] * c["n_height"])
            scale = np.maximum(np.abs(d), 1e-300).max(axis=1, keepdims=True)
            assert np.max(np.abs(got - d) / scale) <= 1e-6
        # the large render's interval is estimated at 1000 steps x 262,144
        # rays / 4.5e10 ray-steps/s = 5.8 ms, so an iteration is the 50 ms
        # minimum: 8 of its intervals, 3 iterations for 24; the small ones
        # (1.5 ms per interval, latency-bound) finish in their first
        assert all(t <= done[0] for t in done[1:])
        assert stats.iterations <= 5
    finally:
        ctx.serve_stop()


def test_results_beyond_the_pinned_pool(ctx):
    """Finished results wait in the server's pinned host pool while it has
    room (the pool is the budget's size below 2 GiB) and in pageable memory
    beyond it; read results give their blocks back.  Every result, from
    either place, equals the render run alone."""
    cfgs = [dict(configs.scaled(configs.TORUS_RT_1024, s), n_dump=8) for s in (40, 24, 32, 16)]
    sizes = [c["n_width"] * c["n_height"] * (8 + 2 * len(c["nu"]) + 1) * 8 for c in cfgs]
    ref = [alone(ctx, c) for c in cfgs]
    ctx.serve_start(hbm_budget=max(sizes) + min(sizes), dumps_per_iter=8)
    try:
        for rep in range(2):  # the second round reuses the blocks the first gave back
            ids = [ctx.submit(c) for c in cfgs]
            assert all(s == api.REQ_DONE for s in wait(ctx, ids))  # none read yet
            for rid, c, (d, info) in zip(ids, cfgs, ref):
                got, ginfo = ctx.result(rid, 8 + 2 * len(c["nu"]), c["n_width"] * c["n_height"])
                scale = np.maximum(np.abs(d), 1e-300).max(axis=1, keepdims=True)
                assert np.max(np.abs(got - d) / scale) <= 1e-6, rep
    finally:
        ctx.serve_stop()
