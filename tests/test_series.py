"""Dynamic spacetimes: a render across a time series of grid snapshots
(the "slow light" loop of sim-org/gray.c:147-294).

CPU: the library's snapshot schedule (gray_series_schedule, host code)
against the oracle's restatement of find_snapshot and the dump loop, on
fixed and random series.  GPU: gray_run_series in FP64 against the
oracle's series trace (geodesic bit-identical), in mixed precision against
the same intervals driven by hand through gray_load_spacetime and
gray_evolve (bit-identical: the streaming changes where levels live, not
what is computed), fast light, the dump callback and a failing loader."""
import numpy as np
import pytest

import oracle as O
from gray_b200 import api

BOX = 40.0
TIMES = [-20.0, -15.0, -10.0, -5.0, 0.0]


def test_schedule_of_a_backward_run():
    # pair of [t_k, t_k+1] bracketing t_init = 0, then each dump end time
    pairs = api.series_schedule(TIMES, 0.0, -2.0, 9)
    # -10 ends interval 5 on the edge of [-10, -5]: the pair stays (t <= t2)
    assert list(pairs) == [3, 3, 3, 2, 2, 2, 1, 1, 0]
    first, ref = O.series_schedule(TIMES, 0.0, -2.0, 9)
    assert first == 3 and list(ref) == list(pairs)


def test_schedule_of_a_forward_run():
    pairs = api.series_schedule(TIMES, -20.0, 2.0, 9)
    assert list(pairs) == [0, 0, 0, 1, 1, 1, 2, 2, 3]
    first, ref = O.series_schedule(TIMES, -20.0, 2.0, 9)
    assert first == 0 and list(ref) == list(pairs)


def test_schedule_frozen_and_rejected():
    assert list(api.series_schedule([7.0], 3.0, -1.0, 4)) == [0, 0, 0, 0]
    # fast light freezes the snapshot of the pair bracketing t_init ([-10, -5])
    assert list(api.series_schedule(TIMES, -7.0, -2.0, 5, fast_light=True)) == [2] * 5
    for args in ((TIMES, 1.0, -2.0, 3),       # t_init after the series
                 (TIMES, 0.0, -2.0, 11),      # final time before it
                 ([0.0, 0.0, 1.0], 0.5, 0.1, 2),  # times not increasing
                 (TIMES, 5.0, -1.0, 2, True)):    # fast light outside the series
        with pytest.raises(api.GrayError) as e:
            api.series_schedule(*args)
        assert e.value.status == api.EINVAL
        assert O.series_schedule(*args) is None


def test_schedule_matches_oracle_on_random_series():
    rng = np.random.default_rng(11)
    for _ in range(400):
        n = int(rng.integers(1, 7))
        times = np.cumsum(rng.uniform(0.5, 4.0, n)) - 10.0
        dt = float(rng.choice([-1, 1]) * rng.uniform(0.1, 3.0))
        t_init = float(rng.uniform(times[0] - 1, times[-1] + 1))
        n_dump = int(rng.integers(0, 12))
        fast = bool(rng.integers(0, 2))
        ref = O.series_schedule(times, t_init, dt, n_dump, fast)
        if ref is None:
            with pytest.raises(api.GrayError):
                api.series_schedule(times, t_init, dt, n_dump, fast)
        else:
            assert list(api.series_schedule(times, t_init, dt, n_dump, fast)) == list(ref[1])


# ------------------------------------------------------------------ GPU

N = 16


@pytest.fixture(scope="module")
def snaps():
    return [O.boosted_ks_grid(N, -BOX, BOX, t, a=0.7, v=0.3, axis=1).astype(np.float32)
            for t in TIMES]


def cfg(**kw):
    c = dict(a_spin=0.0, r_obs=60.0, i_obs=50.0, j_obs=20.0, w_img=30.0, h_img=30.0,
             n_width=8, n_height=6, t_init=0.0, dt_dump=-2.0, n_dump=9, n_sub=50,
             spacetime=api.ST_NUMERICAL)
    c.update(kw)
    return c


@pytest.mark.gpu
@pytest.mark.parametrize("physics", [False, True])
def test_fp64_series_matches_oracle(ctx, snaps, physics):
    c = cfg(r_obs=60.0 if physics else 30.0)
    grid = api.make_grid(N, -BOX, BOX, physics=physics)
    r = ctx.render(dict(c, precision=api.PREC_FP64))
    try:
        ns, loads = r.run_series(grid, TIMES, lambda k: snaps[k])
        got, ginfo = r.state(api.LAYOUT_AOS)
        steps = r.steps()
    finally:
        r.close()
    assert loads == 5  # every snapshot read once: 2 at the start, then one per switch
    ref, rinfo, rsteps = O.dyst_series_trace(c, snaps, TIMES, -BOX, BOX, np.arange(48),
                                            physics=physics)
    assert steps == rsteps.sum()
    fin = np.all(np.isfinite(ref), axis=1)
    assert fin.mean() > 0.5 and np.array_equal(fin, np.all(np.isfinite(got), axis=1))
    assert np.array_equal(got[fin], ref[fin])
    assert np.allclose(ginfo[fin], rinfo[fin], rtol=0, atol=1e-12)
    # the series differs from a frozen spacetime, so the levels really moved
    frozen, _, _ = O.dyst_series_trace(c, snaps, TIMES, -BOX, BOX, np.arange(48),
                                       physics=physics, fast_light=True)
    assert np.max(np.abs(frozen[fin, 1:4] - ref[fin, 1:4])) > 1e-6
    print("series fp64 physics=%s: %d loads, %.2f ms" % (physics, loads, ns * 1e-6))


@pytest.mark.gpu
def test_fp64_forward_series_matches_oracle(ctx, snaps):
    """Forward in time from the first snapshot: the levels advance upward."""
    c = cfg(r_obs=30.0, t_init=-20.0, dt_dump=2.0)
    grid = api.make_grid(N, -BOX, BOX)
    r = ctx.render(dict(c, precision=api.PREC_FP64))
    try:
        _, loads = r.run_series(grid, TIMES, lambda k: snaps[k])
        got, _ = r.state(api.LAYOUT_AOS)
        steps = r.steps()
    finally:
        r.close()
    assert loads == 5
    ref, _, rsteps = O.dyst_series_trace(c, snaps, TIMES, -BOX, BOX, np.arange(48))
    assert steps == rsteps.sum()
    fin = np.all(np.isfinite(ref), axis=1)
    assert fin.mean() > 0.5 and np.array_equal(got[fin], ref[fin])


@pytest.mark.gpu
def test_mixed_series_equals_hand_driven_levels(ctx, snaps):
    c = cfg(n_width=16, n_height=16, nu=(1e10, 2.3e11), flow_te=10.0, flow_b=1e3)
    grid = api.make_grid(N, -BOX, BOX, physics=True)
    dumps = []
    r = ctx.render(dict(c, precision=api.PREC_MIXED))
    try:
        r.run_series(grid, TIMES, lambda k: snaps[k], after_dump=lambda i: dumps.append(
            (i, r.state(api.LAYOUT_AOS)[0])))
        streamed, sinfo = r.state(api.LAYOUT_AOS)
    finally:
        r.close()
    assert [i for i, _ in dumps] == list(range(1, 10))
    assert np.array_equal(dumps[-1][1], streamed)

    pairs = api.series_schedule(TIMES, 0.0, -2.0, 9)
    r = ctx.render(dict(c, precision=api.PREC_MIXED))
    try:
        def levels(k):
            g = api.make_grid(N, -BOX, BOX, TIMES[k], TIMES[k + 1], physics=True)
            ctx.load_spacetime(g, snaps[k], 0)
            ctx.load_spacetime(g, snaps[k + 1], 1)
        levels(pairs[0])
        r.icond()
        for i in range(9):
            if i == 0 or pairs[i] != pairs[i - 1]:
                levels(pairs[i])
            r.evolve(-2.0 * i, -2.0 * (i + 1))
            assert np.array_equal(r.state(api.LAYOUT_AOS)[0], dumps[i][1])
        manual, minfo = r.state(api.LAYOUT_AOS)
    finally:
        r.close()
    fin = np.all(np.isfinite(manual), axis=1)
    assert np.array_equal(streamed[fin], manual[fin])


@pytest.mark.gpu
def test_fast_light_freezes_the_snapshot(ctx, snaps):
    c = cfg(t_init=-7.0, n_dump=4)
    grid = api.make_grid(N, -BOX, BOX, physics=True)
    r = ctx.render(dict(c, precision=api.PREC_FP64))
    try:
        _, loads = r.run_series(grid, TIMES, lambda k: snaps[k], fast_light=True)
        got, _ = r.state(api.LAYOUT_AOS)
    finally:
        r.close()
    assert loads == 1
    ref, _, _ = O.dyst_series_trace(c, snaps, TIMES, -BOX, BOX, np.arange(48), physics=True,
                                    fast_light=True)
    fin = np.all(np.isfinite(ref), axis=1)
    assert np.array_equal(got[fin], ref[fin])


@pytest.mark.gpu
def test_failing_loader_and_bad_series(ctx, snaps):
    grid = api.make_grid(N, -BOX, BOX, physics=True)
    r = ctx.render(dict(cfg(), precision=api.PREC_FP64))
    try:
        def load(k):
            if k == 1:
                raise IOError("snapshot 1 unreadable")
            return snaps[k]
        with pytest.raises(IOError):
            r.run_series(grid, TIMES, load)
        with pytest.raises(api.GrayError) as e:
            r.run_series(grid, TIMES[:2], lambda k: snaps[k])  # final time outside
        assert e.value.status == api.EINVAL
        # the render and the context stay usable
        _, loads = r.run_series(grid, TIMES, lambda k: snaps[k])
        assert loads == 5
    finally:
        r.close()
    kerr = ctx.render(dict(n_width=4, n_height=4))
    try:
        with pytest.raises(api.GrayError) as e:
            kerr.run_series(grid, TIMES, lambda k: snaps[k])
        assert e.value.status == api.EINVAL
    finally:
        kerr.close()
