"""Batches: many renders in one persistent launch, graph capture and replay,
the launch-plan autotuner, and one-ray vs two-ray (f32x2) kernels."""
import numpy as np
import pytest

from gray_b200 import api, configs

pytestmark = pytest.mark.gpu


def small_survey(n=6, hi=40):
    cfgs = configs.survey(n=n, side_lo=8, side_hi=hi)
    for c in cfgs:
        c["n_dump"] = 16  # keep the test short: 500 M of affine parameter
    return cfgs


def alone(ctx, cfg, prec=api.PREC_MIXED):
    r = ctx.render(dict(cfg, precision=prec))
    try:
        r.run()
        return r.state(api.LAYOUT_AOS)[0], r.steps()
    finally:
        r.close()


def rel(a, b):
    return np.max(np.abs(a - b) / np.maximum(np.abs(b).max(axis=1, keepdims=True), 1e-300))


def test_batch_equals_renders_alone(ctx):
    cfgs = small_survey()
    ref = [alone(ctx, c) for c in cfgs]
    rs = [ctx.render(dict(c, precision=api.PREC_MIXED)) for c in cfgs]
    b = ctx.batch(rs)
    try:
        for rep in range(2):  # capture, then graph replay
            ns = b.run()
            assert ns > 0
            assert b.steps() == sum(s for _, s in ref)
            for r, (d, _) in zip(rs, ref):
                got = r.state(api.LAYOUT_AOS)[0]
                assert rel(got, d) <= 1e-10, rep
    finally:
        b.close()
        for r in rs:
            r.close()


def test_one_render_batch_and_table_constants_agree(ctx):
    """A batch of one render runs the one-render launch (the render's
    constants as a kernel parameter) inside its graph; a batch of two reads
    each ray's constants from the table into registers.  Both equal the
    renders run alone bit for bit."""
    cfgs = small_survey(n=2)
    ref = [alone(ctx, c) for c in cfgs]
    for group in ([cfgs[0]], cfgs):
        rs = [ctx.render(dict(c, precision=api.PREC_MIXED)) for c in group]
        b = ctx.batch(rs)
        try:
            for rep in range(2):
                b.run()
                assert b.steps() == sum(s for _, s in ref[:len(group)])
                for r, (d, _) in zip(rs, ref):
                    assert np.array_equal(r.state(api.LAYOUT_AOS)[0], d), (len(group), rep)
        finally:
            b.close()
            for r in rs:
                r.close()


def test_rays_per_thread_variants_agree(ctx):
    """Packed two-ray and scalar kernels, RK4 stages unrolled or looped: the
    looped stages run the same operations in the same order."""
    cfgs = small_survey(n=3)
    old = ctx.get_plan()
    try:
        ctx.set_plan(128, 0, 2)
        two = [alone(ctx, c)[0] for c in cfgs]
        ctx.set_plan(256, 0, 1)
        one = [alone(ctx, c)[0] for c in cfgs]
        ctx.set_plan(256, 0, 1, rk4_rolled=1)
        rolled = [alone(ctx, c)[0] for c in cfgs]
        ctx.set_plan(128, 0, 2, rk4_rolled=1)
        two_rolled = [alone(ctx, c)[0] for c in cfgs]
    finally:
        ctx.set_plan(old.block, old.blocks_per_sm, old.rays_per_thread, old.rk4_rolled)
    for a, b in zip(one, two):
        img = np.linalg.norm(a[:, 8:12] - b[:, 8:12]) / np.linalg.norm(b[:, 8:12])
        assert img <= 1e-5, img
    for a, b in list(zip(one, rolled)) + list(zip(two, two_rolled)):
        assert rel(b, a) <= 1e-6
    print("looped RK4 bit-identical to unrolled: %s" %
          all(np.array_equal(a, b) for a, b in zip(one, rolled)))


def test_plan_measures_and_installs(ctx):
    cfgs = small_survey(n=4)
    rs = [ctx.render(dict(c, precision=api.PREC_MIXED)) for c in cfgs]
    b = ctx.batch(rs)
    old = ctx.get_plan()
    try:
        p = ctx.plan(b, api.PLAN_MEASURE)
        assert p.rays_per_thread in (1, 2) and p.block % 32 == 0 and p.ns > 0
        assert p.rk4_rolled in (0, 1)
        cur = ctx.get_plan()
        assert (cur.block, cur.rays_per_thread, cur.rk4_rolled) == \
            (p.block, p.rays_per_thread, p.rk4_rolled)
        b.run()
        for r, c in zip(rs, cfgs):
            d, _ = alone(ctx, c)
            assert rel(r.state(api.LAYOUT_AOS)[0], d) <= 1e-5
    finally:
        ctx.set_plan(old.block, old.blocks_per_sm, old.rays_per_thread, old.rk4_rolled)
        b.close()
        for r in rs:
            r.close()


def test_batch_vs_fp64_one_at_a_time(ctx):
    """The survey workload's check: batched mixed vs the FP64 kernel run one
    render at a time, image error per render."""
    cfgs = small_survey(n=4, hi=32)
    rs = [ctx.render(dict(c, precision=api.PREC_MIXED)) for c in cfgs]
    b = ctx.batch(rs)
    try:
        b.run()
        for r, c in zip(rs, cfgs):
            d64, _ = alone(ctx, c, api.PREC_FP64)
            got = r.state(api.LAYOUT_AOS)[0]
            for i in range(4):
                ref = d64[:, 8 + i]
                err = np.linalg.norm(got[:, 8 + i] - ref) / np.linalg.norm(ref)
                assert err <= 1e-4, (c["a_spin"], i, err)
    finally:
        b.close()
        for r in rs:
            r.close()


def test_batch_rejects_mixed_kinds(ctx):
    r1 = ctx.render(dict(configs.scaled(configs.TORUS_RT_1024, 8), precision=api.PREC_MIXED))
    r2 = ctx.render(dict(configs.scaled(configs.KERR_SMALL_64, 8), precision=api.PREC_MIXED))
    r3 = ctx.render(dict(configs.scaled(configs.TORUS_RT_1024, 8), precision=api.PREC_FP64))
    try:
        for pair in ([r1, r2], [r1, r3], [r1, r1]):
            with pytest.raises(api.GrayError) as e:
                ctx.batch(pair)
            assert e.value.status == api.EINVAL
        b = ctx.batch([r1])
        # a render cannot be destroyed while a batch refers to it
        assert api.lib().gray_render_destroy(ctx.h, r1.id) == api.ESTATE
        b.close()
    finally:
        for r in (r1, r2, r3):
            r.close()
