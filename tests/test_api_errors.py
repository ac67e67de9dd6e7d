"""Error paths of the C ABI: the HBM budget, calls out of order, unknown
ids and mismatched host buffers.  Each is a status code (never an abort),
and the context stays usable after it: a render made afterwards gives the
same result as in a fresh context."""
import ctypes

import numpy as np
import pytest

from gray_b200 import api, configs

pytestmark = pytest.mark.gpu

SMALL = dict(configs.scaled(configs.KERR_SMALL_64, 16), n_dump=4, precision=api.PREC_FP64)


def run(ctx, cfg):
    r = ctx.render(cfg)
    try:
        r.run()
        return r.state(api.LAYOUT_AOS)[0]
    finally:
        r.close()


def test_budget_refuses_and_context_recovers(ctx):
    ref = run(ctx, SMALL)
    c = api.Context(0, hbm_budget=2 << 20)
    try:
        big = dict(configs.scaled(configs.KERR_SMALL_64, 512), precision=api.PREC_FP64)
        with pytest.raises(api.GrayError) as e:  # 512^2 x 8 doubles = 16 MiB
            c.render(big)
        assert e.value.status == api.EBUDGET
        for _ in range(2):  # the failed create left nothing allocated
            assert np.array_equal(run(c, SMALL), ref)
        r1 = c.render(SMALL)
        try:  # the budget counts live renders: a second 1 MiB one does not fit
            mid = dict(configs.scaled(configs.KERR_SMALL_64, 128), precision=api.PREC_FP64)
            r2 = c.render(mid)
            with pytest.raises(api.GrayError) as e:
                c.render(mid)
            assert e.value.status == api.EBUDGET
            r2.close()
            c.render(mid).close()
        finally:
            r1.close()
    finally:
        c.close()


def test_out_of_order_unknown_and_size_errors(ctx):
    L = api.lib()
    r = ctx.render(SMALL)
    try:
        n = r.n_rays * r.n_data
        buf = np.empty(n, dtype=np.float64)
        info = np.empty(r.n_rays, dtype=np.float64)
        ns = ctypes.c_double(0.0)
        # before icond there is no state to evolve or read
        assert L.gray_evolve_all(ctx.h, r.id, ctypes.byref(ns)) == api.ESTATE
        assert L.gray_read_state(ctx.h, r.id, buf.ctypes.data, buf.nbytes, info.ctypes.data,
                                 info.nbytes, api.LAYOUT_SOA) == api.ESTATE
        r.icond()
        # host buffers of the wrong size, and a layout that does not exist
        assert L.gray_read_state(ctx.h, r.id, buf.ctypes.data, buf.nbytes - 8, None, 0,
                                 api.LAYOUT_SOA) == api.ESIZE
        assert L.gray_read_state(ctx.h, r.id, None, 0, info.ctypes.data, info.nbytes + 8,
                                 api.LAYOUT_SOA) == api.ESIZE
        assert L.gray_read_state(ctx.h, r.id, buf.ctypes.data, buf.nbytes, None, 0,
                                 7) == api.EINVAL
        assert L.gray_write_state(ctx.h, r.id, buf.ctypes.data, buf.nbytes + 8,
                                  api.LAYOUT_SOA) == api.ESIZE
        # ids that were never made, or are gone
        assert L.gray_evolve_all(ctx.h, 987654, ctypes.byref(ns)) == api.ENOTFOUND
        gone = ctx.render(SMALL)
        gid = gone.id
        gone.close()
        assert L.gray_run(ctx.h, gid, ctypes.byref(ns)) == api.ENOTFOUND
        assert L.gray_render_destroy(ctx.h, gid) == api.ENOTFOUND
        # none of that touched the render
        r.evolve_all()
        data, _ = r.state(api.LAYOUT_AOS)
    finally:
        r.close()
    assert np.array_equal(data, run(ctx, SMALL))


def test_dump_count_beyond_int32_is_refused(ctx):
    """n_dump >= 2^31 would overflow the kernels' 32-bit dump counters: every
    create path refuses it with GRAY_EINVAL instead of running the wrong
    number of intervals."""
    for prec in (api.PREC_FP64, api.PREC_MIXED):
        for n_dump in (2 ** 31, 2 ** 32 + 4):
            with pytest.raises(api.GrayError) as e:
                ctx.render(dict(SMALL, precision=prec, n_dump=n_dump))
            assert e.value.status == api.EINVAL
    ok = ctx.render(dict(SMALL, n_dump=2 ** 31 - 1))  # the largest count is accepted
    ok.close()
