"""Parity of the CUDA path with the CPU oracle (through the C ABI).

FP64: the plain kernel and the oracle place every fused multiply-add
identically and use IEEE divide/sqrt, so the geodesic agrees bit for bit;
the torus transfer calls exp/pow, whose last bit may differ between CUDA
and glibc.  Tolerance: 1e-10 relative per ray per component (the FP64
parity bar), with the bit-identical fraction reported.
Mixed: FP32 bulk with FP64 islands; image (I_nu) relative L2 error vs the
FP64 kernel <= 1e-4 per frequency.
"""
import numpy as np
import pytest

import oracle as O
from gray_b200 import api, configs

pytestmark = pytest.mark.gpu

TOL64 = 1e-10


def rel_err(a, b):
    scale = np.maximum(np.abs(b), 1e-300)
    return np.abs(a - b) / np.maximum(scale, np.max(np.abs(b), axis=-1, keepdims=True) * 1e-14)


def run_gpu(ctx, cfg):
    r = ctx.render(cfg)
    try:
        r.run()
        data, info = r.state(api.LAYOUT_AOS)
        return data, info, r.steps()
    finally:
        r.close()


def test_fp64_kerr_small_bit_exact(ctx):
    cfg = configs.scaled(configs.KERR_SMALL_64, 16)
    g, ginfo, gsteps = run_gpu(ctx, dict(cfg, precision=api.PREC_FP64))
    o, oinfo, osteps = O.trace(cfg, np.arange(256))
    assert gsteps == osteps.sum()
    exact = np.mean(np.all(g == o, axis=1))
    err = np.max(np.abs(g - o) / np.maximum(np.abs(o), 1e-300).max(axis=1, keepdims=True))
    print("fp64 bit-identical rays: %.3f, max rel err %.3e" % (exact, err))
    assert err <= TOL64
    assert exact >= 0.99
    assert np.max(np.abs(ginfo - oinfo)) <= 1e-12


def test_fp64_full_kerr_small_64(ctx):
    """The whole 64x64 workload (every ray, every dump) against the oracle."""
    cfg = configs.KERR_SMALL_64
    g, ginfo, gsteps = run_gpu(ctx, dict(cfg, precision=api.PREC_FP64))
    o, oinfo, osteps = O.trace(cfg, np.arange(64 * 64))
    assert gsteps == osteps.sum()
    rel = np.abs(g - o) / np.maximum(np.abs(o), 1e-300).max(axis=1, keepdims=True)
    print("kerr_small_64: bit-identical %.4f, max rel %.3e" % (np.mean(np.all(g == o, axis=1)), rel.max()))
    assert rel.max() <= TOL64


def test_fp64_torus_transfer(ctx):
    cfg = configs.scaled(configs.TORUS_RT_1024, 24)
    g, ginfo, gsteps = run_gpu(ctx, dict(cfg, precision=api.PREC_FP64))
    o, oinfo, osteps = O.trace(cfg, np.arange(24 * 24))
    assert gsteps == osteps.sum()
    geo = np.abs(g[:, :8] - o[:, :8]) / np.abs(o[:, :8]).max(axis=1, keepdims=True)
    rt = np.abs(g[:, 8:] - o[:, 8:]) / np.maximum(np.abs(o[:, 8:]), 1e-30)
    print("torus fp64: geo max rel %.3e, rt max rel %.3e" % (geo.max(), rt.max()))
    assert geo.max() <= TOL64
    assert rt.max() <= TOL64


def test_fp64_dump_by_dump_equals_run(ctx):
    """gray_evolve per dump interval (sim-org/gray.c loop) == gray_run."""
    cfg = dict(configs.scaled(configs.KERR_SMALL_64, 8), n_dump=6, precision=api.PREC_FP64)
    full, _, _ = run_gpu(ctx, cfg)
    r = ctx.render(cfg)
    try:
        r.icond()
        for i in range(6):
            t = cfg["t_init"] + i * cfg["dt_dump"]
            tg = cfg["t_init"] + (i + 1) * cfg["dt_dump"]
            ns = r.evolve(t, tg)
            assert ns > 0
        data, _ = r.state(api.LAYOUT_AOS)
    finally:
        r.close()
    assert np.array_equal(data, full)


def test_layouts_and_kdown(ctx):
    cfg = dict(configs.scaled(configs.TORUS_RT_1024, 8), n_dump=2, precision=api.PREC_FP64)
    r = ctx.render(cfg)
    try:
        r.run()
        soa, info = r.state(api.LAYOUT_SOA)
        aos, info2 = r.state(api.LAYOUT_AOS)
        assert np.array_equal(soa.T, aos)
        assert np.array_equal(info, info2)
        k = r.kdown()
        for g in range(0, 64, 7):
            ko = O.down(cfg["a_spin"], aos[g, :4], aos[g, 4:8])
            assert np.allclose(k[:, g], ko, rtol=1e-14, atol=1e-14)
        # write back in AoS, read in SoA
        r.write_state(aos, api.LAYOUT_AOS)
        soa2, _ = r.state(api.LAYOUT_SOA)
        assert np.array_equal(soa2, soa)
    finally:
        r.close()


def test_mixed_torus_image_error(ctx):
    cfg = configs.scaled(configs.TORUS_RT_1024, 96)
    g64, _, s64 = run_gpu(ctx, dict(cfg, precision=api.PREC_FP64))
    gmx, info, smx = run_gpu(ctx, dict(cfg, precision=api.PREC_MIXED))
    for i in range(4):
        ref = g64[:, 8 + i]
        err = np.linalg.norm(gmx[:, 8 + i] - ref) / np.linalg.norm(ref)
        print("nu_%d image rel L2 err %.3e" % (i, err))
        assert err <= 1e-4
    pos = np.linalg.norm(gmx[:, 1:4] - g64[:, 1:4]) / np.linalg.norm(g64[:, 1:4])
    print("end-position rel L2 err %.3e, steps fp64 %d mixed %d" % (pos, s64, smx))
    assert pos <= 1e-4
    assert abs(smx - s64) <= 1e-3 * s64
    # null constraint relative to |u|^2 (captured rays end with large u)
    norm = np.sum(gmx[:, 4:8] ** 2, axis=1)
    assert np.max(np.abs(info) / norm) < 1e-5


def test_mixed_matches_oracle_geodesics(ctx):
    cfg = configs.scaled(configs.KERR_SMALL_64, 16)
    gmx, info, smx = run_gpu(ctx, dict(cfg, precision=api.PREC_MIXED))
    o, oinfo, osteps = O.trace(cfg, np.arange(256))
    pos = np.linalg.norm(gmx[:, 1:4] - o[:, 1:4]) / np.linalg.norm(o[:, 1:4])
    mom = np.linalg.norm(gmx[:, 4:8] - o[:, 4:8]) / np.linalg.norm(o[:, 4:8])
    print("mixed vs oracle: pos %.3e mom %.3e" % (pos, mom))
    assert pos <= 1e-4 and mom <= 1e-4
    assert abs(smx - osteps.sum()) <= 1e-3 * osteps.sum()


@pytest.mark.parametrize("precision", [api.PREC_FP64, api.PREC_MIXED])
def test_row_blocks_concatenate_to_the_render(ctx, precision):
    """A render split into camera row windows (the multi-GPU row partition
    of one render) gives, block after block, exactly the whole render: rays
    are independent and the window keeps the whole image's pixel map."""
    from gray_b200 import shard
    cfg = dict(configs.scaled(configs.TORUS_RT_1024, 24), n_height=19, n_dump=8,
               precision=precision)
    full, finfo, fsteps = run_gpu(ctx, cfg)
    parts, infos, steps = [], [], 0
    for rank in range(3):
        begin, rows = shard.row_block(cfg["n_height"], rank, 3)
        g, gi, s = run_gpu(ctx, dict(cfg, row_begin=begin, n_rows=rows))
        assert g.shape[0] == rows * cfg["n_width"]
        parts.append(g)
        infos.append(gi)
        steps += s
    assert np.array_equal(np.concatenate(parts), full)
    assert np.array_equal(np.concatenate(infos), finfo)
    assert steps == fsteps


def test_row_window_is_validated(ctx):
    base = dict(configs.scaled(configs.KERR_SMALL_64, 8), precision=api.PREC_FP64)
    for bad in (dict(row_begin=1, n_rows=0), dict(row_begin=8, n_rows=1),
                dict(row_begin=6, n_rows=3)):
        with pytest.raises(api.GrayError) as e:
            ctx.render(dict(base, **bad))
        assert e.value.status == api.EINVAL
