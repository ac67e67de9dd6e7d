"""The allocation-free entry point, gray_run_mixed_noalloc.

Callers whose allocator already owns the device memory, or that cannot take
the synchronisation of cudaMalloc, hand in their own state buffers and get
the mixed-precision render without the library allocating anything; the
kernel's scratch is a static device array.  This test calls it through the
C ABI with buffers allocated by the caller (torch here), twice in a row on
the same buffers, and checks each result against the ordinary entry point
(gray_render_create + gray_run) within the FP64 parity tolerance.  The file
is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

from gray_b200 import api, configs

pytestmark = pytest.mark.gpu

TOL = 1e-10  # the parity tolerance of the FP64 tests


def reference_run(ctx, cfg):
    r = ctx.render(dict(cfg, precision=api.PREC_MIXED))
    try:
        r.run()
        data, info = r.state(api.LAYOUT_SOA)
        return data, info, r.steps()
    finally:
        r.close()


def test_noalloc_matches_ordinary_entry_point(ctx):
    import torch

    cfgs = [configs.scaled(configs.TORUS_RT_1024, 40),
            dict(configs.scaled(configs.TORUS_RT_1024, 24), a_spin=0.5, i_obs=60.0)]
    refs = [reference_run(ctx, c) for c in cfgs]

    descs = (api.RenderDesc * len(cfgs))(*[api.make_desc(dict(c, precision=api.PREC_MIXED))
                                           for c in cfgs])
    nd = 8 + 2 * len(cfgs[0]["nu"])
    states = [torch.empty((nd, c["n_width"] * c["n_height"]), dtype=torch.float64, device="cuda")
              for c in cfgs]
    infos = [torch.empty(c["n_width"] * c["n_height"], dtype=torch.float64, device="cuda")
             for c in cfgs]
    sp = (ctypes.c_void_p * len(cfgs))(*[t.data_ptr() for t in states])
    ip = (ctypes.c_void_p * len(cfgs))(*[t.data_ptr() for t in infos])
    stream = torch.cuda.Stream()
    L = api.lib()
    for call in range(2):
        for t in states + infos:
            t.fill_(np.nan)  # nothing stale may survive into the comparison
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        steps = ctypes.c_uint64(0)
        st = L.gray_run_mixed_noalloc(torch.cuda.current_device(), descs, len(cfgs), sp, ip,
                                      ctypes.c_void_p(stream.cuda_stream), ctypes.byref(steps))
        assert st == api.OK, api.strerror(st)
        torch.cuda.synchronize()
        if call == 1:
            # the first call may load the kernels' module; after it, a call
            # takes no device memory at all
            assert torch.cuda.mem_get_info()[0] == free_before
        assert steps.value == sum(r[2] for r in refs)
        for k, (data, info, _) in enumerate(refs):
            got = states[k].cpu().numpy()
            gi = infos[k].cpu().numpy()
            scale = np.maximum(np.abs(data), 1e-300).max(axis=1, keepdims=True)
            err = np.max(np.abs(got - data) / scale)
            print("call %d render %d: max rel diff %.3e, identical %s"
                  % (call, k, err, np.array_equal(got, data)))
            assert err <= TOL
            assert np.max(np.abs(gi - info)) <= TOL * max(1.0, np.max(np.abs(info)))


def test_noalloc_one_render(ctx):
    """One render: the call's launch takes the render's constants as a
    kernel parameter; the result is the ordinary entry point's."""
    import torch

    cfg = dict(configs.scaled(configs.TORUS_RT_1024, 32), a_spin=0.9, i_obs=45.0)
    data, info, steps_ref = reference_run(ctx, cfg)
    desc = (api.RenderDesc * 1)(api.make_desc(dict(cfg, precision=api.PREC_MIXED)))
    nr = cfg["n_width"] * cfg["n_height"]
    state = torch.full((8 + 2 * len(cfg["nu"]), nr), float("nan"), dtype=torch.float64,
                       device="cuda")
    inf = torch.full((nr,), float("nan"), dtype=torch.float64, device="cuda")
    sp = (ctypes.c_void_p * 1)(state.data_ptr())
    ip = (ctypes.c_void_p * 1)(inf.data_ptr())
    steps = ctypes.c_uint64(0)
    torch.cuda.synchronize()
    st = api.lib().gray_run_mixed_noalloc(torch.cuda.current_device(), desc, 1, sp, ip,
                                          ctypes.c_void_p(0), ctypes.byref(steps))
    assert st == api.OK, api.strerror(st)
    torch.cuda.synchronize()
    assert steps.value == steps_ref
    scale = np.maximum(np.abs(data), 1e-300).max(axis=1, keepdims=True)
    assert np.max(np.abs(state.cpu().numpy() - data) / scale) <= TOL
    assert np.max(np.abs(inf.cpu().numpy() - info)) <= TOL * max(1.0, np.max(np.abs(info)))


def test_noalloc_rejects_sizes_beyond_the_scratch():
    L = api.lib()
    n = api.NOALLOC_MAX_RENDERS + 1
    descs = (api.RenderDesc * n)(*[api.make_desc(dict(configs.scaled(configs.TORUS_RT_1024, 8),
                                                      precision=api.PREC_MIXED))
                                   for _ in range(n)])
    ptrs = (ctypes.c_void_p * n)()
    assert L.gray_run_mixed_noalloc(0, descs, n, ptrs, ptrs, None, None) == api.EINVAL
    assert L.gray_run_mixed_noalloc(0, descs, 0, ptrs, ptrs, None, None) == api.EINVAL
