"""CPU-side checks of the C ABI: the library loads and exports exactly
what include/gray_cuda.h declares; argument validation needs no GPU."""
import ctypes
import os
import re

from gray_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions(path):
    src = open(path).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b(gray_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_header_matches_python_export_list():
    assert header_functions(os.path.join(ROOT, "include", "gray_cuda.h")) == sorted(api.EXPORTS)


def test_library_exports_every_declared_symbol():
    L = api.lib()
    for name in header_functions(os.path.join(ROOT, "include", "gray_cuda.h")):
        assert hasattr(L, name), name


def test_strerror_and_version():
    assert api.lib().gray_abi_version() == api.ABI_VERSION == 3
    assert api.strerror(api.EINVAL).startswith("invalid")
    assert api.strerror(api.EBUDGET).startswith("request exceeds")
    assert api.strerror(12345) == "unknown status"


def test_null_context_is_rejected():
    L = api.lib()
    assert L.gray_sync(None) == api.EINVAL
    assert L.gray_set_stream(None, None) == api.EINVAL
    rid = ctypes.c_int(0)
    d = api.make_desc({})
    assert L.gray_render_create(None, ctypes.byref(d), ctypes.byref(rid)) == api.EINVAL
    assert L.gray_icond(None, 1) == api.ENOTFOUND
    assert L.gray_hbm_used(None) == 0


def test_desc_defaults_follow_reference_opts():
    d = api.make_desc({})
    # sim/Kerr.opts, sim/infcam.opts, sim/gray.opts, sim-org/setup.opts
    assert (d.m_bh, d.a_spin) == (4e6, 0.0)
    assert (d.w_img, d.h_img, d.r_obs, d.i_obs, d.j_obs) == (64.0, 64.0, 1024.0, 60.0, 0.0)
    assert (d.n_width, d.n_height) == (512, 512)
    assert (d.t_init, d.dt_dump, d.n_dump, d.n_sub) == (0.0, -32.0, 64, 1024)
    assert d.n_freq == 0 and d.flow == api.FLOW_NONE


def test_bench_h2d_bytes_match_the_render_table(tmp_path):
    """bench.py's host-to-device bytes per render are sizeof(MixedRender)."""
    import shutil
    import subprocess
    import sys
    cxx, inc = shutil.which("g++"), "/usr/local/cuda/include"
    if not cxx or not os.path.isdir(inc):
        import pytest
        pytest.skip("no host compiler or CUDA headers")
    src = tmp_path / "sz.cpp"
    src.write_text('#include "%s"\n#include <cstdio>\nint main(){printf("%%zu", sizeof(MixedRender));}\n'
                   % os.path.join(ROOT, "gray_b200", "csrc", "mixed_table.h"))
    exe = tmp_path / "sz"
    subprocess.run([cxx, "-I", inc, str(src), "-o", str(exe)], check=True)
    size = int(subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout)
    sys.path.insert(0, ROOT)
    import bench
    assert bench.H2D_BYTES_PER_RENDER == size


def test_missing_library_fails_loudly(tmp_path):
    """No CPU fallback: without libgray_cuda.so every entry point raises."""
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, %r)\n"
            "from gray_b200 import api\n"
            "api.LIB_PATH = %r\n"
            "try:\n"
            "    api.Context(0)\n"
            "except RuntimeError as e:\n"
            "    print('raised:', e)\n" % (ROOT, str(tmp_path / "absent.so")))
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    assert "raised:" in p.stdout and "not built" in p.stdout


def test_dump_count_beyond_int32_is_refused_before_any_device_call():
    """The persistent kernels count dump intervals in 32-bit integers, so
    every entry point refuses n_dump >= 2^31.  The allocation-free entry
    point validates its descriptors before it looks for a device, so this
    runs without a GPU."""
    from gray_b200 import configs
    L = api.lib()
    cfg = dict(configs.scaled(configs.TORUS_RT_1024, 8), precision=api.PREC_MIXED)
    ptrs = (ctypes.c_void_p * 1)(ctypes.c_void_p(16))  # never dereferenced
    for n_dump, want in ((2 ** 31, api.EINVAL), (2 ** 32 + 4, api.EINVAL)):
        d = (api.RenderDesc * 1)(api.make_desc(dict(cfg, n_dump=n_dump)))
        assert L.gray_run_mixed_noalloc(0, d, 1, ptrs, ptrs, None, None) == want
