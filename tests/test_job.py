"""The lux-job surface in C (gray_b200/host/gray_job.c): option names,
aliases and defaults of the reference's .opts tables, conf() semantics, the
raw dump format of sim-org/io.c:39-72, and (GPU) the `gray` CLI against the
oracle."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from gray_b200 import api, h5

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "gray_b200", "lib", "libgray_job.so")
CLI = os.path.join(ROOT, "gray_b200", "lib", "gray")
UNKNOWN = 1


class Job:
    def __init__(self):
        api.lib()  # libgray_cuda.so first (libgray_job.so links to it)
        L = ctypes.CDLL(LIB)
        L.gray_job_mkmod.restype = ctypes.c_void_p
        L.gray_job_mkmod.argtypes = [ctypes.c_void_p]
        L.gray_job_rmmod.argtypes = [ctypes.c_void_p]
        L.gray_job_desc.argtypes = [ctypes.c_void_p, ctypes.POINTER(api.RenderDesc)]
        L.gray_job_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t]
        L.gray_write_raw.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t]
        L.gray_read_raw.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t]
        self.L = L
        self.h = L.gray_job_mkmod(None)
        assert self.h
        CONF = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_char_p)
        RUN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p)
        # struct gray_lux_job: the vtable {conf, init, exec} is the first member
        vt = ctypes.cast(self.h, ctypes.POINTER(ctypes.c_void_p))
        self.conf_fn = CONF(vt[0])
        self.init_fn = RUN(vt[1])

    def conf(self, arg):
        return self.conf_fn(self.h, arg.encode())

    def init(self):
        return self.init_fn(self.h)

    def get(self, name):
        buf = ctypes.create_string_buffer(512)
        assert self.L.gray_job_get(self.h, name.encode(), buf, 512) == 0
        return buf.value.decode()

    def desc(self):
        d = api.RenderDesc()
        assert self.L.gray_job_desc(self.h, ctypes.byref(d)) == 0
        return d

    def close(self):
        self.L.gray_job_rmmod(self.h)


@pytest.fixture
def job():
    j = Job()
    yield j
    j.close()


def test_defaults_are_the_reference_opts(job):
    expect = {
        # sim/gray.opts
        "i_platform": "0", "i_device": "0", "spacetime": "Kerr", "initcond": "infcam",
        "t_init": "0", "dt_dump": "-32", "i_init": "0", "n_dump": "64", "rayfile": "ray%04d.h5",
        # sim/Kerr.opts
        "m_bh": "4000000", "a_spin": "0",
        # sim/infcam.opts
        "w_img": "64", "h_img": "64", "r_obs": "1024", "i_obs": "60", "j_obs": "0",
        "coordinates": "pxcenter", "n_width": "512", "n_height": "512",
        # sim-org/setup.opts
        "precision": "4", "scheme": "RK4", "morder": "AoS", "kflags": "-w",
        "outfile": "%04d.raw", "n_sub": "1024",
        # sim-org/param.opts
        "M_ADM": "4300000", "dyst_file": "data.h5", "enable_fast_light": "0",
        "n_electron": "1000000", "beta_crit": "1", "R_high": "1", "R_low": "1", "nu": "",
    }
    for k, v in expect.items():
        assert job.get(k) == v, k


def test_aliases_and_values(job):
    for arg in ["a=0.9", "M=10", "w=40", "h=30", "r=1000", "i=17", "j=5", "W=96", "H=48",
                "t0=1", "dt=-31.25", "i0=0", "N=7", "n=1000", "p=8", "mo=SoA", "ml=AoS",
                "st=KS", "ic=infcam", "id=0", "ip=0", "type=gpu", "out=", "nu=1,2,4,8",
                "torus_kappa=125.8988", "term=rplus"]:
        assert job.conf(arg) == 0, arg
    d = job.desc()
    assert (d.a_spin, d.m_bh, d.w_img, d.h_img, d.r_obs, d.i_obs, d.j_obs) == (0.9, 10, 40, 30, 1000, 17, 5)
    assert (d.n_width, d.n_height, d.n_dump, d.n_sub) == (96, 48, 7, 1000)
    assert (d.t_init, d.dt_dump) == (1.0, -31.25)
    assert d.precision == api.PREC_FP64
    assert d.n_freq == 4 and list(d.nu)[:4] == [1, 2, 4, 8] and d.flow == api.FLOW_TORUS
    assert d.term == api.TERM_RPLUS
    assert job.get("nu") == "1,2,4,8"
    assert job.get("outfile") == ""
    assert job.conf("p=single") == 0 and job.desc().precision == api.PREC_MIXED


def test_conf_rejects_without_side_effects(job):
    assert job.conf("bogus=1") == UNKNOWN
    assert job.conf("no_equals_sign") == UNKNOWN
    assert job.conf("a=0.3") == 0
    for bad in ["a=abc", "a=", "N=-1", "W=1x", "st=Minkowski", "ic=pinhole", "scm=RK45",
                "p=16", "nu=1,-2", "nu=1,2,3,4,5,6,7,8,9", "flow=disk",
                "out=%s.raw", "out=%d_%d.raw", "out=x%", "out=%ld.raw", "out=%n",
                "ray=%f.h5"]:
        assert job.conf(bad) == api.EINVAL, bad
    assert job.get("a_spin") == "0.29999999999999999"
    assert job.get("spacetime") == "Kerr"
    # a dump-name pattern with one integer conversion (or none) is accepted
    for good in ["out=run%%_%06d.raw", "out=%.4x", "out=final.raw", "out="]:
        assert job.conf(good) == 0, good


def test_raw_dump_format(job, tmp_path):
    """sim-org/io.c:58-67: {sz, n_data, W, H} as size_t, data, info."""
    w, h, nd = 5, 3, 10
    data = np.arange(w * h * nd, dtype=np.float64).reshape(w * h, nd)
    info = -np.arange(w * h, dtype=np.float64)
    path = str(tmp_path / "0007.raw")
    assert job.L.gray_write_raw(path.encode(), data.ctypes.data, info.ctypes.data, nd, w, h) == 0
    raw = open(path, "rb").read()
    hdr = np.frombuffer(raw[:32], dtype=np.uint64)
    assert list(hdr) == [8, nd, w, h]
    body = np.frombuffer(raw[32:], dtype=np.float64)
    assert np.array_equal(body[: w * h * nd].reshape(w * h, nd), data)
    assert np.array_equal(body[w * h * nd:], info)


def test_raw_dump_reads_back(job, tmp_path):
    """The load path of a dump (sim-org/io.c:37 leaves it a TODO)."""
    w, h, nd = 4, 3, 12
    data = np.random.default_rng(5).normal(size=(w * h, nd))
    info = np.linspace(-1, 1, w * h)
    path = str(tmp_path / "0003.raw").encode()
    assert job.L.gray_write_raw(path, data.ctypes.data, info.ctypes.data, nd, w, h) == 0
    d2, i2 = np.zeros_like(data), np.zeros_like(info)
    assert job.L.gray_read_raw(path, d2.ctypes.data, i2.ctypes.data, nd, w, h) == 0
    assert np.array_equal(d2, data) and np.array_equal(i2, info)
    assert job.L.gray_read_raw(path, d2.ctypes.data, i2.ctypes.data, nd - 2, w, h) == api.ESIZE
    assert job.L.gray_read_raw(path, d2.ctypes.data, i2.ctypes.data, nd, h, w) == api.ESIZE
    missing = str(tmp_path / "none.raw").encode()
    assert job.L.gray_read_raw(missing, d2.ctypes.data, i2.ctypes.data, nd, w, h) == api.ENOTFOUND
    with open(path, "r+b") as f:  # cut the info block short
        f.truncate(32 + w * h * nd * 8 + 8)
    assert job.L.gray_read_raw(path, d2.ctypes.data, i2.ctypes.data, nd, w, h) == api.ESIZE


def read_raw(path):
    raw = open(path, "rb").read()
    sz, nd, w, h = (int(x) for x in np.frombuffer(raw[:32], dtype=np.uint64))
    body = np.frombuffer(raw[32:], dtype=np.float64)
    return body[: w * h * nd].reshape(w * h, nd), body[w * h * nd:]


@pytest.mark.gpu
def test_cli_dumps_match_oracle(tmp_path):
    args = ["a=0.9", "r=1000", "i=60", "w=40", "h=40", "W=12", "H=10", "dt=-31.25",
            "n=1000", "N=3", "p=8", "out=" + str(tmp_path / "%04d.raw"),
            "ray=" + str(tmp_path / "ray%04d.h5")]
    res = subprocess.run([CLI] + args, capture_output=True, text=True, timeout=300,
                         cwd=tmp_path)
    assert res.returncode == 0, res.stderr
    assert "3: -62.5 -> -93.8: DONE" in res.stdout
    cfg = dict(a_spin=0.9, r_obs=1000.0, i_obs=60.0, w_img=40.0, h_img=40.0, n_width=12,
               n_height=10, dt_dump=-31.25, n_sub=1000)
    for i in range(4):
        data, info = read_raw(str(tmp_path / ("%04d.raw" % i)))
        if i == 0:
            ref = O.icond(cfg, range(120))
        else:
            ref, _, _ = O.trace(dict(cfg, n_dump=i), np.arange(120))
        assert np.array_equal(data, ref), i
        assert np.max(np.abs(info)) < 1e-9
        # sim/gray.c:170-176: the same rays in /rays of ray%04d.h5 after each interval
        ray = tmp_path / ("ray%04d.h5" % i)
        assert ray.exists() == (i > 0)
        if i > 0:
            with h5.File(str(ray)) as f:
                assert f.info("rays") == ((12, 10, 8), 8)
                assert np.array_equal(f.read("rays").reshape(120, 8), data)


@pytest.mark.gpu
def test_cli_resumes_from_a_dump(tmp_path):
    """i_init=2 with dump 2 on disk continues from it: the later dumps are
    the uninterrupted run's, bit for bit; without the file the run starts
    from the camera as the reference does."""
    common = ["a=0.9", "r=1000", "i=60", "w=40", "h=40", "W=8", "H=6", "dt=-31.25",
              "n=1000", "N=4", "p=8", "ray="]
    full, part = tmp_path / "full", tmp_path / "part"
    full.mkdir()
    part.mkdir()
    res = subprocess.run([CLI] + common + ["out=" + str(full / "%04d.raw")],
                         capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    (part / "0002.raw").write_bytes((full / "0002.raw").read_bytes())
    res = subprocess.run([CLI] + common + ["i0=2", "out=" + str(part / "%04d.raw")],
                         capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    assert "2:  resumed from its dump" in res.stdout
    for i in (3, 4):
        a, _ = read_raw(str(full / ("%04d.raw" % i)))
        b, _ = read_raw(str(part / ("%04d.raw" % i)))
        assert np.array_equal(a, b), i
    assert not (part / "0001.raw").exists()


@pytest.mark.gpu
def test_cli_dump_follows_precision_and_memory_order(tmp_path):
    """sim-org/io.c:52-67 writes the device buffer as it is: p=4 runs dump
    4-byte reals, morder=SoA dumps component-major.  The same p=4 render
    dumped both ways holds the same numbers."""
    common = ["a=0.9", "r=1000", "i=60", "w=40", "h=40", "W=8", "H=6", "dt=-31.25",
              "n=1000", "N=2", "p=4"]
    out = {}
    for mo in ("AoS", "SoA"):
        d = tmp_path / mo
        d.mkdir()
        res = subprocess.run([CLI] + common + ["mo=" + mo, "out=" + str(d / "%04d.raw"),
                                               "ray=" + str(d / "ray%04d.h5")],
                             capture_output=True, text=True, timeout=300)
        assert res.returncode == 0, res.stderr
        raw = (d / "0002.raw").read_bytes()
        hdr = [int(x) for x in np.frombuffer(raw[:32], dtype=np.uint64)]
        assert hdr == [4, 8, 8, 6]
        body = np.frombuffer(raw[32:], dtype=np.float32)
        assert body.size == 48 * 8 + 48
        out[mo] = body[:48 * 8], body[48 * 8:]
    with h5.File(str(tmp_path / "SoA" / "ray0002.h5")) as f:
        assert f.info("rays") == ((8, 6, 8), 4)  # the run's real: float for p=4
        assert np.array_equal(f.read("rays", np.float32).reshape(48, 8),
                              out["AoS"][0].reshape(48, 8))
    aos, soa = out["AoS"][0].reshape(48, 8), out["SoA"][0].reshape(8, 48)
    assert np.array_equal(aos, soa.T) and np.array_equal(out["AoS"][1], out["SoA"][1])
    # and the numbers are the mixed render's, rounded to float
    cfg = dict(a_spin=0.9, r_obs=1000.0, i_obs=60.0, w_img=40.0, h_img=40.0, n_width=8,
               n_height=6, dt_dump=-31.25, n_sub=1000, n_dump=2)
    ref, _, _ = O.trace(cfg, np.arange(48))
    scale = np.abs(ref).max(axis=1, keepdims=True)
    assert np.max(np.abs(aos - ref) / scale) <= 1e-4


def test_dyst_options_and_file_checks_need_no_gpu(job, tmp_path):
    """spacetime=dyst reads dyst_file (sim-org/param.opts:6); a missing or
    unreadable file is refused by init before any device is touched."""
    assert job.conf("st=dyst") == 0 and job.conf("flow=thermal") == 0
    assert job.desc().spacetime == api.ST_NUMERICAL
    assert job.conf("data=" + str(tmp_path / "absent.h5")) == 0
    assert job.init() == api.ENOTFOUND
    bad = tmp_path / "uniform.h5"
    n = 5
    u = np.linspace(-40, 40, n)
    h5.write_spacetime(str(bad), u, u, u, ["0"], [np.zeros((n, n, n, 51), np.float32)])
    assert job.conf("data=" + str(bad)) == 0
    assert job.init() == api.EINVAL  # not on the fisheye map interp.cl assumes


@pytest.mark.gpu
def test_cli_dyst_from_hdf5_file(tmp_path):
    """`gray st=dyst data=file.h5` end to end: a two-snapshot boosted-KS file
    written in the reference's layout, read by the job, streamed through the
    snapshot series; every dump equals the oracle's trace on the same grid
    (reference semantics, in-box camera), and the /rays files hold it too."""
    n, box, t1, t2 = 20, 40.0, -10.0, 0.0
    lv = [O.boosted_ks_grid(n, -box, box, t, a=0.7, v=0.3, axis=1) for t in (t1, t2)]
    xs = O.fisheye_nodes(-box, box, n).astype(np.float32)
    path = str(tmp_path / "data.h5")
    h5.write_spacetime(path, xs, xs, xs, ["-10", "0"], [a.astype(np.float32) for a in lv])
    args = ["st=dyst", "data=" + path, "a=0", "r=30", "i=50", "j=20", "w=30", "h=30",
            "W=8", "H=6", "dt=-2", "N=3", "n=100", "p=8", "out=" + str(tmp_path / "%04d.raw"),
            "ray=" + str(tmp_path / "ray%04d.h5")]
    res = subprocess.run([CLI] + args, capture_output=True, text=True, timeout=300, cwd=tmp_path)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "2 snapshot(s)" in res.stdout and "3: -4.0 -> -6.0: DONE" in res.stdout
    og = O.Grid([a.astype(np.float32) for a in lv], [t1, -box, -box, -box, t2, box, box, box])
    cfg = dict(a_spin=0.0, r_obs=30.0, i_obs=50.0, j_obs=20.0, w_img=30.0, h_img=30.0,
               n_width=8, n_height=6, dt_dump=-2.0, n_sub=100)
    for i in range(1, 4):
        data, _ = read_raw(str(tmp_path / ("%04d.raw" % i)))
        ref, _, _ = O.dyst_trace(dict(cfg, n_dump=i), og, np.arange(48))
        fin = np.all(np.isfinite(ref), axis=1)
        assert np.array_equal(np.all(np.isfinite(data), axis=1), fin)
        err = np.max(np.abs(data[fin] - ref[fin]) / np.abs(ref[fin]).max(axis=1, keepdims=True))
        assert err <= 1e-10, (i, err)
        with h5.File(str(tmp_path / ("ray%04d.h5" % i))) as f:
            assert np.array_equal(f.read("rays").reshape(48, 8), data, equal_nan=True)
