"""ctypes front end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only to check or time against the CUDA path.  The product
package (gray_b200) never imports it.

The C library (oracle/gray_oracle.c) is a plain FP64 restatement of the
reference's OpenCL kernels (luxsrc/gray sim-org/KS.cl, phys.cl, RK4.cl,
driver.cl, rt.cl, interp.cl, dyst.cl); see the citations there.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liborc.so")
MAX_FREQ = 8
TERM_EPS, TERM_RPLUS = 0, 1
FLOW_NONE, FLOW_TORUS = 0, 1


class OrcDesc(ctypes.Structure):
    _fields_ = [
        ("a_spin", ctypes.c_double),
        ("w_img", ctypes.c_double), ("h_img", ctypes.c_double),
        ("r_obs", ctypes.c_double), ("i_obs", ctypes.c_double),
        ("j_obs", ctypes.c_double),
        ("w_rays", ctypes.c_int64), ("h_rays", ctypes.c_int64),
        ("t_init", ctypes.c_double), ("dt_dump", ctypes.c_double),
        ("n_sub", ctypes.c_int64), ("n_dump", ctypes.c_int64),
        ("term", ctypes.c_int),
        ("n_freq", ctypes.c_int),
        ("nu", ctypes.c_double * MAX_FREQ),
        ("flow", ctypes.c_int),
        ("torus_n0", ctypes.c_double), ("torus_kappa", ctypes.c_double),
        ("torus_hr", ctypes.c_double),
        ("m_adm", ctypes.c_double), ("flow_te", ctypes.c_double), ("flow_b", ctypes.c_double),
    ]


FLOW_THERMAL = 2


class OrcGrid(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("box", ctypes.c_float * 8),
        ("fields", ctypes.c_void_p * 2),
        ("bug_gzz", ctypes.c_int),
        ("physics", ctypes.c_int),
    ]


def build():
    """Compile the oracle with its Makefile (plain gcc, no GPU needed)."""
    subprocess.check_call(["make", "-s", "-C", HERE])


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        d, i64 = ctypes.c_double, ctypes.c_int64
        pd, pi64 = P(d), P(i64)
        L.orc_getrr.restype = d
        L.orc_getrr.argtypes = [d, pd]
        L.orc_geteps.restype = d
        L.orc_geteps.argtypes = [d, pd]
        L.orc_down.argtypes = [d, pd, pd, pd]
        L.orc_getuu.restype = d
        L.orc_getuu.argtypes = [d, pd]
        L.orc_ks_rhs.argtypes = [d, pd, pd]
        L.orc_camera.argtypes = [P(OrcDesc), pd]
        L.orc_icond.argtypes = [P(OrcDesc), pd, i64, pd]
        L.orc_getdt.restype = d
        L.orc_getdt.argtypes = [P(OrcDesc), pd, d]
        L.orc_rhs.argtypes = [P(OrcDesc), pd, pd]
        L.orc_integrate.argtypes = [P(OrcDesc), pd, d]
        L.orc_evolve_ray.restype = i64
        L.orc_evolve_ray.argtypes = [P(OrcDesc), pd, d, i64]
        L.orc_trace.restype = ctypes.c_int
        L.orc_trace.argtypes = [P(OrcDesc), pi64, i64, pd, pd, pi64, ctypes.c_int]
        L.orc32_trace.restype = ctypes.c_int
        L.orc32_trace.argtypes = [P(OrcDesc), pi64, i64, pd, pi64, ctypes.c_int]
        L.orc_evolve_states.restype = ctypes.c_int
        L.orc_evolve_states.argtypes = [P(OrcDesc), pd, i64, pd, pi64, ctypes.c_int]
        L.orc_rplus.restype = d
        L.orc_rplus.argtypes = [d]
        L.orc_risco.restype = d
        L.orc_risco.argtypes = [d]
        L.orc_interp.restype = d
        L.orc_interp.argtypes = [P(OrcGrid), pd, ctypes.c_int]
        L.orc_dyst_rhs.argtypes = [P(OrcGrid), pd, pd]
        L.orc_dyst_down.argtypes = [P(OrcGrid), pd, pd, pd]
        L.orc_dyst_icond.argtypes = [P(OrcDesc), pd, i64, pd]
        L.orc_dyst_getdt.restype = d
        L.orc_dyst_getdt.argtypes = [d]
        L.orc_dyst_evolve_ray.restype = i64
        L.orc_dyst_evolve_ray.argtypes = [P(OrcDesc), P(OrcGrid), pd, d, i64]
        L.orc_dyst_trace.restype = ctypes.c_int
        L.orc_dyst_trace.argtypes = [P(OrcDesc), P(OrcGrid), pi64, i64, pd, pd,
                                     pi64, ctypes.c_int]
        L.orc_boosted_ks.argtypes = [d, d, d, ctypes.c_int, pd, pd]
        for name, n in (("orc_log_K2it", 1), ("orc_B_Planck", 2), ("orc_Gaunt", 2),
                        ("orc_L_j_ff", 4), ("orc_L_j_syn", 6)):
            fn = getattr(L, name)
            fn.restype = d
            fn.argtypes = [d] * n
        L.orc_dyst_rhs_rt.argtypes = [P(OrcDesc), P(OrcGrid), pd, pd]
        L.orc_getsphKS.argtypes = [d, pd, ctypes.c_int, pd]
        L.orc_getBL.argtypes = [d, d, pd, ctypes.c_int, pd]
        L.orc_getsphKSu.argtypes = [d, pd, pd, ctypes.c_int, pd]
        L.orc_getBLu.argtypes = [d, pd, pd, ctypes.c_int, pd]
        L.orc_series_schedule.restype = ctypes.c_int
        L.orc_series_schedule.argtypes = [pd, i64, d, d, i64, ctypes.c_int, pi64, pi64]
        L.orc_dyst_series_trace.restype = ctypes.c_int
        L.orc_dyst_series_trace.argtypes = [P(OrcDesc), P(OrcGrid), P(ctypes.c_void_p), pd,
                                            i64, ctypes.c_int, pi64, i64, pd, pd, pi64,
                                            ctypes.c_int]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _pi(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))


def make_desc(cfg):
    """Build an OrcDesc from a plain dict using the .opts field names."""
    d = OrcDesc()
    d.a_spin = cfg.get("a_spin", 0.0)
    d.w_img = cfg.get("w_img", 64.0)
    d.h_img = cfg.get("h_img", 64.0)
    d.r_obs = cfg.get("r_obs", 1024.0)
    d.i_obs = cfg.get("i_obs", 60.0)
    d.j_obs = cfg.get("j_obs", 0.0)
    d.w_rays = cfg.get("n_width", 512)
    d.h_rays = cfg.get("n_height", 512)
    d.t_init = cfg.get("t_init", 0.0)
    d.dt_dump = cfg.get("dt_dump", -32.0)
    d.n_sub = cfg.get("n_sub", 1024)
    d.n_dump = cfg.get("n_dump", 64)
    d.term = cfg.get("term", TERM_EPS)
    nu = list(cfg.get("nu", []))
    d.n_freq = len(nu)
    for i, v in enumerate(nu):
        d.nu[i] = v
    d.flow = cfg.get("flow", FLOW_TORUS if nu else FLOW_NONE)
    d.torus_n0 = cfg.get("torus_n0", 1.0)
    d.torus_kappa = cfg.get("torus_kappa", 1.0)
    d.torus_hr = cfg.get("torus_hr", 0.3)
    d.m_adm = cfg.get("m_adm", 4.3e6)
    d.flow_te = cfg.get("flow_te", 1e12)
    d.flow_b = cfg.get("flow_b", 0.0)
    return d


def n_data(cfg):
    return 8 + 2 * len(cfg.get("nu", []))


def trace(cfg, rays, nthreads=0):
    """icond + every dump interval for the given ray indices.

    Returns (states [n, n_data], info [n], steps [n])."""
    L = lib()
    d = make_desc(cfg)
    rays = np.ascontiguousarray(rays, dtype=np.int64)
    n = rays.size
    out = np.zeros((n, n_data(cfg)))
    info = np.zeros(n)
    steps = np.zeros(n, dtype=np.int64)
    rc = L.orc_trace(ctypes.byref(d), _pi(rays), n, _p(out), _p(info), _pi(steps), nthreads)
    if rc != 0:
        raise ValueError("oracle rejected the configuration")
    return out, info, steps


def trace32(cfg, rays, nthreads=0):
    """The analytic trace with every real in float (gray_oracle32.c, the
    single-precision CPU baseline).  Returns (states [n, n_data], steps [n])."""
    L = lib()
    d = make_desc(cfg)
    rays = np.ascontiguousarray(rays, dtype=np.int64)
    n = rays.size
    out = np.zeros((n, n_data(cfg)))
    steps = np.zeros(n, dtype=np.int64)
    if L.orc32_trace(ctypes.byref(d), _pi(rays), n, _p(out), _pi(steps), nthreads) != 0:
        raise ValueError("oracle rejected the configuration")
    return out, steps


def icond(cfg, rays):
    L = lib()
    d = make_desc(cfg)
    cam = np.zeros(4)
    L.orc_camera(ctypes.byref(d), _p(cam))
    out = np.zeros((len(rays), n_data(cfg)))
    for k, r in enumerate(rays):
        row = np.zeros(n_data(cfg))
        L.orc_icond(ctypes.byref(d), _p(cam), int(r), _p(row))
        out[k] = row
    return out


def ks_rhs(a, s):
    s = np.ascontiguousarray(s, dtype=np.float64)
    ds = np.zeros(8)
    lib().orc_ks_rhs(a, _p(s), _p(ds))
    return ds


def rhs(cfg, s):
    d = make_desc(cfg)
    s = np.ascontiguousarray(s, dtype=np.float64)
    ds = np.zeros_like(s)
    lib().orc_rhs(ctypes.byref(d), _p(s), _p(ds))
    return ds


def integrate(cfg, s, dt):
    d = make_desc(cfg)
    s = np.array(s, dtype=np.float64)
    lib().orc_integrate(ctypes.byref(d), _p(s), dt)
    return s


def down(a, q, u):
    q = np.ascontiguousarray(q, dtype=np.float64)
    u = np.ascontiguousarray(u, dtype=np.float64)
    k = np.zeros(4)
    lib().orc_down(a, _p(q), _p(u), _p(k))
    return k


def getuu(a, s):
    s = np.ascontiguousarray(s, dtype=np.float64)
    return lib().orc_getuu(a, _p(s))


def getrr(a, q):
    q = np.ascontiguousarray(q, dtype=np.float64)
    return lib().orc_getrr(a, _p(q))


def geteps(a, q):
    q = np.ascontiguousarray(q, dtype=np.float64)
    return lib().orc_geteps(a, _p(q))


def getdt(cfg, q, dt):
    d = make_desc(cfg)
    q = np.ascontiguousarray(q, dtype=np.float64)
    return lib().orc_getdt(ctypes.byref(d), _p(q), dt)


def rplus(a):
    return lib().orc_rplus(a)


def risco(a):
    return lib().orc_risco(a)


def boosted_ks(m, a, v, axis, q):
    q = np.ascontiguousarray(q, dtype=np.float64)
    out = np.zeros(50)
    lib().orc_boosted_ks(m, a, v, axis, _p(q), _p(out))
    return out


# ---------------------------------------------------------------- grids

class Grid:
    """Keeps the numpy field arrays alive next to the OrcGrid struct."""

    def __init__(self, fields, box, bug_gzz=False, physics=False):
        self.fields = [np.ascontiguousarray(f, dtype=np.float32) for f in fields]
        nz, ny, nx, nc = self.fields[0].shape
        assert nc == 51
        g = OrcGrid()
        g.nx, g.ny, g.nz = nx, ny, nz
        for i in range(8):
            g.box[i] = box[i]
        g.fields[0] = self.fields[0].ctypes.data
        g.fields[1] = self.fields[-1].ctypes.data
        g.bug_gzz = int(bug_gzz)
        g.physics = int(physics)
        self.g = g


def fisheye_nodes(lo, hi, n):
    """Fisheye node coordinates x = sinh((A i + B)^3) (tools/generate_data.py:49-58)."""
    B = np.cbrt(np.arcsinh(lo))
    A = (np.cbrt(np.arcsinh(hi)) - B) / (n - 1)
    f = A * np.arange(n) + B
    return np.sinh(f * f * f)


def boosted_ks_grid(n, lo, hi, t, m=1.0, a=0.7, v=0.3, axis=1, rho=True):
    """Sample the boosted KS fields on a fisheye grid (slow, for small n).
    n, lo, hi are numbers (a cube) or (x, y, z) triples."""
    n3 = (n,) * 3 if np.isscalar(n) else tuple(n)
    lo3 = (lo,) * 3 if np.isscalar(lo) else tuple(lo)
    hi3 = (hi,) * 3 if np.isscalar(hi) else tuple(hi)
    ax = [fisheye_nodes(lo3[c], hi3[c], n3[c]) for c in range(3)]
    out = np.zeros((n3[2], n3[1], n3[0], 51), dtype=np.float64)
    L = lib()
    q = np.zeros(4)
    buf = np.zeros(50)
    # the origin node (odd n) gives rho = 1/0 = inf, as tools/generate_data.py does
    with np.errstate(divide="ignore", over="ignore", invalid="ignore"):
        for k, z in enumerate(ax[2]):
            for j, y in enumerate(ax[1]):
                for i, x in enumerate(ax[0]):
                    q[:] = (t, x, y, z)
                    L.orc_boosted_ks(m, a, v, axis, _p(q), _p(buf))
                    out[k, j, i, :50] = buf
                    out[k, j, i, 50] = 1.0 / np.sqrt(x * x + y * y + z * z) if rho else 0.0
        out = np.nan_to_num(out)
        return out.astype(np.float32)


def dyst_rhs(grid, s):
    s = np.ascontiguousarray(s, dtype=np.float64)
    ds = np.zeros(8)
    lib().orc_dyst_rhs(ctypes.byref(grid.g), _p(s), _p(ds))
    return ds


def _dyst_desc(cfg):
    """Numerical renders carry the thermal flow when they have frequencies."""
    if cfg.get("nu") and "flow" not in cfg:
        cfg = dict(cfg, flow=FLOW_THERMAL)
    return make_desc(cfg)


def dyst_rhs_rt(cfg, grid, s):
    """Geodesic and thermal-transfer RHS at state s (8 + 2 n_freq)."""
    d = _dyst_desc(cfg)
    s = np.ascontiguousarray(s, dtype=np.float64)
    ds = np.zeros(8 + 2 * d.n_freq)
    lib().orc_dyst_rhs_rt(ctypes.byref(d), ctypes.byref(grid.g), _p(s), _p(ds))
    return ds


def dyst_trace(cfg, grid, rays, nthreads=0):
    L = lib()
    d = _dyst_desc(cfg)
    rays = np.ascontiguousarray(rays, dtype=np.int64)
    n = rays.size
    out = np.zeros((n, n_data(cfg)))
    info = np.zeros(n)
    steps = np.zeros(n, dtype=np.int64)
    rc = L.orc_dyst_trace(ctypes.byref(d), ctypes.byref(grid.g), _pi(rays), n, _p(out),
                          _p(info), _pi(steps), nthreads)
    if rc != 0:
        raise ValueError("oracle rejected the configuration")
    return out, info, steps


def emissivities():
    """The rt.cl emissivity functions of the oracle, by name."""
    L = lib()
    return {"log_K2it": L.orc_log_K2it, "B_Planck": L.orc_B_Planck, "Gaunt": L.orc_Gaunt,
            "L_j_ff": L.orc_L_j_ff, "L_j_syn": L.orc_L_j_syn}


def series_schedule(times, t_init, dt_dump, n_dump, fast_light=False):
    """Snapshot pair of t_init and of each dump interval (sim-org/gray.c:41-57,
    183-293), or None where the reference stops."""
    t = np.ascontiguousarray(times, dtype=np.float64)
    first = np.zeros(1, dtype=np.int64)
    pairs = np.zeros(max(n_dump, 1), dtype=np.int64)
    rc = lib().orc_series_schedule(_p(t), t.size, float(t_init), float(dt_dump), int(n_dump),
                                   int(bool(fast_light)), _pi(first), _pi(pairs))
    return None if rc else (int(first[0]), pairs[:n_dump].copy())


def dyst_series_trace(cfg, snaps, times, lo, hi, rays, physics=False, bug_gzz=False,
                      fast_light=False, nthreads=0):
    """dyst trace across a snapshot series (snaps[k]: [nz][ny][nx][51] at times[k]);
    every interval runs on the pair sim-org/gray.c chooses for it."""
    L = lib()
    d = _dyst_desc(cfg)
    snaps = [np.ascontiguousarray(a, dtype=np.float32) for a in snaps]
    nz, ny, nx, _ = snaps[0].shape
    g = OrcGrid()
    g.nx, g.ny, g.nz = nx, ny, nz
    for i, v in enumerate([0.0, lo, lo, lo, 0.0, hi, hi, hi]):
        g.box[i] = v
    g.bug_gzz, g.physics = int(bug_gzz), int(physics)
    ptrs = (ctypes.c_void_p * len(snaps))(*[a.ctypes.data for a in snaps])
    t = np.ascontiguousarray(times, dtype=np.float64)
    rays = np.ascontiguousarray(rays, dtype=np.int64)
    n = rays.size
    out = np.zeros((n, n_data(cfg)))
    info = np.zeros(n)
    steps = np.zeros(n, dtype=np.int64)
    rc = L.orc_dyst_series_trace(ctypes.byref(d), ctypes.byref(g), ptrs, _p(t), t.size,
                                 int(bool(fast_light)), _pi(rays), n, _p(out), _p(info),
                                 _pi(steps), nthreads)
    if rc != 0:
        raise ValueError("oracle rejected the series")
    return out, info, steps


def coords(a, s, system="bl", r_match=10.0, as_written=False):
    """Output coordinates of one 8-component KS state (KS.cl:63-153):
    (t, r, theta, phi, u^t, u^r, u^theta, u^phi) in spherical KS ("sph")
    or Boyer-Lindquist ("bl")."""
    L = lib()
    s = np.ascontiguousarray(s, dtype=np.float64)
    q, u = np.ascontiguousarray(s[:4]), np.ascontiguousarray(s[4:8])
    x, v = np.zeros(4), np.zeros(4)
    w = int(bool(as_written))
    if system == "sph":
        L.orc_getsphKS(a, _p(q), w, _p(x))
        L.orc_getsphKSu(a, _p(q), _p(u), w, _p(v))
    else:
        L.orc_getBL(a, r_match, _p(q), w, _p(x))
        L.orc_getBLu(a, _p(q), _p(u), w, _p(v))
    return np.r_[x, v]


# ---------------------------------------------------------------------------
# The reference's own kernel sources built for the CPU (oracle/_ref, see
# oracle/ref_shim): the pins of the restatement above.  Present only where
# the reference tree was available at build time.

REF_DIR = os.path.join(HERE, "_ref")
_ref = {}


def ref_available():
    return all(os.path.exists(os.path.join(REF_DIR, f))
               for f in ("libref_ks.so", "libref_dyst.so"))


def _reflib(name):
    if name not in _ref:
        _ref[name] = ctypes.CDLL(os.path.join(REF_DIR, name))
    return _ref[name]


class RefKsDesc(ctypes.Structure):
    _fields_ = ([(n, ctypes.c_double) for n in ("a_spin", "w_img", "h_img", "r_obs", "i_obs",
                                                "j_obs")] +
                [("w_rays", ctypes.c_int64), ("h_rays", ctypes.c_int64),
                 ("t_init", ctypes.c_double), ("dt_dump", ctypes.c_double),
                 ("n_sub", ctypes.c_int64), ("n_dump", ctypes.c_int64)])


class RefDystDesc(ctypes.Structure):
    _fields_ = ([(n, ctypes.c_double) for n in ("w_img", "h_img", "r_obs", "i_obs", "j_obs")] +
                [("w_rays", ctypes.c_int64), ("h_rays", ctypes.c_int64),
                 ("t_init", ctypes.c_double), ("dt_dump", ctypes.c_double),
                 ("n_sub", ctypes.c_int64), ("n_dump", ctypes.c_int64),
                 ("nu", ctypes.c_double), ("m_adm", ctypes.c_double),
                 ("box", ctypes.c_double * 8), ("nx", ctypes.c_int), ("ny", ctypes.c_int),
                 ("nz", ctypes.c_int)])


def ref_ks_rhs(a, s):
    """KS.cl gr_rhs() itself at state s[8]."""
    L = _reflib("libref_ks.so")
    s = np.ascontiguousarray(s, dtype=np.float64)
    ds = np.zeros(8)
    L.ref_ks_rhs(ctypes.c_double(a), _p(s), _p(ds))
    return ds


def ref_ks_func(name, a, q, u=None):
    """KS.cl getrr / geteps (scalar) or down (4-vector) itself."""
    L = _reflib("libref_ks.so")
    q = np.ascontiguousarray(q, dtype=np.float64)
    if name == "down":
        u = np.ascontiguousarray(u, dtype=np.float64)
        k = np.zeros(4)
        L.ref_ks_down(ctypes.c_double(a), _p(q), _p(u), _p(k))
        return k
    f = getattr(L, "ref_ks_" + name)
    f.restype = ctypes.c_double
    return f(ctypes.c_double(a), _p(q))


def ref_ks_trace(cfg, rays, nthreads=1, with_steps=False):
    """icond_drv + evolve_drv of the reference's analytic program over the
    listed rays on nthreads host threads (0: all): (states [n, 8], info [n])
    and, with_steps, the accepted RK4 steps of each ray."""
    L = _reflib("libref_ks.so")
    d = RefKsDesc(cfg.get("a_spin", 0.0), cfg.get("w_img", 64.0), cfg.get("h_img", 64.0),
                  cfg.get("r_obs", 1024.0), cfg.get("i_obs", 60.0), cfg.get("j_obs", 0.0),
                  cfg["n_width"], cfg["n_height"], cfg.get("t_init", 0.0),
                  cfg.get("dt_dump", -32.0), cfg.get("n_sub", 1024), cfg.get("n_dump", 64))
    rays = np.ascontiguousarray(rays, dtype=np.int64)
    out, info = np.zeros((rays.size, 8)), np.zeros(rays.size)
    steps = np.zeros(rays.size, dtype=np.int64)
    if nthreads <= 0:
        nthreads = os.cpu_count() or 1
    if L.ref_ks_trace(ctypes.byref(d), _pi(rays), ctypes.c_int64(rays.size), _p(out),
                      _p(info), _pi(steps), ctypes.c_int(nthreads)) != 0:
        raise ValueError("ray index outside the image")
    return (out, info, steps) if with_steps else (out, info)


def ref_dyst_trace(cfg, levels, box, rays):
    """icond_drv + evolve_drv of the reference's numerical-spacetime program
    with one frequency of thermal transfer (flow.cl's template flow, rt.cl's
    emissivities): (states [n, 10], info [n]).  levels are two [nz, ny, nx,
    51] float32 arrays at box[0] and box[4]."""
    L = _reflib("libref_dyst.so")
    lv = [np.ascontiguousarray(a, dtype=np.float32) for a in levels]
    nz, ny, nx, _ = lv[0].shape
    d = RefDystDesc(cfg.get("w_img", 64.0), cfg.get("h_img", 64.0), cfg.get("r_obs", 1024.0),
                    cfg.get("i_obs", 60.0), cfg.get("j_obs", 0.0), cfg["n_width"],
                    cfg["n_height"], cfg.get("t_init", 0.0), cfg.get("dt_dump", -32.0),
                    cfg.get("n_sub", 1024), cfg.get("n_dump", 64), cfg["nu"][0],
                    cfg.get("m_adm", 4.3e6), (ctypes.c_double * 8)(*box), nx, ny, nz)
    rays = np.ascontiguousarray(rays, dtype=np.int64)
    out, info = np.zeros((rays.size, 10)), np.zeros(rays.size)
    if L.ref_dyst_trace(ctypes.byref(d), ctypes.c_void_p(lv[0].ctypes.data),
                        ctypes.c_void_p(lv[1].ctypes.data), _pi(rays),
                        ctypes.c_int64(rays.size), _p(out), _p(info)) != 0:
        raise ValueError("ray index outside the image")
    return out, info
