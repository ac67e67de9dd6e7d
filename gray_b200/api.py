"""Python view of the C ABI in include/gray_cuda.h (ctypes, no torch types).

This mirrors the lux-job surface of the reference (sim/gray.opts,
sim/Kerr.opts, sim/infcam.opts, sim-org/setup.opts, sim-org/param.opts):
a RenderDesc carries the same run-time parameter names, and Context.run()
does what sim-org/gray.c:_exec does for the analytic spacetime (icond, then
one evolve per dump interval) on the GPU.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libgray_cuda.so")
MAX_FREQ = 8
ABI_VERSION = 3  # GRAY_ABI_VERSION of include/gray_cuda.h

OK, EINVAL, ENOMEM, ECUDA, ENODEV, EBUDGET, ETIMEOUT, ENOTFOUND, ESTATE, ESIZE, ESOURCE = (
    0, -1, -2, -3, -4, -5, -6, -7, -8, -9, -10)
PREC_FP64, PREC_MIXED = 0, 1
ST_KERR, ST_NUMERICAL = 0, 1
FLOW_NONE, FLOW_TORUS, FLOW_THERMAL = 0, 1, 2
TERM_EPS, TERM_RPLUS = 0, 1
LAYOUT_SOA, LAYOUT_AOS = 0, 1
COORDS_SPH_KS, COORDS_BL = 0, 1
COORDS_AS_WRITTEN = 1

# Every symbol include/gray_cuda.h declares.
EXPORTS = [
    "gray_strerror", "gray_abi_version", "gray_create", "gray_destroy",
    "gray_set_stream", "gray_sync", "gray_hbm_used", "gray_render_create",
    "gray_render_destroy", "gray_icond", "gray_evolve", "gray_run", "gray_evolve_all",
    "gray_read_state", "gray_write_state", "gray_read_kdown", "gray_read_coords",
    "gray_ray_steps",
    "gray_gather_steps",
    "gray_load_spacetime", "gray_load_spacetime_interleaved",
    "gray_make_boosted_ks", "gray_swap_levels", "gray_measure_peak",
    "gray_run_mixed_noalloc", "gray_read_spacetime",
    "gray_series_schedule", "gray_run_series",
    "gray_batch_create", "gray_batch_destroy", "gray_batch_run", "gray_batch_steps",
    "gray_plan", "gray_set_plan", "gray_get_plan",
    "gray_serve_clock", "gray_serve_start", "gray_serve_submit", "gray_serve_poll",
    "gray_serve_result", "gray_serve_cancel", "gray_serve_get_stats", "gray_serve_stop",
]
REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED, REQ_CANCELLED = 0, 1, 2, 3, 4
PLAN_ESTIMATE, PLAN_MEASURE = 0, 1
NOALLOC_MAX_RENDERS = 32


class GrayError(RuntimeError):
    def __init__(self, status, what):
        super().__init__("%s: %s (%d)" % (what, strerror(status), status))
        self.status = status


class RenderDesc(ctypes.Structure):
    _fields_ = [
        ("m_bh", ctypes.c_double), ("a_spin", ctypes.c_double),
        ("w_img", ctypes.c_double), ("h_img", ctypes.c_double),
        ("r_obs", ctypes.c_double), ("i_obs", ctypes.c_double),
        ("j_obs", ctypes.c_double),
        ("n_width", ctypes.c_uint64), ("n_height", ctypes.c_uint64),
        ("t_init", ctypes.c_double), ("dt_dump", ctypes.c_double),
        ("n_sub", ctypes.c_uint64), ("n_dump", ctypes.c_uint64),
        ("term", ctypes.c_int32),
        ("n_freq", ctypes.c_int32), ("nu", ctypes.c_double * MAX_FREQ),
        ("flow", ctypes.c_int32),
        ("torus_n0", ctypes.c_double), ("torus_kappa", ctypes.c_double),
        ("torus_hr", ctypes.c_double),
        ("spacetime", ctypes.c_int32), ("precision", ctypes.c_int32),
        ("m_adm", ctypes.c_double), ("flow_te", ctypes.c_double),
        ("flow_b", ctypes.c_double),
        ("row_begin", ctypes.c_uint64), ("n_rows", ctypes.c_uint64),
    ]


class LaunchPlan(ctypes.Structure):
    _fields_ = [("block", ctypes.c_int32), ("blocks_per_sm", ctypes.c_int32),
                ("rays_per_thread", ctypes.c_int32), ("rk4_rolled", ctypes.c_int32),
                ("ns", ctypes.c_double)]

    def as_dict(self):
        return {"block": self.block, "blocks_per_sm": self.blocks_per_sm,
                "rays_per_thread": self.rays_per_thread, "rk4_rolled": self.rk4_rolled,
                "trial_ns": self.ns}


class ServeConfig(ctypes.Structure):
    _fields_ = [("hbm_budget", ctypes.c_size_t), ("max_inflight", ctypes.c_int32),
                ("dumps_per_iter", ctypes.c_int32)]


class RequestStatus(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int32), ("status", ctypes.c_int32),
                ("t_submit", ctypes.c_double), ("t_admit", ctypes.c_double),
                ("t_done", ctypes.c_double), ("n_rays", ctypes.c_uint64)]


class ServeStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_uint64), ("ray_steps", ctypes.c_uint64 * 2),
                ("completed", ctypes.c_uint64), ("failed", ctypes.c_uint64),
                ("cancelled", ctypes.c_uint64), ("busy_s", ctypes.c_double)]


class GridDesc(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("box", ctypes.c_float * 8),
        ("bug_gzz", ctypes.c_int32), ("physics", ctypes.c_int32),
    ]


LOAD_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64,
                           ctypes.POINTER(ctypes.c_float))
DUMP_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64)


class SnapshotSource(ctypes.Structure):
    _fields_ = [("n_times", ctypes.c_uint64), ("times", ctypes.POINTER(ctypes.c_double)),
                ("user", ctypes.c_void_p), ("load", LOAD_FN)]


# Reference defaults (sim/gray.opts, sim/Kerr.opts, sim/infcam.opts,
# sim-org/setup.opts, sim-org/param.opts M_ADM; flow.cl:51-52 te and b).
DEFAULTS = dict(m_bh=4e6, a_spin=0.0, w_img=64.0, h_img=64.0, r_obs=1024.0,
                i_obs=60.0, j_obs=0.0, n_width=512, n_height=512, t_init=0.0,
                dt_dump=-32.0, n_sub=1024, n_dump=64, term=TERM_EPS, nu=(),
                flow=None, torus_n0=1.0, torus_kappa=1.0, torus_hr=0.3,
                spacetime=ST_KERR, precision=PREC_FP64, m_adm=4.3e6,
                flow_te=1e12, flow_b=0.0, row_begin=0, n_rows=0)


def make_desc(cfg):
    c = dict(DEFAULTS)
    c.update(cfg)
    d = RenderDesc()
    for k in ("m_bh", "a_spin", "w_img", "h_img", "r_obs", "i_obs", "j_obs",
              "t_init", "dt_dump", "torus_n0", "torus_kappa", "torus_hr",
              "m_adm", "flow_te", "flow_b"):
        setattr(d, k, float(c[k]))
    for k in ("n_width", "n_height", "n_sub", "n_dump", "term", "spacetime", "precision",
              "row_begin", "n_rows"):
        setattr(d, k, int(c[k]))
    nu = list(c["nu"])
    if len(nu) > MAX_FREQ:
        raise ValueError("at most %d frequencies" % MAX_FREQ)
    d.n_freq = len(nu)
    for i, v in enumerate(nu):
        d.nu[i] = float(v)
    flow = c["flow"]
    if flow is None:  # the transfer model each spacetime carries
        flow = (FLOW_NONE if not nu else
                FLOW_THERMAL if d.spacetime == ST_NUMERICAL else FLOW_TORUS)
    d.flow = int(flow)
    return d


_lib = None


def lib():
    """Load libgray_cuda.so; raise loudly when it is missing (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                "libgray_cuda.so is not built (%s); run __graft_entry__.build()" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        vp, i, sz, d, u64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t, ctypes.c_double, ctypes.c_uint64
        L.gray_strerror.restype = ctypes.c_char_p
        L.gray_strerror.argtypes = [i]
        L.gray_abi_version.restype = i
        L.gray_create.restype = vp
        L.gray_create.argtypes = [i, sz, P(i)]
        L.gray_destroy.argtypes = [vp]
        L.gray_destroy.restype = None
        L.gray_set_stream.argtypes = [vp, vp]
        L.gray_sync.argtypes = [vp]
        L.gray_hbm_used.restype = sz
        L.gray_hbm_used.argtypes = [vp]
        L.gray_render_create.argtypes = [vp, P(RenderDesc), P(i)]
        L.gray_render_destroy.argtypes = [vp, i]
        L.gray_icond.argtypes = [vp, i]
        L.gray_evolve.argtypes = [vp, i, d, d, u64, P(d)]
        L.gray_run.argtypes = [vp, i, P(d)]
        L.gray_evolve_all.argtypes = [vp, i, P(d)]
        L.gray_read_state.argtypes = [vp, i, vp, sz, vp, sz, i]
        L.gray_write_state.argtypes = [vp, i, vp, sz, i]
        L.gray_read_kdown.argtypes = [vp, i, vp, sz]
        L.gray_read_coords.argtypes = [vp, i, i, d, i, vp, sz]
        L.gray_ray_steps.argtypes = [vp, i, P(u64)]
        L.gray_gather_steps.argtypes = [vp, i, P(u64)]
        L.gray_load_spacetime.argtypes = [vp, P(GridDesc), P(ctypes.c_void_p), i]
        L.gray_load_spacetime_interleaved.argtypes = [vp, P(GridDesc), vp, i]
        L.gray_make_boosted_ks.argtypes = [vp, P(GridDesc), d, d, i, d, i]
        L.gray_swap_levels.argtypes = [vp]
        L.gray_measure_peak.argtypes = [vp, i, P(d)]
        L.gray_run_mixed_noalloc.argtypes = [i, P(RenderDesc), i, P(vp), P(vp), vp, P(u64)]
        L.gray_read_spacetime.argtypes = [vp, i, vp, sz]
        L.gray_batch_create.argtypes = [vp, P(i), i, P(i)]
        L.gray_batch_destroy.argtypes = [vp, i]
        L.gray_batch_run.argtypes = [vp, i, P(d)]
        L.gray_batch_steps.argtypes = [vp, i, P(u64)]
        L.gray_plan.argtypes = [vp, i, i, P(LaunchPlan)]
        L.gray_set_plan.argtypes = [vp, P(LaunchPlan)]
        L.gray_get_plan.argtypes = [vp, P(LaunchPlan)]
        L.gray_serve_clock.restype = d
        L.gray_serve_clock.argtypes = []
        L.gray_serve_start.argtypes = [vp, P(ServeConfig)]
        L.gray_serve_submit.argtypes = [vp, P(RenderDesc), P(u64)]
        L.gray_serve_poll.argtypes = [vp, u64, P(RequestStatus)]
        L.gray_serve_result.argtypes = [vp, u64, vp, sz, vp, sz]
        L.gray_serve_cancel.argtypes = [vp, u64]
        L.gray_serve_get_stats.argtypes = [vp, P(ServeStats)]
        L.gray_serve_stop.argtypes = [vp, i]
        L.gray_series_schedule.argtypes = [P(d), u64, d, d, u64, i, P(ctypes.c_int64)]
        L.gray_run_series.argtypes = [vp, i, P(GridDesc), P(SnapshotSource), i, DUMP_FN,
                                      P(d), P(u64)]
        if L.gray_abi_version() != ABI_VERSION:
            raise RuntimeError("libgray_cuda.so has ABI %d, this module expects %d; rebuild"
                               % (L.gray_abi_version(), ABI_VERSION))
        _lib = L
    return _lib


def strerror(status):
    return lib().gray_strerror(status).decode()


def _ck(status, what):
    if status != OK:
        raise GrayError(status, what)


def make_grid(n, lo, hi, t1=0.0, t2=0.0, bug_gzz=False, physics=False):
    g = GridDesc()
    g.nx, g.ny, g.nz = (n, n, n) if isinstance(n, int) else n
    lo3 = (lo,) * 3 if not hasattr(lo, "__len__") else lo
    hi3 = (hi,) * 3 if not hasattr(hi, "__len__") else hi
    box = [t1, lo3[0], lo3[1], lo3[2], t2, hi3[0], hi3[1], hi3[2]]
    for k in range(8):
        g.box[k] = box[k]
    g.bug_gzz = int(bug_gzz)
    g.physics = int(physics)
    return g


class Render:
    def __init__(self, ctx, cfg):
        self.ctx = ctx
        self.desc = make_desc(cfg)
        rid = ctypes.c_int(0)
        _ck(lib().gray_render_create(ctx.h, ctypes.byref(self.desc), ctypes.byref(rid)),
            "gray_render_create")
        self.id = rid.value
        self.n_rays = self.desc.n_width * (self.desc.n_rows or self.desc.n_height)
        self.n_data = 8 + 2 * self.desc.n_freq

    def icond(self):
        _ck(lib().gray_icond(self.ctx.h, self.id), "gray_icond")

    def evolve(self, t, target, n_sub=None, wait=True):
        ns = ctypes.c_double(0.0)
        n_sub = self.desc.n_sub if n_sub is None else n_sub
        _ck(lib().gray_evolve(self.ctx.h, self.id, t, target, n_sub,
                              ctypes.byref(ns) if wait else None), "gray_evolve")
        return ns.value

    def run(self, wait=True):
        ns = ctypes.c_double(0.0)
        _ck(lib().gray_run(self.ctx.h, self.id, ctypes.byref(ns) if wait else None),
            "gray_run")
        return ns.value

    def evolve_all(self, wait=True):
        ns = ctypes.c_double(0.0)
        _ck(lib().gray_evolve_all(self.ctx.h, self.id, ctypes.byref(ns) if wait else None),
            "gray_evolve_all")
        return ns.value

    def state(self, layout=LAYOUT_SOA, out=None, info_out=None):
        if out is None:
            shape = (self.n_data, self.n_rays) if layout == LAYOUT_SOA else (self.n_rays, self.n_data)
            out = np.empty(shape, dtype=np.float64)
        if info_out is None:
            info_out = np.empty(self.n_rays, dtype=np.float64)
        _ck(lib().gray_read_state(self.ctx.h, self.id, out.ctypes.data, out.nbytes,
                                  info_out.ctypes.data, info_out.nbytes, layout),
            "gray_read_state")
        return out, info_out

    def write_state(self, data, layout=LAYOUT_SOA):
        data = np.ascontiguousarray(data, dtype=np.float64)
        _ck(lib().gray_write_state(self.ctx.h, self.id, data.ctypes.data, data.nbytes, layout),
            "gray_write_state")

    def kdown(self):
        k = np.empty((4, self.n_rays), dtype=np.float64)
        _ck(lib().gray_read_kdown(self.ctx.h, self.id, k.ctypes.data, k.nbytes), "gray_read_kdown")
        return k

    def coords(self, system=COORDS_BL, r_match=10.0, flags=0):
        """(8, n_rays): t, r, theta, phi, u^t, u^r, u^theta, u^phi (KS.cl:63-153)."""
        out = np.empty((8, self.n_rays), dtype=np.float64)
        _ck(lib().gray_read_coords(self.ctx.h, self.id, system, float(r_match), flags,
                                   out.ctypes.data, out.nbytes), "gray_read_coords")
        return out

    def steps(self):
        v = ctypes.c_uint64(0)
        _ck(lib().gray_ray_steps(self.ctx.h, self.id, ctypes.byref(v)), "gray_ray_steps")
        return v.value

    def gather_steps(self):
        v = ctypes.c_uint64(0)
        _ck(lib().gray_gather_steps(self.ctx.h, self.id, ctypes.byref(v)), "gray_gather_steps")
        return v.value

    def run_series(self, grid, times, load, fast_light=False, after_dump=None):
        """icond + every dump interval across a snapshot series
        (gray_run_series).  load(k) returns snapshot k as nz*ny*nx*51 floats
        (interleaved, or [z][y][x][51]); after_dump(i), if given, runs after
        interval i.  Returns (device ns, number of load calls)."""
        times = np.ascontiguousarray(times, dtype=np.float64)
        npts = grid.nx * grid.ny * grid.nz
        err = []

        def _load(user, k, fields):
            try:
                a = np.ascontiguousarray(load(int(k)), dtype=np.float32).reshape(-1)
                if a.size != npts * 51:
                    raise ValueError("snapshot %d has %d floats, want %d" % (k, a.size, npts * 51))
                ctypes.memmove(fields, a.ctypes.data, a.nbytes)
                return 0
            except Exception as e:  # reported after the call returns
                err.append(e)
                return 1

        def _dump(user, i):
            try:
                after_dump(int(i))
                return 0
            except Exception as e:
                err.append(e)
                return 1

        load_cb = LOAD_FN(_load)
        dump_cb = DUMP_FN(_dump) if after_dump else DUMP_FN()
        src = SnapshotSource(times.size, times.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                             None, load_cb)
        ns = ctypes.c_double(0.0)
        loads = ctypes.c_uint64(0)
        st = lib().gray_run_series(self.ctx.h, self.id, ctypes.byref(grid), ctypes.byref(src),
                                   int(bool(fast_light)), dump_cb, ctypes.byref(ns),
                                   ctypes.byref(loads))
        if err:
            raise err[0]
        _ck(st, "gray_run_series")
        return ns.value, loads.value

    def close(self):
        if self.id:
            lib().gray_render_destroy(self.ctx.h, self.id)
            self.id = 0


def series_schedule(times, t_init, dt_dump, n_dump, fast_light=False):
    """The snapshot pair of each dump interval (gray_series_schedule)."""
    times = np.ascontiguousarray(times, dtype=np.float64)
    pairs = np.zeros(max(int(n_dump), 1), dtype=np.int64)
    _ck(lib().gray_series_schedule(times.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                   times.size, float(t_init), float(dt_dump), int(n_dump),
                                   int(bool(fast_light)),
                                   pairs.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))),
        "gray_series_schedule")
    return pairs[:int(n_dump)]


class Batch:
    """Many mixed-precision renders in one persistent launch (graph-replayed)."""

    def __init__(self, ctx, renders):
        self.ctx = ctx
        self.renders = list(renders)
        ids = (ctypes.c_int * len(self.renders))(*[r.id for r in self.renders])
        bid = ctypes.c_int(0)
        _ck(lib().gray_batch_create(ctx.h, ids, len(self.renders), ctypes.byref(bid)),
            "gray_batch_create")
        self.id = bid.value

    def run(self, wait=True):
        ns = ctypes.c_double(0.0)
        _ck(lib().gray_batch_run(self.ctx.h, self.id, ctypes.byref(ns) if wait else None),
            "gray_batch_run")
        return ns.value

    def steps(self):
        v = ctypes.c_uint64(0)
        _ck(lib().gray_batch_steps(self.ctx.h, self.id, ctypes.byref(v)), "gray_batch_steps")
        return v.value

    def close(self):
        if self.id:
            lib().gray_batch_destroy(self.ctx.h, self.id)
            self.id = 0


class Context:
    """One CUDA device; owns every device allocation (gray_create)."""

    def __init__(self, device=0, hbm_budget=0):
        st = ctypes.c_int(0)
        h = lib().gray_create(device, hbm_budget, ctypes.byref(st))
        if not h:
            raise GrayError(st.value, "gray_create")
        self.h = h

    def render(self, cfg):
        return Render(self, cfg)

    def set_stream(self, stream_ptr):
        _ck(lib().gray_set_stream(self.h, stream_ptr), "gray_set_stream")

    def sync(self):
        _ck(lib().gray_sync(self.h), "gray_sync")

    def hbm_used(self):
        return lib().gray_hbm_used(self.h)

    def load_spacetime(self, grid, fields, level):
        """fields: [nz, ny, nx, 51] float32 array (interleaved) or a list of
        51 [nz, ny, nx] arrays in io.c order."""
        if isinstance(fields, np.ndarray):
            f = np.ascontiguousarray(fields, dtype=np.float32)
            _ck(lib().gray_load_spacetime_interleaved(self.h, ctypes.byref(grid),
                                                      f.ctypes.data, level),
                "gray_load_spacetime_interleaved")
        else:
            arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in fields]
            ptrs = (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
            _ck(lib().gray_load_spacetime(self.h, ctypes.byref(grid), ptrs, level),
                "gray_load_spacetime")

    def make_boosted_ks(self, grid, a, v, axis, t, level):
        _ck(lib().gray_make_boosted_ks(self.h, ctypes.byref(grid), a, v, axis, t, level),
            "gray_make_boosted_ks")

    def measure_peak(self, precision):
        v = ctypes.c_double(0.0)
        _ck(lib().gray_measure_peak(self.h, precision, ctypes.byref(v)), "gray_measure_peak")
        return v.value

    def batch(self, renders):
        return Batch(self, renders)

    def plan(self, batch, flags=PLAN_MEASURE):
        p = LaunchPlan()
        _ck(lib().gray_plan(self.h, batch.id, flags, ctypes.byref(p)), "gray_plan")
        return p

    def set_plan(self, block, blocks_per_sm=0, rays_per_thread=2, rk4_rolled=0):
        p = LaunchPlan(block, blocks_per_sm, rays_per_thread, rk4_rolled, 0.0)
        _ck(lib().gray_set_plan(self.h, ctypes.byref(p)), "gray_set_plan")

    def get_plan(self):
        p = LaunchPlan()
        _ck(lib().gray_get_plan(self.h, ctypes.byref(p)), "gray_get_plan")
        return p

    # ---- serving (continuous batching)
    def serve_start(self, hbm_budget=0, max_inflight=0, dumps_per_iter=0):
        cfg = ServeConfig(hbm_budget, max_inflight, dumps_per_iter)
        _ck(lib().gray_serve_start(self.h, ctypes.byref(cfg)), "gray_serve_start")

    def submit(self, cfg):
        d = make_desc(dict(cfg, precision=cfg.get("precision", PREC_MIXED)))
        rid = ctypes.c_uint64(0)
        _ck(lib().gray_serve_submit(self.h, ctypes.byref(d), ctypes.byref(rid)), "gray_serve_submit")
        return rid.value

    def poll(self, rid):
        s = RequestStatus()
        _ck(lib().gray_serve_poll(self.h, rid, ctypes.byref(s)), "gray_serve_poll")
        return s

    def result(self, rid, n_data, n_rays):
        data = np.empty((n_data, n_rays), dtype=np.float64)
        info = np.empty(n_rays, dtype=np.float64)
        _ck(lib().gray_serve_result(self.h, rid, data.ctypes.data, data.nbytes,
                                    info.ctypes.data, info.nbytes), "gray_serve_result")
        return data, info

    def release(self, rid):
        """Drop a finished / failed / cancelled request; returns its status."""
        return lib().gray_serve_result(self.h, rid, None, 0, None, 0)

    def cancel(self, rid):
        _ck(lib().gray_serve_cancel(self.h, rid), "gray_serve_cancel")

    def serve_stats(self):
        s = ServeStats()
        st = lib().gray_serve_get_stats(self.h, ctypes.byref(s))
        return s, st

    def serve_stop(self, drain=False):
        return lib().gray_serve_stop(self.h, 1 if drain else 0)

    @staticmethod
    def clock():
        return lib().gray_serve_clock()

    def read_spacetime(self, grid, level):
        out = np.empty((grid.nz, grid.ny, grid.nx, 51), dtype=np.float32)
        _ck(lib().gray_read_spacetime(self.h, level, out.ctypes.data, out.nbytes),
            "gray_read_spacetime")
        return out

    def swap_levels(self):
        _ck(lib().gray_swap_levels(self.h), "gray_swap_levels")

    def close(self):
        if self.h:
            lib().gray_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
