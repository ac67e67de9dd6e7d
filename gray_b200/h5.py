"""Python view of include/gray_h5.h: GRay2's HDF5 spacetime files
(sim-org/io.c:149-533, README.md:40-60) and /rays dump files
(sim/gray.c:170-176), read and written by the library's own C code
(gray_b200/host/gray_h5.c, in libgray_job.so) without libhdf5."""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libgray_job.so")

OK, EINVAL, ENOMEM, ENOTFOUND, ESIZE, EFORMAT, EIO, EEXIST = 0, -1, -2, -7, -9, -20, -21, -22
NFIELD = 51

_lib = None


class H5Error(RuntimeError):
    def __init__(self, status, what):
        super().__init__("%s: %s (%d)" % (what, lib().gray_h5_strerror(status).decode(), status))
        self.status = status


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libgray_job.so is not built (run __graft_entry__.build())")
        from gray_b200 import api
        api.lib()  # libgray_job.so links against libgray_cuda.so
        L = ctypes.CDLL(LIB_PATH)
        P, vp, u64, i, c = ctypes.POINTER, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_char_p
        L.gray_h5_strerror.restype = c
        L.gray_h5_strerror.argtypes = [i]
        L.gray_h5_open.argtypes = [c, P(vp)]
        L.gray_h5_close.argtypes = [vp]
        L.gray_h5_member.argtypes = [vp, c, u64, c, ctypes.c_size_t, P(u64)]
        L.gray_h5_dataset_info.argtypes = [vp, c, P(i), P(u64), P(i)]
        L.gray_h5_read.argtypes = [vp, c, i, vp, u64]
        L.gray_h5_spacetime_open.argtypes = [c, P(vp)]
        L.gray_h5_spacetime_close.argtypes = [vp]
        L.gray_h5_spacetime_times.restype = u64
        L.gray_h5_spacetime_times.argtypes = [vp, P(P(ctypes.c_double))]
        L.gray_h5_spacetime_grid.argtypes = [vp, P(i), P(ctypes.c_float), P(ctypes.c_float)]
        L.gray_h5_spacetime_load.argtypes = [vp, u64, vp]
        L.gray_h5_write_spacetime.argtypes = [c, i, i, i, vp, vp, vp, u64, P(c), P(vp)]
        L.gray_h5_write_rays.argtypes = [c, vp, i, u64, u64, u64]
        _lib = L
    return _lib


def _ck(status, what):
    if status != OK:
        raise H5Error(status, what)


class File:
    """A classic-format HDF5 file opened for reading."""

    def __init__(self, path):
        self.h = ctypes.c_void_p()
        _ck(lib().gray_h5_open(path.encode(), ctypes.byref(self.h)), "gray_h5_open")

    def members(self, group="/"):
        n = ctypes.c_uint64(0)
        _ck(lib().gray_h5_member(self.h, group.encode(), 0, None, 0, ctypes.byref(n)),
            "gray_h5_member")
        out = []
        buf = ctypes.create_string_buffer(1024)
        for k in range(n.value):
            _ck(lib().gray_h5_member(self.h, group.encode(), k, buf, 1024, None), "gray_h5_member")
            out.append(buf.value.decode())
        return out

    def info(self, path):
        rank, es = ctypes.c_int(0), ctypes.c_int(0)
        dims = (ctypes.c_uint64 * 8)()
        _ck(lib().gray_h5_dataset_info(self.h, path.encode(), ctypes.byref(rank), dims,
                                       ctypes.byref(es)), "gray_h5_dataset_info")
        return tuple(dims[k] for k in range(rank.value)), es.value

    def read(self, path, dtype=np.float64):
        shape, _ = self.info(path)
        out = np.empty(shape, dtype=dtype)
        _ck(lib().gray_h5_read(self.h, path.encode(), out.itemsize, out.ctypes.data, out.size),
            "gray_h5_read")
        return out

    def close(self):
        if self.h:
            lib().gray_h5_close(self.h)
            self.h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Spacetime:
    """A spacetime file as sim-org/io.c reads it: sorted snapshot times,
    grid shape and box, and snapshot k as [nz, ny, nx, 51] floats."""

    def __init__(self, path):
        self.h = ctypes.c_void_p()
        _ck(lib().gray_h5_spacetime_open(path.encode(), ctypes.byref(self.h)),
            "gray_h5_spacetime_open")
        t = ctypes.POINTER(ctypes.c_double)()
        n = lib().gray_h5_spacetime_times(self.h, ctypes.byref(t))
        self.times = [t[k] for k in range(n)]
        nn = (ctypes.c_int * 3)()
        lo, hi = (ctypes.c_float * 3)(), (ctypes.c_float * 3)()
        lib().gray_h5_spacetime_grid(self.h, nn, lo, hi)
        self.n = tuple(nn)            # points along x, y, z
        self.lo, self.hi = tuple(lo), tuple(hi)

    def load(self, k, out=None):
        nx, ny, nz = self.n
        if out is None:
            out = np.empty((nz, ny, nx, NFIELD), dtype=np.float32)
        _ck(lib().gray_h5_spacetime_load(self.h, k, out.ctypes.data), "gray_h5_spacetime_load")
        return out

    def close(self):
        if self.h:
            lib().gray_h5_spacetime_close(self.h)
            self.h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def write_spacetime(path, x, y, z, time_names, levels):
    """Write a spacetime file: coordinates x, y, z (1-D) and one snapshot
    group per name with the 51 fields of levels[k] ([nz, ny, nx, 51])."""
    xs = [np.ascontiguousarray(a, dtype=np.float32) for a in (x, y, z)]
    lv = [np.ascontiguousarray(a, dtype=np.float32) for a in levels]
    names = (ctypes.c_char_p * len(time_names))(*[str(t).encode() for t in time_names])
    ptrs = (ctypes.c_void_p * len(lv))(*[a.ctypes.data for a in lv])
    for a in lv:
        if a.shape != (xs[2].size, xs[1].size, xs[0].size, NFIELD):
            raise ValueError("level shape %s" % (a.shape,))
    _ck(lib().gray_h5_write_spacetime(path.encode(), xs[0].size, xs[1].size, xs[2].size,
                                      xs[0].ctypes.data, xs[1].ctypes.data, xs[2].ctypes.data,
                                      len(lv), names, ptrs), "gray_h5_write_spacetime")


def write_rays(path, state, n_width, n_height, elem_size=8):
    """sim/gray.c:170-176: /rays of shape {n_width, n_height, n_data} from an
    AoS state [n_rays, n_data] (ray order), as float (4) or double (8)."""
    a = np.ascontiguousarray(state, dtype=np.float32 if elem_size == 4 else np.float64)
    _ck(lib().gray_h5_write_rays(path.encode(), a.ctypes.data, elem_size, n_width, n_height,
                                 a.shape[-1]), "gray_h5_write_rays")
