"""GRay2's HDF5 files without libhdf5 (gray_b200/host/gray_h5.c).

No HDF5 library exists on either machine to cross-check against (no
libhdf5, no h5py).  One file written by libhdf5 does: scipy ships a MATLAB
v7.3 test file, which is a classic-format HDF5 file behind a 512-byte user
block.  The reader is pinned to it; the writer is not pinned to libhdf5.
These tests check that:
 - the reader reads that libhdf5 file (user block and base address,
   layout message v2, fill-value message v1, attribute, modification-time
   and NIL messages skipped) to the exact values MATLAB stored;
 - what the writer writes reads back exactly (spacetime files in the
   README.md:40-60 / io.c:356-428 layout, /rays files of sim/gray.c:170-176);
 - the written bytes carry the published HDF5 format fields, parsed here by
   a second, independent reader in Python (superblock v0, v1 object
   headers, symbol-table groups, local heap, v1 B-tree, dataset messages);
 - the reader follows io.c's rules (times from the non-'g' groups, sorted by
   value; box from the first and last coordinate) and refuses what it
   cannot read (not HDF5, truncated, non-fisheye coordinates, missing
   datasets) with an error instead of misreading it.
"""
import os
import struct

import numpy as np
import pytest

from gray_b200 import h5

UNDEF = 0xffffffffffffffff


def fisheye(n, lo, hi):
    """tools/generate_data.py:49-58"""
    B = np.cbrt(np.arcsinh(lo))
    A = (np.cbrt(np.arcsinh(hi)) - B) / (n - 1)
    return np.sinh((A * np.arange(n) + B) ** 3).astype(np.float32)


def spacetime(tmp_path, names=("0", "10"), n=(5, 6, 7), seed=1):
    rng = np.random.default_rng(seed)
    x, y, z = fisheye(n[0], -40, 40), fisheye(n[1], -30, 35), fisheye(n[2], -20, 50)
    levels = [rng.standard_normal((n[2], n[1], n[0], 51)).astype(np.float32) for _ in names]
    path = str(tmp_path / "data.h5")
    h5.write_spacetime(path, x, y, z, names, levels)
    return path, (x, y, z), levels


# ---------------------------------------------------------------- round trips

def test_spacetime_round_trip_follows_io_c(tmp_path):
    names = ("10", "0", "2.5", "-5")  # stored by name, sorted by value on open
    path, (x, y, z), levels = spacetime(tmp_path, names)
    with h5.Spacetime(path) as s:
        assert s.times == [-5.0, 0.0, 2.5, 10.0]
        assert s.n == (5, 6, 7)
        assert s.lo == (x[0], y[0], z[0]) and s.hi == (x[-1], y[-1], z[-1])
        order = np.argsort([float(t) for t in names])
        for k, j in enumerate(order):
            assert np.array_equal(s.load(k), levels[j])
    with h5.File(path) as f:
        assert f.members("/") == sorted(["grid"] + list(names))
        assert f.members("grid") == ["x", "y", "z"]
        members = f.members("10")
        assert len(members) == 51 and "Gamma_tzz" in members and "g_xy" in members
        assert "rho" in members
        # io.c order: Gamma i-major then j <= k, g i <= j, rho
        assert np.array_equal(f.read("10/Gamma_ttx", np.float32), levels[0][..., 1])
        assert np.array_equal(f.read("10/Gamma_txy", np.float32), levels[0][..., 5])
        assert np.array_equal(f.read("10/Gamma_xtt", np.float32), levels[0][..., 10])
        assert np.array_equal(f.read("10/g_tt", np.float32), levels[0][..., 40])
        assert np.array_equal(f.read("10/g_zz", np.float32), levels[0][..., 49])
        assert np.array_equal(f.read("10/rho", np.float32), levels[0][..., 50])
        assert f.info("grid/x") == ((5,), 4)
        assert f.info("0/rho") == ((7, 6, 5), 4)


@pytest.mark.parametrize("elem", [4, 8])
def test_rays_round_trip_and_exclusive_create(tmp_path, elem):
    rng = np.random.default_rng(2)
    w, hgt, nd = 6, 4, 16
    state = rng.standard_normal((w * hgt, nd))
    path = str(tmp_path / "ray0001.h5")
    h5.write_rays(path, state, w, hgt, elem)
    with h5.File(path) as f:
        assert f.members("/") == ["rays"]
        assert f.info("rays") == ((w, hgt, nd), elem)
        got = f.read("rays")
    want = state.astype(np.float32 if elem == 4 else np.float64).astype(np.float64)
    assert np.array_equal(got.reshape(w * hgt, nd), want)
    with pytest.raises(h5.H5Error) as e:  # H5F_ACC_EXCL (sim/gray.c:175)
        h5.write_rays(path, state, w, hgt, elem)
    assert e.value.status == h5.EEXIST


def test_many_members_span_several_symbol_table_nodes(tmp_path):
    """51 datasets per snapshot and 30 snapshots: several SNODs per group
    under one B-tree node."""
    names = [str(k) for k in range(30)]
    path, _, levels = spacetime(tmp_path, names, n=(3, 3, 3))
    with h5.Spacetime(path) as s:
        assert s.times == [float(k) for k in range(30)]
        assert np.array_equal(s.load(17), levels[17])


# ------------------------------------------ the published format, independently

class Raw:
    """A second reader of the few structures the writer emits, following
    the HDF5 file format specification field by field."""

    def __init__(self, path):
        self.b = open(path, "rb").read()

    def u(self, off, n):
        return int.from_bytes(self.b[off:off + n], "little")

    def superblock(self):
        b = self.b
        assert b[:8] == b"\x89HDF\r\n\x1a\n"
        assert b[8] == 0 and b[9] == 0 and b[10] == 0 and b[12] == 0  # versions
        assert b[13] == 8 and b[14] == 8  # sizes of offsets and lengths
        assert self.u(16, 2) == 4 and self.u(18, 2) == 16  # leaf K, internal K
        assert self.u(24, 8) == 0 and self.u(32, 8) == UNDEF and self.u(48, 8) == UNDEF
        assert self.u(40, 8) == len(b)  # end-of-file address
        assert self.u(56, 8) == 0 and self.u(72, 4) == 1  # root entry, cache type 1
        return self.u(64, 8), self.u(80, 8), self.u(88, 8)

    def messages(self, oh):
        assert self.b[oh] == 1  # version-1 object header
        n, size = self.u(oh + 2, 2), self.u(oh + 8, 4)
        assert self.u(oh + 4, 4) == 1  # reference count
        out, at = [], oh + 16
        while at < oh + 16 + size:
            t, s = self.u(at, 2), self.u(at + 2, 2)
            assert s % 8 == 0  # padded to 8 bytes
            out.append((t, at + 8, s))
            at += 8 + s
        assert len(out) == n and at == oh + 16 + size
        return out

    def group(self, oh):
        msgs = self.messages(oh)
        (t, body, s), = msgs
        assert t == 0x11 and s == 16
        tree, heap = self.u(body, 8), self.u(body + 8, 8)
        assert self.b[heap:heap + 4] == b"HEAP" and self.b[heap + 4] == 0
        dsize, seg = self.u(heap + 8, 8), self.u(heap + 24, 8)
        assert self.b[seg:seg + 8] == bytes(8)  # offset 0: the empty name
        assert self.b[tree:tree + 4] == b"TREE" and self.b[tree + 4] == 0  # group nodes
        assert self.b[tree + 5] == 0 and self.u(tree + 8, 8) == UNDEF  # leaf, no siblings
        used, names = self.u(tree + 6, 2), {}
        assert self.u(tree + 24, 8) == 0  # key 0: the empty name
        prev_last = ""
        for i in range(used):
            snod = self.u(tree + 32 + 16 * i, 8)
            key = self.u(tree + 40 + 16 * i, 8)
            assert self.b[snod:snod + 4] == b"SNOD" and self.b[snod + 4] == 1
            k = self.u(snod + 6, 2)
            assert 1 <= k <= 8  # 2 x leaf K entries per node
            for e in range(k):
                at = snod + 8 + 40 * e
                off = self.u(at, 8)
                assert off < dsize
                name = self.b[seg + off:self.b.index(b"\0", seg + off)].decode()
                assert name > prev_last  # sorted across nodes
                prev_last = name
                names[name] = (self.u(at + 8, 8), self.u(at + 16, 4))
            # key i+1 is the heap offset of the node's last name
            last = self.b[seg + key:self.b.index(b"\0", seg + key)].decode()
            assert last == prev_last
        return names

    def dataset(self, oh):
        msgs = {t: (body, s) for t, body, s in self.messages(oh)}
        assert set(msgs) == {0x1, 0x3, 0x5, 0x8}
        sp, _ = msgs[0x1]
        assert self.b[sp] == 1  # dataspace version 1
        rank = self.b[sp + 1]
        dims = tuple(self.u(sp + 8 + 8 * k, 8) for k in range(rank))
        ty, _ = msgs[0x3]
        assert self.b[ty] == 0x11  # version 1, class 1 (floating point)
        assert self.b[ty + 1] == 0x20  # little-endian, implied mantissa msb
        size = self.u(ty + 4, 4)
        prec, eloc, esz, mloc, msz, bias = struct.unpack_from("<HBBBBI", self.b, ty + 10)
        assert (size, self.b[ty + 2], prec, eloc, esz, mloc, msz, bias) in (
            (4, 31, 32, 23, 8, 0, 23, 127), (8, 63, 64, 52, 11, 0, 52, 1023))
        fv, _ = msgs[0x5]
        assert self.b[fv] == 2  # fill value message version 2
        ly, _ = msgs[0x8]
        assert self.b[ly] == 3 and self.b[ly + 1] == 1  # layout v3, contiguous
        addr, nbytes = self.u(ly + 2, 8), self.u(ly + 10, 8)
        assert nbytes == size * int(np.prod(dims))
        dt = np.float32 if size == 4 else np.float64
        return dims, np.frombuffer(self.b[addr:addr + nbytes], dtype="<" + dt().dtype.char)


def test_written_bytes_follow_the_published_format(tmp_path):
    path, (x, _, _), levels = spacetime(tmp_path, ("0", "10"))
    r = Raw(path)
    root, tree, heap = r.superblock()
    top = r.group(root)
    assert sorted(top) == ["0", "10", "grid"]
    assert all(cache == 1 for _, cache in top.values())  # groups cache B-tree + heap
    grid = r.group(top["grid"][0])
    dims, xs = r.dataset(grid["x"][0])
    assert dims == (5,) and np.array_equal(xs, x)
    snap = r.group(top["10"][0])
    assert len(snap) == 51 and all(cache == 0 for _, cache in snap.values())
    dims, g = r.dataset(snap["Gamma_zzz"][0])
    assert dims == (7, 6, 5) and np.array_equal(g.reshape(dims), levels[1][..., 39])

    rays = str(tmp_path / "ray0003.h5")
    st = np.arange(2 * 3 * 8, dtype=np.float64).reshape(6, 8)
    h5.write_rays(rays, st, 2, 3)
    r = Raw(rays)
    root, _, _ = r.superblock()
    top = r.group(root)
    dims, v = r.dataset(top["rays"][0])
    assert dims == (2, 3, 8) and np.array_equal(v, st.ravel())


# ------------------------------------------------------------------- refusals

def test_reader_refuses_what_it_cannot_read(tmp_path):
    path, _, _ = spacetime(tmp_path)
    with pytest.raises(h5.H5Error) as e:
        h5.File(str(tmp_path / "absent.h5"))
    assert e.value.status == h5.ENOTFOUND
    junk = tmp_path / "junk.h5"
    junk.write_bytes(b"not an hdf5 file" * 64)
    with pytest.raises(h5.H5Error) as e:
        h5.File(str(junk))
    assert e.value.status == h5.EFORMAT
    # truncated: the structures point past the end of the file
    data = open(path, "rb").read()
    cut = tmp_path / "cut.h5"
    cut.write_bytes(data[:len(data) // 3])
    with pytest.raises(h5.H5Error) as e:
        with h5.Spacetime(str(cut)) as s:
            s.load(1)
    assert e.value.status in (h5.EFORMAT, h5.ENOTFOUND)
    with h5.File(path) as f:
        with pytest.raises(h5.H5Error) as e:
            f.read("0/Gamma_qqq")
        assert e.value.status == h5.ENOTFOUND
        with pytest.raises(h5.H5Error) as e:
            f.read("grid")  # a group, not a dataset
        assert e.value.status == h5.ENOTFOUND


def test_non_fisheye_coordinates_are_refused(tmp_path):
    """interp.cl:89-96 maps positions with the n = 3 fisheye formula; a file
    whose coordinates do not follow it would be interpolated at the wrong
    places, so it is refused."""
    n = 6
    lv = [np.zeros((n, n, n, 51), np.float32)]
    uniform = np.linspace(-40, 40, n).astype(np.float32)
    path = str(tmp_path / "uniform.h5")
    h5.write_spacetime(path, uniform, uniform, uniform, ["0"], lv)
    with pytest.raises(h5.H5Error) as e:
        h5.Spacetime(path)
    assert e.value.status == h5.EFORMAT
    assert os.path.exists(path)


# ------------------------------------------------------- a file libhdf5 wrote

def libhdf5_file():
    """scipy's MATLAB 7.4 test file saved in the v7.3 (HDF5) format: one
    9 x 1 double dataset, 0:pi/4:2*pi, with a MATLAB_class attribute."""
    scipy = pytest.importorskip("scipy")
    path = os.path.join(os.path.dirname(scipy.__file__), "io", "matlab", "tests", "data",
                        "testhdf5_7.4_GLNX86.mat")
    if not os.path.exists(path):
        pytest.skip("scipy's MATLAB test data is not installed")
    return path


def test_reads_a_file_written_by_libhdf5():
    path = libhdf5_file()
    data = open(path, "rb").read()
    assert data[512:520] == b"\x89HDF\r\n\x1a\n"  # behind the MAT user block
    with h5.File(path) as f:
        assert f.members("/") == ["testdouble"]
        dims, elem = f.info("testdouble")
        assert dims == (9, 1) and elem == 8
        v = f.read("/testdouble")
        assert v.dtype == np.float64 and v.shape == (9, 1)
        assert np.array_equal(v.ravel(), np.arange(9) * (np.pi / 4))
        with pytest.raises(h5.H5Error) as e:
            f.read("testsingle")
        assert e.value.status == h5.ENOTFOUND
    with pytest.raises(h5.H5Error) as e:  # no grid group: not a spacetime file
        h5.Spacetime(path)
    assert e.value.status in (h5.ENOTFOUND, h5.EFORMAT)
