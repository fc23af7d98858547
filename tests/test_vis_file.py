"""The .vis writer (oskb_vis_file_*, host code) against the oracle written
through the reference's own binary-format library (oracle/ref_vis_shim.c
and binary/src/*.c): the two files must be byte-identical, and every chunk
must read back through the reference's reader with its CRC-32C checked.
CPU only: the writer takes host buffers."""
import ctypes
import os

import numpy as np
import pytest

import oskar_b200 as ob
from oracle_lib import ROOT

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "liboskar_ref_binary.so")
pytestmark = pytest.mark.skipif(not os.path.exists(REF_BIN),
                                reason="reference sources not present")

DCM, FC = 0x08 | 0x20 | 0x40, 0x04 | 0x20


def _lib():
    lib = ctypes.CDLL(REF_BIN)
    I, D, P, S = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, \
        ctypes.c_char_p
    lib.orcvis_create.restype = P
    lib.orcvis_create.argtypes = ([S] + [I] * 10 + [D] * 6 + [I] + [D] * 5 +
                                  [P] * 10 + [S] * 6)
    lib.orcvis_write_block.argtypes = [P] + [I] * 5 + [P] * 5
    lib.orcvis_close.argtypes = [P]
    return lib


def _case(seed, amp_type=DCM, coord=0x08, nst=7, ntime=3, nch=2,
          autos=True, elements=True, settings="[interferometer]\nx=1\n"):
    rng = np.random.default_rng(seed)
    real = np.float64 if coord == 0x08 else np.float32
    vreal = np.float64 if amp_type & 0x08 else np.float32
    ncomp = 8 if amp_type & 0x40 else 2
    c = dict(amp_type=amp_type, coord=coord, nst=nst, ntime=ntime, nch=nch,
             autos=autos, settings=settings)
    c["station"] = [rng.normal(0, 1e3, nst).astype(real) for _ in range(3)]
    c["diam"] = rng.uniform(30, 40, nst)
    c["names"] = ["s%04d (station %d)" % (i, i % 3) for i in range(nst)]
    if elements:
        c["num_el"] = rng.integers(0, 5, nst).astype(np.int32)
        tot = int(c["num_el"].sum())
        c["el"] = [rng.normal(0, 10, tot).astype(real) for _ in range(3)]
        c["feed"] = rng.uniform(0, np.pi, 6 * tot)
    else:
        c["num_el"], c["el"], c["feed"] = None, [None] * 3, None
    nbl = nst * (nst - 1) // 2
    c["blocks"] = []
    for b in range(2):
        c["blocks"].append(dict(
            cross=rng.normal(size=ntime * nch * nbl * ncomp).astype(vreal),
            autos=(rng.normal(size=ntime * nch * nst * ncomp).astype(vreal)
                   if autos else None),
            uvw=[rng.normal(0, 1e3, ntime * nst).astype(real)
                 for _ in range(3)]))
    return c


def _args(c, path):
    names = (ctypes.c_char_p * c["nst"])(*[n.encode() for n in c["names"]])
    p = lambda a: None if a is None else a.ctypes.data
    enc = lambda s: None if s is None else s.encode()
    return [path.encode(), c["amp_type"], c["coord"], 2, 2 * c["ntime"],
            c["nch"], c["nch"], c["nst"], int(c["autos"]), 1, 1, 100e6,
            1e6, 1e5, 51544.5, 60.0, 10.0, 0, 30.5, -26.5, 116.76, -26.82,
            377.0, *[p(a) for a in c["station"]], p(c["diam"]),
            ctypes.addressof(names), p(c["num_el"]),
            *[p(a) for a in c["el"]], p(c["feed"]), enc("telescope.tm"),
            enc(c["settings"]), b"2026-01-01, 00:00:00 (UTC)", b"2.12.0",
            b"/work", b"astro"], names


def _write(c, path, ours):
    args, keep = _args(c, path)
    if ours:
        lib = ob.load()
        st = ctypes.c_int(0)
        h = lib.oskb_vis_file_create(*args, ctypes.byref(st))
        assert st.value == 0 and h
        write = lambda *a: ob.call("oskb_vis_file_write_block", h, *a)
        close = lambda: lib.oskb_vis_file_close(h)
    else:
        lib = _lib()
        h = lib.orcvis_create(*args)
        write = lambda *a: lib.orcvis_write_block(h, *[
            x if isinstance(x, int) else
            (x.ctypes.data if x is not None else None) for x in a])
        close = lambda: lib.orcvis_close(h)
    for b, blk in enumerate(c["blocks"]):
        st = write(b, b * c["ntime"], 0, c["ntime"], c["nch"], blk["cross"],
                   blk["autos"], *blk["uvw"])
        assert st == 0
    assert close() == 0
    del keep


@pytest.mark.parametrize("kw", [
    dict(), dict(amp_type=FC, coord=0x04, autos=False),
    dict(elements=False, settings=None), dict(nst=1, autos=True),
    dict(nst=40, ntime=2, nch=3)])
def test_vis_file_byte_identical(tmp_path, kw):
    c = _case(5, **kw)
    a, b = str(tmp_path / "ours.vis"), str(tmp_path / "ref.vis")
    _write(c, a, True)
    _write(c, b, False)
    da, db = open(a, "rb").read(), open(b, "rb").read()
    assert len(da) == len(db) and da == db


def test_vis_file_reads_back_with_reference_reader(tmp_path):
    c = _case(9)
    path = str(tmp_path / "ours.vis")
    _write(c, path, True)
    lib = _lib()
    lib.orcvis_read.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                ctypes.c_int, ctypes.c_int, ctypes.c_size_t,
                                ctypes.c_void_p]
    fn = path.encode()
    nst, nbl = c["nst"], c["nst"] * (c["nst"] - 1) // 2
    # header: number of stations, amp type, frequencies
    v = ctypes.c_int(0)
    assert lib.orcvis_read(fn, 0x02, 11, 11, 0, 4, ctypes.byref(v)) == 0
    assert v.value == nst
    f = ctypes.c_double(0)
    assert lib.orcvis_read(fn, 0x08, 11, 23, 0, 8, ctypes.byref(f)) == 0
    assert f.value == 100e6
    x = np.zeros(nst)
    assert lib.orcvis_read(fn, 0x08, 11, 32, 0, x.nbytes, x.ctypes.data) == 0
    assert np.array_equal(x, c["station"][0])
    for b, blk in enumerate(c["blocks"]):
        dims = np.zeros(6, np.int32)
        assert lib.orcvis_read(fn, 0x02, 12, 1, b, dims.nbytes,
                               dims.ctypes.data) == 0
        assert list(dims) == [b * c["ntime"], 0, c["ntime"], c["nch"], nbl,
                              nst]
        got = np.zeros_like(blk["cross"])
        assert lib.orcvis_read(fn, DCM, 12, 3, b, got.nbytes,
                               got.ctypes.data) == 0
        assert np.array_equal(got, blk["cross"])
        w = np.zeros_like(blk["uvw"][2])
        assert lib.orcvis_read(fn, 0x08, 12, 9, b, w.nbytes,
                               w.ctypes.data) == 0
        assert np.array_equal(w, blk["uvw"][2])
    # every chunk is indexed; corrupting one payload byte fails its CRC
    n = lib.orcvis_num_tags(fn)
    expect = 4 + 1 + 27 + 3 * nst + nst + 1 + 6 * nst + 2 * 6
    assert n == expect
    data = bytearray(open(path, "rb").read())
    data[-10] ^= 0xFF
    bad = str(tmp_path / "bad.vis")
    open(bad, "wb").write(data)
    w = np.zeros_like(c["blocks"][1]["uvw"][2])
    assert lib.orcvis_read(bad.encode(), 0x08, 12, 9, 1, w.nbytes,
                           w.ctypes.data) != 0


def test_vis_file_errors(tmp_path):
    lib = ob.load()
    st = ctypes.c_int(0)
    c = _case(1)
    args, keep = _args(c, str(tmp_path / "x.vis"))
    args[1] = 0x08  # not complex
    assert not lib.oskb_vis_file_create(*args, ctypes.byref(st))
    assert st.value == -3
    st.value = 0
    args, keep = _args(c, str(tmp_path / "no" / "such" / "dir.vis"))
    assert not lib.oskb_vis_file_create(*args, ctypes.byref(st))
    assert st.value != 0
