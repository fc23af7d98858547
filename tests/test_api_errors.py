"""Host-side behaviour of the OSKAR-named API (no GPU needed): containers,
status propagation and the reference's error codes for bad locations, types
and dimensions, mirroring the checks of oskar_cross_correlate.c:73-108,
oskar_jones_join.c:25-35, oskar_evaluate_jones_K.c:46-62 and the type
matrix of oskar/interferometer/test/Test_Jones.cpp."""
import ctypes

import numpy as np
import pytest

from oskar_b200 import oskar_api as oa
from oskar_b200._lib import load

C = oa.OSKAR_COMPLEX
M = oa.OSKAR_MATRIX
D, S = oa.OSKAR_DOUBLE, oa.OSKAR_SINGLE
CPU = oa.OSKAR_CPU


@pytest.fixture
def lib():
    return load()


def st0():
    return ctypes.c_int(0)


def test_element_sizes(lib):
    assert lib.oskar_mem_element_size(D) == 8
    assert lib.oskar_mem_element_size(S | C) == 8
    assert lib.oskar_mem_element_size(D | C | M) == 64
    assert lib.oskar_mem_element_size(S | C | M) == 32


def test_mem_roundtrip_cpu(lib):
    a = np.arange(24, dtype=np.float64)
    m = oa.mem_from_numpy(a, D | C, CPU)
    assert lib.oskar_mem_length(m) == 12
    assert lib.oskar_mem_is_complex(m) == 1 and lib.oskar_mem_is_matrix(m) == 0
    assert lib.oskar_mem_precision(m) == D and lib.oskar_mem_location(m) == CPU
    assert np.array_equal(oa.mem_to_numpy(m), a)
    st = st0()
    lib.oskar_mem_clear_contents(m, oa.status_ptr(st))
    assert not oa.mem_to_numpy(m).any()
    oa.free_mem(m)


def test_bad_types_and_status(lib):
    st = st0()
    assert lib.oskar_mem_create(0x10, CPU, 4, oa.status_ptr(st)) is None
    assert st.value == -13  # OSKAR_ERR_BAD_DATA_TYPE
    # a non-zero status on entry: nothing happens
    st = ctypes.c_int(-99)
    assert lib.oskar_mem_create(D, CPU, 4, oa.status_ptr(st)) is None
    assert st.value == -99
    st = st0()
    assert lib.oskar_jones_create(D, CPU, 2, 2, oa.status_ptr(st)) is None
    assert st.value == -13  # Jones must be complex


def test_copy_contents_checks(lib):
    a = oa.mem_from_numpy(np.zeros(4), D, CPU)
    b = oa.mem_from_numpy(np.zeros(4, np.float32), S, CPU)
    st = st0()
    lib.oskar_mem_copy_contents(a, b, 0, 0, 4, oa.status_ptr(st))
    assert st.value == -9
    c = oa.mem_from_numpy(np.zeros(2), D, CPU)
    st = st0()
    lib.oskar_mem_copy_contents(c, a, 0, 0, 4, oa.status_ptr(st))
    assert st.value == -5
    oa.free_mem(a, b, c)


def test_jones_join_dimension_mismatch(lib):
    j1 = oa.jones_from_numpy(np.zeros(8 * 6), D | C | M, 2, 3, CPU)
    j2 = oa.jones_from_numpy(np.zeros(8 * 4), D | C | M, 2, 2, CPU)
    st = st0()
    lib.oskar_jones_join(None, j1, j2, oa.status_ptr(st))
    assert st.value == -11
    oa.free_jones(j1, j2)


def test_jones_join_cpu_location_is_rejected(lib):
    """There is no CPU compute path: CPU data gives OSKAR_ERR_BAD_LOCATION,
    type mismatches are reported first, as in the reference."""
    j1 = oa.jones_from_numpy(np.zeros(8 * 4), D | C | M, 2, 2, CPU)
    j2 = oa.jones_from_numpy(np.zeros(2 * 4), D | C, 2, 2, CPU)
    j3 = oa.jones_from_numpy(np.zeros(8 * 4, np.float32), S | C | M, 2, 2,
                             CPU)
    st = st0()
    lib.oskar_jones_join(None, j1, j2, oa.status_ptr(st))
    assert st.value == -14
    st = st0()
    lib.oskar_jones_join(j3, j1, j2, oa.status_ptr(st))
    assert st.value == -9
    oa.free_jones(j1, j2, j3)


def _xcorr_args(lib, loc_uvw=CPU, uvw_type=D, nuvw=4, vis_type=D | C | M):
    nst, nsrc = 4, 5
    j = oa.jones_from_numpy(np.zeros(8 * nst * nsrc), D | C | M, nst, nsrc,
                            CPU)
    flux = [oa.mem_from_numpy(np.ones(nsrc), D, CPU) for _ in range(4)]
    dirs = [oa.mem_from_numpy(np.ones(nsrc), D, CPU) for _ in range(3)]
    real = np.float64 if uvw_type == D else np.float32
    uvw = [oa.mem_from_numpy(np.ones(nuvw, real), uvw_type, loc_uvw)
           for _ in range(3)]
    vis = oa.mem_from_numpy(np.zeros(8 * 6), vis_type, CPU)
    tel = oa.telescope(D, CPU, np.zeros(nst), np.zeros(nst))
    return j, flux, dirs, uvw, vis, tel, nsrc


@pytest.mark.parametrize("case,code", [("type", -9), ("dims", -11),
                                       ("vis_type", -9), ("cpu", -14)])
def test_cross_correlate_checks(lib, case, code):
    kw = {"type": dict(uvw_type=S), "dims": dict(nuvw=3),
          "vis_type": dict(vis_type=S | C | M), "cpu": {}}[case]
    j, flux, dirs, uvw, vis, tel, nsrc = _xcorr_args(lib, **kw)
    st = st0()
    lib.oskar_cross_correlate(0, 0, nsrc, j, oa.mem_array(*flux),
                              oa.mem_array(*dirs), oa.mem_array(*dirs), tel,
                              oa.mem_array(*uvw), 1.0, 100e6, 0, vis,
                              oa.status_ptr(st))
    assert st.value == code
    assert not oa.mem_to_numpy(vis).any()  # nothing written
    oa.free_jones(j)
    oa.free_mem(*flux, *dirs, *uvw, vis)
    oa.free_telescope(tel)


def test_evaluate_jones_K_checks(lib):
    K = oa.jones_from_numpy(np.zeros(2 * 6), D | C, 2, 3, CPU)
    a = [oa.mem_from_numpy(np.ones(3), D, CPU) for _ in range(3)]
    b = [oa.mem_from_numpy(np.ones(2, np.float32), S, CPU)
         for _ in range(3)]
    f = oa.mem_from_numpy(np.ones(3), D, CPU)
    st = st0()
    lib.oskar_evaluate_jones_K(K, 3, *a, *b, 100e6, f, 0.0, 10.0, 0,
                               oa.status_ptr(st))
    assert st.value == -9
    oa.free_jones(K)
    oa.free_mem(*a, *b, f)


def test_conversion_wrapper_checks(lib):
    a = oa.mem_from_numpy(np.zeros(5), D, CPU)
    b = oa.mem_from_numpy(np.zeros(5, np.float32), S, CPU)
    st = st0()
    lib.oskar_convert_station_uvw_to_baseline_uvw(0, 5, 0, a, a, a, 0, a,
                                                  a, b, oa.status_ptr(st))
    assert st.value == -9
    st = st0()
    lib.oskar_convert_station_uvw_to_baseline_uvw(0, 5, 0, a, a, a, 0, a,
                                                  a, a, oa.status_ptr(st))
    assert st.value == -14  # no CPU compute path
    st = st0()
    lib.oskar_convert_lon_lat_to_relative_directions(5, a, a, 0.0, 0.0, a,
                                                     a, None,
                                                     oa.status_ptr(st))
    assert st.value == -14
    st = ctypes.c_int(-3)
    lib.oskar_convert_apparent_ra_dec_to_enu_directions(
        5, a, a, 0.0, 0.0, 0, a, a, a, oa.status_ptr(st))
    assert st.value == -3  # status on entry is kept
    oa.free_mem(a, b)


def test_hierarchical_station_description_checks():
    """The tree description of oskb_station_beam_hierarchical is checked on
    the host before any device work: workspace size 0 and
    OSKB_ERR_INVALID_ARGUMENT (-3) for a bad tree."""
    from oskar_b200._lib import call
    i32 = lambda *v: np.asarray(v, np.int32)
    ws = lambda nt, cs, nd=100, L=None: call(
        "oskb_station_beam_hierarchical_workspace_bytes", 8,
        len(nt) if L is None else L, i32(*nt), i32(*cs), nd, check=False)
    # three levels: 2 leaf layouts, 2 sub-station types of 3 and 4 children,
    # one station of 5 children
    good = ws((2, 2, 1), (0, 3, 7, 12))
    assert good > 0
    # beam buffers 2 x 8 x 100 FP64 (level 0) and 2 x 8 x 100 (level 1), 5
    # weights, 2 pointings, 5 zero indices, each rounded up to 256 bytes
    r = lambda b: (b + 255) // 256 * 256
    assert good == r(12800) + r(12800) + r(80) + r(48) + r(20)
    assert ws((2, 2, 1), (0, 3, 7, 12), nd=-1) == 0
    assert ws((2, 2, 2), (0, 3, 7, 12, 14)) == 0      # top level not 1
    assert ws((2, 2, 1), (1, 3, 7, 12)) == 0          # CSR not from 0
    assert ws((2, 2, 1), (0, 3, 3, 12)) == 0          # a childless node
    assert ws((2, 0, 1), (0, 3)) == 0                 # a level of no types
    assert ws((2,), (0, 3)) == 0                      # one level only
    assert ws((1,) * 17, tuple(range(17))) == 0       # more than 16 levels
    assert ws((1,) * 16, tuple(range(16))) > 0
    el = np.zeros(4)
    st = call("oskb_station_beam_hierarchical_d", 3, i32(2, 2, 2), 2, el,
              el, el, el, el, 1.0, 1, i32(1, 1, 1), i32(0, 3, 7, 12, 14), el,
              el, el, None, 0, 1, 1e8, np.zeros(9), 10, el, el, el, el,
              1 << 20, el, None, check=False)
    assert st == -3
