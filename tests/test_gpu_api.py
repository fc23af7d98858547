"""The OSKAR-named API on the GPU, written the way the reference's own tests
drive these functions (oskar/correlate/test/Test_cross_correlate.cpp,
oskar/interferometer/test/Test_Jones.cpp, Test_evaluate_jones_K.cpp):
oskar_Mem / oskar_Jones / oskar_Telescope objects in, visibilities out,
checked against the CPU oracle on the same inputs."""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(),
                                 reason="needs a CUDA device")]

from oskar_b200 import oskar_api as oa  # noqa: E402
from oskar_b200._lib import load  # noqa: E402
from oracle_lib import oracle  # noqa: E402
from xcorr_cases import XcorrCase  # noqa: E402

C, M = oa.OSKAR_COMPLEX, oa.OSKAR_MATRIX
D, S = oa.OSKAR_DOUBLE, oa.OSKAR_SINGLE
GPU = oa.OSKAR_GPU


def rel(got, ref):
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    return max(np.linalg.norm(got - ref) / np.linalg.norm(ref),
               np.max(np.abs(got - ref)) / np.max(np.abs(ref)))


def run_api(c, prec, gast, bandwidth_hz, casa, env=None, monkeypatch=None):
    lib = load()
    mtype = prec | C | (M if c.matrix else 0)
    real = np.float64 if prec == D else np.float32
    nst, nsrc = c.num_st, c.num_src
    j = oa.jones_from_numpy(c.jones, mtype, nst, nsrc, GPU)
    flux = [oa.mem_from_numpy(getattr(c, k), prec, GPU) for k in "IQUV"]
    dirs = [oa.mem_from_numpy(getattr(c, k), prec, GPU) for k in "lmn"]
    ext = [oa.mem_from_numpy(getattr(c, k), prec, GPU) for k in "abc"]
    uvw = [oa.mem_from_numpy(getattr(c, k), prec, GPU)
           for k in ("st_u", "st_v", "st_w")]
    tel = oa.telescope(prec, GPU, c.st_x.astype(real), c.st_y.astype(real))
    lib.oskar_telescope_set_channel_bandwidth(tel, bandwidth_hz)
    lib.oskar_telescope_set_time_average(tel, c.time_avg)
    lib.oskar_telescope_set_phase_centre(tel, oa.OSKAR_COORDS_RADEC, 0.0,
                                         c.dec0)
    vis = oa.mem_from_numpy(c.vis0, mtype, GPU)
    st = oa.ctypes.c_int(0)
    lib.oskar_cross_correlate(casa, int(c.gaussian), nsrc, j,
                              oa.mem_array(*flux), oa.mem_array(*dirs),
                              oa.mem_array(*ext), tel, oa.mem_array(*uvw),
                              gast, c.freq, c.offset_out, vis,
                              oa.status_ptr(st))
    out = oa.mem_to_numpy(vis)
    oa.free_jones(j)
    oa.free_mem(*flux, *dirs, *ext, *uvw, vis)
    oa.free_telescope(tel)
    assert st.value == 0
    return out


@pytest.mark.parametrize("prec", [D, S])
@pytest.mark.parametrize("matrix", [True, False])
@pytest.mark.parametrize("gaussian", [False, True])
@pytest.mark.parametrize("time_avg,bandwidth", [(0.0, 0.0), (10.0, 0.0),
                                                (0.0, 10e3), (10.0, 10e3)])
def test_cross_correlate_grid(prec, matrix, gaussian, time_avg, bandwidth):
    """Test_cross_correlate.cpp:254-346: gast = 1, 100 MHz, CASA phase
    convention on, 19 stations x 277 sources."""
    real = np.float64 if prec == D else np.float32
    c = XcorrCase(19, 277, real=real, matrix=matrix, gaussian=gaussian,
                  bandwidth_hz=bandwidth, time_avg=time_avg, casa=1,
                  offset_out=2)
    gast = 1.0
    c.gha0 = gast - 0.0
    got = run_api(c, prec, gast, bandwidth, 1)
    ref = c.vis0.copy()
    oracle().call("xcorr_" + ("matrix_" if matrix else "scalar_")
                  + ("d" if prec == D else "f"), real, 1, int(gaussian),
                  *c.oracle_args(ref))
    assert rel(got, ref) <= (1e-12 if prec == D else 1e-5)


def test_cross_correlate_tensor_core_env(monkeypatch):
    """OSKAR_CORRELATE=TC routes point sources without smearing to the
    tensor-core kernel (1e-6)."""
    c = XcorrCase(60, 900, ranges="physical", seed=4)
    monkeypatch.setenv("OSKAR_CORRELATE", "TC")
    got = run_api(c, D, 1.0, 0.0, 0)
    ref = c.vis0.copy()
    oracle().call("xcorr_matrix_d", np.float64, 0, 0, *c.oracle_args(ref))
    err = rel(got - c.vis0, ref - c.vis0)
    assert 0 < err <= 1e-6  # TC, so not bit-exact with FP64


@pytest.mark.parametrize("psd", [True, False])
def test_cross_correlate_fp64_class_env(psd, monkeypatch):
    """OSKAR_CORRELATE=TC64 routes FP64 point sources without smearing to
    the FP64-class tensor-core form (1e-12); a brightness matrix that is not
    positive semi-definite sends the call to the direct kernel."""
    c = XcorrCase(60, 900, ranges="physical", seed=5)
    if not psd:
        c.Q[3] = 3.0 * c.I[3]
    monkeypatch.setenv("OSKAR_CORRELATE", "TC64")
    got = run_api(c, D, 1.0, 0.0, 0)
    ref = c.vis0.copy()
    oracle().call("xcorr_matrix_d", np.float64, 0, 0, *c.oracle_args(ref))
    assert rel(got - c.vis0, ref - c.vis0) <= 1e-12
    # the FP64-class form ran (its status words report the brightness)
    flags = (oa.ctypes.c_int * 2)()
    assert load().oskb_tc_status(None, oa.ctypes.addressof(flags),
                                 oa.ctypes.addressof(flags) + 4) == 0
    assert flags[0] == (0 if psd else 1) and flags[1] == 0


@pytest.mark.parametrize("psd", [True, False])
def test_cross_correlate_tensor_core_env_fp32(psd, monkeypatch):
    """OSKAR_CORRELATE=TC routes FP32 point sources without smearing to the
    integer tensor-core form (FP32 in and out, within FP32's 1e-5); a
    brightness matrix that is not positive semi-definite sends the call to
    the direct kernel."""
    c = XcorrCase(60, 900, real=np.float32, ranges="physical", seed=6)
    if not psd:
        c.Q[3] = 3.0 * c.I[3]
    monkeypatch.setenv("OSKAR_CORRELATE", "TC")
    got = run_api(c, S, 1.0, 0.0, 0)
    ref = c.vis0.copy()
    oracle().call("xcorr_matrix_f", np.float32, 0, 0, *c.oracle_args(ref))
    assert rel(got - c.vis0, ref - c.vis0) <= 1e-5
    flags = (oa.ctypes.c_int * 2)()
    assert load().oskb_tc_status(None, oa.ctypes.addressof(flags),
                                 oa.ctypes.addressof(flags) + 4) == 0
    assert flags[0] == (0 if psd else 1) and flags[1] == 0


def test_jones_join_identity_known_answer():
    """Test_Jones.cpp:187-286: joining with identity leaves Jones unchanged,
    in place and out of place, matrix x matrix and scalar x matrix."""
    lib = load()
    rng = np.random.default_rng(1)
    nst, nsrc = 7, 33
    a = rng.normal(size=8 * nst * nsrc)
    ident = np.zeros((nst * nsrc, 8))
    ident[:, 0] = ident[:, 6] = 1
    ones = np.zeros((nst * nsrc, 2))
    ones[:, 0] = 1
    j1 = oa.jones_from_numpy(a, D | C | M, nst, nsrc, GPU)
    j2 = oa.jones_from_numpy(ident, D | C | M, nst, nsrc, GPU)
    j3 = oa.jones_from_numpy(np.zeros_like(a), D | C | M, nst, nsrc, GPU)
    js = oa.jones_from_numpy(ones, D | C, nst, nsrc, GPU)
    st = oa.ctypes.c_int(0)
    lib.oskar_jones_join(j3, j1, j2, oa.status_ptr(st))
    assert st.value == 0
    assert np.array_equal(oa.mem_to_numpy(lib.oskar_jones_mem(j3)), a)
    lib.oskar_jones_join(None, j1, js, oa.status_ptr(st))  # in place, m x c
    assert st.value == 0
    assert np.array_equal(oa.mem_to_numpy(lib.oskar_jones_mem(j1)), a)
    oa.free_jones(j1, j2, j3, js)


def test_evaluate_jones_K_api():
    """Test_evaluate_jones_K.cpp: 100 stations x 1000 sources."""
    lib = load()
    rng = np.random.default_rng(3)
    ns, nst = 1000, 100
    l, m, n = (rng.uniform(0.1, 0.9, ns) for _ in range(3))
    u, v, w = (rng.uniform(-1e3, 1e3, nst) for _ in range(3))
    f = rng.uniform(0, 2, ns)
    freq = 100e6
    ref = np.zeros(2 * ns * nst)
    oracle().call("jones_k_d", np.float64, ns, l, m, n, nst, u, v, w,
                  2 * math.pi * freq / 299792458.0, f, 0.5, 1.5, 0, ref)
    K = oa.jones_from_numpy(np.zeros(2 * ns * nst), D | C, nst, ns, GPU)
    mems = [oa.mem_from_numpy(x, D, GPU) for x in (l, m, n, u, v, w, f)]
    st = oa.ctypes.c_int(0)
    lib.oskar_evaluate_jones_K(K, ns, *mems[:6], freq, mems[6], 0.5, 1.5, 0,
                               oa.status_ptr(st))
    assert st.value == 0
    assert rel(oa.mem_to_numpy(lib.oskar_jones_mem(K)), ref) <= 1e-12
    oa.free_jones(K)
    oa.free_mem(*mems)


def test_dftw_api_grows_output():
    """oskar_dftw ensures the output holds offset_out + num_out entries."""
    lib = load()
    rng = np.random.default_rng(6)
    n_in, n_out, off = 64, 300, 5
    k = 2 * math.pi * 100e6 / 299792458.0
    w = rng.uniform(-1, 1, 2 * n_in)
    xi, yi, zi = (rng.uniform(-20, 20, n_in) for _ in range(3))
    xo, yo, zo = (rng.uniform(-1, 1, n_out) for _ in range(3))
    data = rng.uniform(-1, 1, n_in * n_out * 8)
    ref = np.zeros((n_out + off) * 8)
    oracle().call("dftw_d", np.float64, 1, 1, n_in, k, w, xi, yi, zi, 0,
                  n_out, xo, yo, zo, None, data, 1, 1, off, ref, 1.0 / n_in)
    mw = oa.mem_from_numpy(w, D | C, GPU)
    coords = [oa.mem_from_numpy(x, D, GPU) for x in (xi, yi, zi, xo, yo, zo)]
    md = oa.mem_from_numpy(data, D | C | M, GPU)
    out = oa.mem_from_numpy(np.zeros(8), D | C | M, GPU)  # 1 entry only
    st = oa.ctypes.c_int(0)
    lib.oskar_dftw(1, n_in, k, mw, *coords[:3], 0, n_out, *coords[3:], None,
                   md, 1, 1, off, out, oa.status_ptr(st))
    assert st.value == 0
    assert lib.oskar_mem_length(out) == n_out + off
    assert rel(oa.mem_to_numpy(out)[8 * off:], ref[8 * off:]) <= 1e-12
    oa.free_mem(mw, *coords, md, out)


def test_auto_correlate_api():
    lib = load()
    c = XcorrCase(9, 101)
    ref = np.zeros(8 * 9)
    oracle().call("acorr_matrix_d", np.float64, c.num_src, c.num_st, 0,
                  c.jones, c.I, c.Q, c.U, c.V, ref)
    j = oa.jones_from_numpy(c.jones, D | C | M, 9, 101, GPU)
    flux = [oa.mem_from_numpy(getattr(c, k), D, GPU) for k in "IQUV"]
    vis = oa.mem_from_numpy(np.zeros(8 * 9), D | C | M, GPU)
    st = oa.ctypes.c_int(0)
    lib.oskar_auto_correlate(101, j, oa.mem_array(*flux), 0, vis,
                             oa.status_ptr(st))
    assert st.value == 0
    assert rel(oa.mem_to_numpy(vis), ref) <= 1e-12
    oa.free_jones(j)
    oa.free_mem(*flux, vis)


@pytest.mark.parametrize("prec", [D, S])
def test_conversion_wrappers(prec):
    """oskar_convert_station_uvw_to_baseline_uvw,
    oskar_convert_lon_lat_to_relative_directions and
    oskar_convert_apparent_ra_dec_to_enu_directions on oskar_Mem arrays,
    against the oracle."""
    lib = load()
    real = np.float64 if prec == D else np.float32
    s = "d" if prec == D else "f"
    rng = np.random.default_rng(9)
    nst = 40
    uvw = [rng.uniform(-1e4, 1e4, nst).astype(real) for _ in range(3)]
    mu = [oa.mem_from_numpy(a, prec, GPU) for a in uvw]
    mb = [oa.mem_from_numpy(np.zeros(1, real), prec, GPU) for _ in range(3)]
    st = oa.ctypes.c_int(0)
    lib.oskar_convert_station_uvw_to_baseline_uvw(1, nst, 0, *mu, 0, *mb,
                                                  oa.status_ptr(st))
    assert st.value == 0
    nbl = nst * (nst - 1) // 2
    ref = [np.zeros(nbl, real) for _ in range(3)]
    oracle().call("station_uvw_to_baseline_uvw_" + s, real, 1, nst, 0,
                  *uvw, 0, *ref)
    for m, r in zip(mb, ref):
        assert lib.oskar_mem_length(m) == nbl
        assert np.array_equal(oa.mem_to_numpy(m), r)
    n = 999
    lon = rng.uniform(0, 6, n).astype(real)
    lat = rng.uniform(-1.5, 1.5, n).astype(real)
    ml, mlat = (oa.mem_from_numpy(a, prec, GPU) for a in (lon, lat))
    out = [oa.mem_from_numpy(np.zeros(n, real), prec, GPU) for _ in range(3)]
    lib.oskar_convert_lon_lat_to_relative_directions(n, ml, mlat, 0.2, -0.6,
                                                     *out, oa.status_ptr(st))
    assert st.value == 0
    ref = [np.zeros(n, real) for _ in range(3)]
    oracle().call("lon_lat_to_relative_directions_" + s, real, n, lon, lat,
                  real(0.2), real(np.cos(-0.6)), real(np.sin(-0.6)), *ref)
    tol = 1e-14 if prec == D else 2e-6
    for m, r in zip(out, ref):
        assert np.max(np.abs(oa.mem_to_numpy(m) - r)) <= tol
    xyz = [oa.mem_from_numpy(np.zeros(n + 2, real), prec, GPU)
           for _ in range(3)]
    lib.oskar_convert_apparent_ra_dec_to_enu_directions(
        n, ml, mlat, 1.3, -0.47, 2, *xyz, oa.status_ptr(st))
    assert st.value == 0
    ref = [np.zeros(n + 2, real) for _ in range(3)]
    oracle().call("ra_dec_to_enu_directions_" + s, real, n, lon, lat,
                  real(1.3), real(np.sin(-0.47)), real(np.cos(-0.47)), 2,
                  *ref)
    for m, r in zip(xyz, ref):
        assert np.max(np.abs(oa.mem_to_numpy(m) - r)) <= tol
    oa.free_mem(*mu, *mb, ml, mlat, *out, *xyz)
