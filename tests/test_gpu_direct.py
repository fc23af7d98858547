"""GPU parity of the direct kernels against the CPU oracle.

Every call goes through the C ABI (include/oskar_b200.h) with device buffers
from torch. Tolerances:
  - FP64: max |gpu - oracle| <= 1e-12 * max |oracle| and L2 relative
    <= 1e-12 (the reference's own FP64 CPU-vs-GPU test allows 1e-10 max,
    oskar/correlate/test/Test_cross_correlate.cpp:18-38);
  - FP32: the same two measures <= 1e-5 (the reference's FP32 test allows
    2e-2 max / 1e-5 mean relative).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(),
                                 reason="needs a CUDA device")]

import oskar_b200 as ob  # noqa: E402
from oracle_lib import oracle, suffix  # noqa: E402
from xcorr_cases import XcorrCase  # noqa: E402

TOL = {np.float64: 1e-12, np.float32: 1e-5}


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def assert_close(got, ref, real, tol=None):
    tol = TOL[real] if tol is None else tol
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    scale = np.max(np.abs(ref)) + 1e-300
    err_max = np.max(np.abs(got - ref)) / scale
    err_l2 = np.linalg.norm(got - ref) / (np.linalg.norm(ref) + 1e-300)
    assert err_max <= tol and err_l2 <= tol, (err_max, err_l2)


def run_gpu_xcorr(c, real):
    vis = dev(c.vis0)
    d = {k: dev(getattr(c, k)) for k in ("jones", "I", "Q", "U", "V", "l",
                                         "m", "n", "a", "b", "c", "st_u",
                                         "st_v", "st_w", "st_x", "st_y")}
    s = suffix(real)
    common = (c.uv_min, min(c.uv_max, 3.0e38), c.inv_wavelength,
              c.frac_bandwidth, c.time_avg, c.gha0, c.dec0, vis,
              ob.stream_ptr())
    if c.matrix:
        ob.call("oskb_cross_correlate_" + s, c.casa, int(c.gaussian),
                c.num_src, c.num_st, c.offset_out, d["jones"], d["I"],
                d["Q"], d["U"], d["V"], d["l"], d["m"], d["n"], d["a"],
                d["b"], d["c"], d["st_u"], d["st_v"], d["st_w"], d["st_x"],
                d["st_y"], *common)
    else:
        ob.call("oskb_cross_correlate_scalar_" + s, c.casa, int(c.gaussian),
                c.num_src, c.num_st, c.offset_out, d["jones"], d["I"],
                d["l"], d["m"], d["n"], d["a"], d["b"], d["c"], d["st_u"],
                d["st_v"], d["st_w"], d["st_x"], d["st_y"], *common)
    torch.cuda.synchronize()
    return vis.cpu().numpy()


def run_oracle_xcorr(c, real):
    v = c.vis0.copy()
    oracle().call("xcorr_" + ("matrix_" if c.matrix else "scalar_")
                  + suffix(real), real, c.casa, int(c.gaussian),
                  *c.oracle_args(v))
    return v


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("matrix", [True, False])
@pytest.mark.parametrize("gaussian", [False, True])
@pytest.mark.parametrize("bw,ts", [(0.0, 0.0), (10e3, 0.0), (0.0, 10.0),
                                   (10e3, 10.0)])
@pytest.mark.parametrize("casa", [0, 1])
def test_xcorr_grid(real, matrix, gaussian, bw, ts, casa):
    """The reference test grid (Test_cross_correlate.cpp:254-346):
    19 stations x 277 sources, point/Gaussian x bandwidth/time smearing."""
    c = XcorrCase(19, 277, real=real, matrix=matrix, gaussian=gaussian,
                  bandwidth_hz=bw, time_avg=ts, casa=casa, offset_out=3)
    assert_close(run_gpu_xcorr(c, real), run_oracle_xcorr(c, real), real)


@pytest.mark.parametrize("num_st,num_src", [(2, 1), (3, 17), (31, 33),
                                            (33, 16), (65, 100), (130, 513)])
@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_xcorr_ragged_sizes(num_st, num_src, real):
    """Sizes that are not multiples of the 32-station tile or the 16-source
    chunk, on a physical (phase-rotating) input distribution."""
    c = XcorrCase(num_st, num_src, real=real, ranges="physical",
                  bandwidth_hz=100e3, time_avg=10.0, gaussian=True, seed=7)
    assert_close(run_gpu_xcorr(c, real), run_oracle_xcorr(c, real), real)


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_xcorr_uv_filter(real):
    c = XcorrCase(40, 64, real=real, uv_min=0.5, uv_max=1.2)
    got, ref = run_gpu_xcorr(c, real), run_oracle_xcorr(c, real)
    assert_close(got, ref, real)
    changed = np.any((got != c.vis0).reshape(-1, 8), axis=1)
    assert changed.any() and not changed.all()  # filtered baselines kept


@pytest.mark.parametrize("slices", ["1", "3", "7"])
@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_xcorr_source_slices(slices, real, monkeypatch):
    """The source loop split across CTAs (partial sums per slice, reduced in
    slice order) gives the oracle's result for any slice count, with the uv
    filter on so that filtered baselines must come out untouched."""
    monkeypatch.setenv("OSKB_XCORR_SLICES", slices)
    c = XcorrCase(70, 300, real=real, uv_min=0.5, uv_max=1.2, offset_out=5,
                  bandwidth_hz=10e3)
    got, ref = run_gpu_xcorr(c, real), run_oracle_xcorr(c, real)
    assert_close(got, ref, real)
    changed = np.any((got != c.vis0).reshape(-1, 8), axis=1)
    assert changed.any() and not changed.all()


def test_xcorr_slices_deterministic():
    """Two runs with the default slicing give bit-identical output, also
    when the scratch pool that holds the slices' partial sums has been
    handed back to the driver in between."""
    c = XcorrCase(100, 5000, ranges="physical", seed=9)
    first = run_gpu_xcorr(c, np.float64)
    assert np.array_equal(first, run_gpu_xcorr(c, np.float64))
    assert ob.load().oskb_scratch_release() == 0
    assert np.array_equal(first, run_gpu_xcorr(c, np.float64))


@pytest.mark.parametrize("casa", [0, 1])
@pytest.mark.parametrize("slices", ["1", "4"])
def test_xcorr_fp64_tensor_core_vs_simt(casa, slices, monkeypatch):
    """FP64 point sources without smearing on the FP64 tensor pipe
    (mma.sync f64, the default; OSKB_XCORR_DMMA=0 selects SIMT) agree with
    the SIMT kernel and the oracle to 1e-13, with the uv filter, an output
    offset and slices."""
    monkeypatch.setenv("OSKB_XCORR_SLICES", slices)
    c = XcorrCase(75, 1003, casa=casa, uv_min=0.5, uv_max=1.2,
                  offset_out=7, seed=5)
    ref = run_oracle_xcorr(c, np.float64)
    monkeypatch.setenv("OSKB_XCORR_DMMA", "1")
    tc = run_gpu_xcorr(c, np.float64)
    monkeypatch.setenv("OSKB_XCORR_DMMA", "0")
    simt = run_gpu_xcorr(c, np.float64)
    assert_close(tc, ref, np.float64, 1e-13)
    assert_close(tc, simt, np.float64, 1e-13)
    changed = np.any((tc != c.vis0).reshape(-1, 8), axis=1)
    assert changed.any() and not changed.all()


@pytest.mark.parametrize("nsrc", [1, 5, 8, 13, 16, 17, 40])
def test_xcorr_fp64_tensor_core_chunk_counts(nsrc, monkeypatch):
    """The FP64 tensor-core pipeline (two chunks staged ahead, one
    transformed while the other's products run) for one, two, three and
    more chunks per item, full and partial."""
    monkeypatch.setenv("OSKB_XCORR_SLICES", "1")
    c = XcorrCase(41, nsrc, seed=nsrc)
    ref = run_oracle_xcorr(c, np.float64)
    monkeypatch.setenv("OSKB_XCORR_DMMA", "1")
    assert_close(run_gpu_xcorr(c, np.float64), ref, np.float64, 1e-13)


def test_xcorr_empty_inputs():
    c = XcorrCase(5, 4)
    vis = dev(c.vis0)
    # zero sources / one station: no work, vis untouched, status 0
    for ns, nst in [(0, 5), (4, 1), (4, 0)]:
        ob.call("oskb_cross_correlate_d", 0, 0, ns, nst, 0, None, None,
                None, None, None, None, None, None, None, None, None, None,
                None, None, None, None, 0.0, 1e30, 1.0, 0.0, 0.0, 0.0, 0.0,
                vis, ob.stream_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(vis.cpu().numpy(), c.vis0)
    # missing arrays with work to do: the reference's invalid-argument code
    st = ob.call("oskb_cross_correlate_d", 0, 0, 4, 5, 0, None, None, None,
                 None, None, None, None, None, None, None, None, None, None,
                 None, None, None, 0.0, 1e30, 1.0, 0.0, 0.0, 0.0, 0.0, vis,
                 ob.stream_ptr(), check=False)
    assert st == -3


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("matrix", [True, False])
def test_auto_correlate(real, matrix):
    c = XcorrCase(9, 101, real=real, matrix=matrix)
    nc = 8 if matrix else 2
    v0 = np.random.default_rng(5).uniform(-1, 1, 12 * nc).astype(real)
    ref = v0.copy()
    if matrix:
        oracle().call("acorr_matrix_" + suffix(real), real, c.num_src,
                      c.num_st, 2, c.jones, c.I, c.Q, c.U, c.V, ref)
    else:
        oracle().call("acorr_scalar_" + suffix(real), real, c.num_src,
                      c.num_st, 2, c.jones, c.I, ref)
    vis = dev(v0)
    ob.call("oskb_auto_correlate_" + suffix(real), int(matrix), c.num_src,
            c.num_st, 2, dev(c.jones), dev(c.I), dev(c.Q), dev(c.U),
            dev(c.V), vis, ob.stream_ptr())
    torch.cuda.synchronize()
    assert_close(vis.cpu().numpy(), ref, real)


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("ignore_w", [0, 1])
def test_jones_k(real, ignore_w):
    rng = np.random.default_rng(3)
    ns, nst = 1000, 100
    l, m, n = (rng.uniform(0.1, 0.9, ns).astype(real) for _ in range(3))
    u, v, w = (rng.uniform(-1e3, 1e3, nst).astype(real) for _ in range(3))
    f = rng.uniform(0, 2, ns).astype(real)
    k = 2 * np.pi * 100e6 / 299792458.0
    ref = np.zeros(2 * ns * nst, real)
    oracle().call("jones_k_" + suffix(real), real, ns, l, m, n, nst, u, v, w,
                  k, f, 0.5, 1.5, ignore_w, ref)
    out = torch.zeros(2 * ns * nst, dtype=torch.float64 if real == np.float64
                      else torch.float32, device="cuda")
    ob.call("oskb_evaluate_jones_K_" + suffix(real), ns, dev(l), dev(m),
            dev(n), nst, dev(u), dev(v), dev(w), k, dev(f), 0.5, 1.5,
            ignore_w, out, ob.stream_ptr())
    torch.cuda.synchronize()
    # phases reach ~4e3 rad: FP32 phase rounding dominates (|dphi| ~ 3e-4)
    assert_close(out.cpu().numpy(), ref, real,
                 tol=1e-12 if real == np.float64 else 5e-4)


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("kind,name,na,nb,nc", [
    (1, "cc_c", 2, 2, 2), (2, "cc_m", 2, 2, 8), (3, "cm_m", 2, 8, 8),
    (4, "mc_m", 8, 2, 8), (5, "mm_m", 8, 8, 8)])
def test_jones_join(real, kind, name, na, nb, nc):
    rng = np.random.default_rng(4)
    n = 12345
    a = rng.uniform(-2, 2, n * na).astype(real)
    b = rng.uniform(-2, 2, n * nb).astype(real)
    ref = np.zeros(n * nc, real)
    oracle().call("mem_mul_%s_%s" % (name, suffix(real)), real, n, a, b, ref)
    da, db = dev(a), dev(b)
    out = torch.zeros(n * nc, dtype=da.dtype, device="cuda")
    ob.call("oskb_mem_multiply_" + suffix(real), kind, 0, 0, 0, n, da, db,
            out, ob.stream_ptr())
    torch.cuda.synchronize()
    assert_close(out.cpu().numpy(), ref, real, tol=1e-15 if real ==
                 np.float64 else 1e-6)
    if na == nc:  # in-place join J1 = J1 * J2, as oskar_jones_join(j1,j1,j2)
        ob.call("oskb_mem_multiply_" + suffix(real), kind, 0, 0, 0, n, da,
                db, da, ob.stream_ptr())
        torch.cuda.synchronize()
        assert_close(da.cpu().numpy(), ref, real, tol=1e-15 if real ==
                     np.float64 else 1e-6)


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("matrix,is_3d,use_idx,ex,ey",
                         [(0, 0, 0, 1, 1), (0, 1, 1, 1, 1), (1, 0, 0, 1, 1),
                          (1, 1, 1, 1, 1), (1, 1, 1, 1, 0), (1, 0, 1, 0, 1)])
def test_dftw(real, matrix, is_3d, use_idx, ex, ey):
    """oskar_dftw c2c/m2m, 2-D/3-D (Test_evaluate_array_pattern.cpp)."""
    rng = np.random.default_rng(6)
    n_in, n_out, n_types, off_c, off_o = 700, 1301, 3, 5, 7
    k = 2 * np.pi * 100e6 / 299792458.0
    ph = rng.uniform(0, 2 * np.pi, n_in)
    w = np.stack([np.cos(ph), np.sin(ph)], 1).ravel().astype(real)
    xi, yi, zi = (rng.uniform(-20, 20, n_in).astype(real) for _ in range(3))
    xo, yo, zo = (rng.uniform(-1, 1, n_out + off_c).astype(real)
                  for _ in range(3))
    idx = rng.integers(0, n_types, n_in).astype(np.int32) if use_idx else None
    nd = n_types if use_idx else n_in
    nc = 8 if matrix else 2
    data = rng.uniform(-1, 1, nd * n_out * nc).astype(real)
    out0 = rng.uniform(-1, 1, (n_out + off_o) * nc).astype(real)
    ref = out0.copy()
    oracle().call("dftw_" + suffix(real), real, matrix, is_3d, n_in, k, w,
                  xi, yi, zi if is_3d else None, off_c, n_out, xo, yo,
                  zo if is_3d else None, idx, data, ex, ey, off_o, ref,
                  1.0 / n_in)
    out = dev(out0)
    ob.call("oskb_dftw_" + suffix(real), matrix, n_in, k, dev(w), dev(xi),
            dev(yi), dev(zi) if is_3d else None, off_c, n_out, dev(xo),
            dev(yo), dev(zo) if is_3d else None,
            dev(idx) if use_idx else None, dev(data), ex, ey, off_o, out,
            1.0 / n_in, ob.stream_ptr())
    torch.cuda.synchronize()
    assert_close(out.cpu().numpy(), ref, real,
                 tol=1e-12 if real == np.float64 else 2e-5)


@pytest.mark.parametrize("n_in", [40, 700])
def test_dftw_non_finite_and_huge_phases(n_in):
    """FP64 phases the shared table does not cover (NaN, and beyond 2^51
    table steps) go through the exact path: one NaN element coordinate
    makes every direction NaN, as in the oracle; an element 1e15 m away
    (phase ~ 1e15 rad, whose value no two formulas agree on) is given zero
    weight, so the sums must still match the oracle's to 1e-12 with every
    CTA taking the exact path for that chunk. n_in = 40 runs the CTAs
    without the table, 700 with it."""
    rng = np.random.default_rng(12)
    n_out = 900
    k = 2 * np.pi * 100e6 / 299792458.0
    ph = rng.uniform(0, 2 * np.pi, n_in)
    w = np.stack([np.cos(ph), np.sin(ph)], 1).ravel()
    xi, yi = (rng.uniform(-20, 20, n_in) for _ in range(2))
    xo, yo = (rng.uniform(-1, 1, n_out) for _ in range(2))
    data = rng.uniform(-1, 1, n_in * n_out * 2)
    xi_far = xi.copy()
    xi_far[n_in // 2] = 1e15
    w_far = w.copy()
    w_far[2 * (n_in // 2):2 * (n_in // 2) + 2] = 0.0
    xi_nan = xi.copy()
    xi_nan[n_in // 3] = np.nan
    for x_el, w in ((xi_far, w_far), (xi_nan, w)):
        ref = np.zeros(n_out * 2)
        oracle().call("dftw_d", np.float64, 0, 0, n_in, k, w, x_el, yi,
                      None, 0, n_out, xo, yo, None, None, data, 1, 1, 0,
                      ref, 1.0 / n_in)
        out = torch.zeros(n_out * 2, dtype=torch.float64, device="cuda")
        ob.call("oskb_dftw_d", 0, n_in, k, dev(w), dev(x_el), dev(yi),
                None, 0, n_out, dev(xo), dev(yo), None, None, dev(data), 1,
                1, 0, out, 1.0 / n_in, ob.stream_ptr())
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        if np.isnan(x_el).any():
            assert np.all(np.isnan(ref)) and np.all(np.isnan(got))
        else:
            assert_close(got, ref, np.float64, tol=1e-12)


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_element_weights(real):
    rng = np.random.default_rng(7)
    n = 256
    x, y, z, cab = (rng.uniform(-20, 20, n).astype(real) for _ in range(4))
    k = 2 * np.pi * 110e6 / 299792458.0
    ref = np.zeros(2 * n, real)
    oracle().call("element_weights_dft_" + suffix(real), real, n, x, y, z,
                  cab, k, 0.3, -0.2, 0.93, ref)
    out = torch.zeros(2 * n, dtype=torch.float64 if real == np.float64 else
                      torch.float32, device="cuda")
    ob.call("oskb_evaluate_element_weights_dft_" + suffix(real), n, dev(x),
            dev(y), dev(z), dev(cab), k, 0.3, -0.2, 0.93, out,
            ob.stream_ptr())
    torch.cuda.synchronize()
    # FP32 phases reach ~100 rad, where one ulp is ~8e-6 rad: the GPU's fused
    # multiply-adds and the CPU's separate roundings differ at that level.
    assert_close(out.cpu().numpy(), ref, real,
                 tol=1e-13 if real == np.float64 else 1e-4)


def test_station_uvw():
    rng = np.random.default_rng(8)
    n = 512
    x, y, z = (rng.uniform(-3e4, 3e4, n) for _ in range(3))
    ra0, dec0, gast = 0.1, -0.52, 1.3
    ha = gast - ra0
    ref = [np.zeros(n + 2) for _ in range(3)]
    oracle().call("ecef_to_station_uvw_d", np.float64, n, x, y, z,
                  np.sin(ha), np.cos(ha), np.sin(dec0), np.cos(dec0), 0, 2,
                  *ref)
    out = [torch.zeros(n + 2, dtype=torch.float64, device="cuda")
           for _ in range(3)]
    ob.call("oskb_convert_ecef_to_station_uvw_d", n, dev(x), dev(y), dev(z),
            ra0, dec0, gast, 0, 2, *out, ob.stream_ptr())
    torch.cuda.synchronize()
    for o, r in zip(out, ref):
        assert_close(o.cpu().numpy(), r, np.float64, tol=1e-15)
