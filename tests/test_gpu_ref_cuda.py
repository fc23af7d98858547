"""This library's CUDA cross-correlation against the reference's own CUDA
kernels (correlate/src/oskar_cross_correlate{,_scalar}_cuda.cu, compiled
for sm_100a from the reference's sources by `make -C oracle ref_cuda`), on
the same device inputs: parity for every variant, and the speed of both on
512-station cases. The reference launchers pick their kernel as on any GPU
of compute capability >= 7.0 (oskar_cross_correlate_cuda.cu:653-695: the
"NON_SM" warp-per-baseline kernel).

Set OSKB_REPORT_DIR to write the timings to <dir>/ref_cuda_timing.json."""
import json
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
from oracle_lib import reference_cuda, reference_cuda_xcorr, suffix  # noqa
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(),
                                 reason="needs a CUDA device"),
              pytest.mark.skipif(reference_cuda() is None,
                                 reason="reference CUDA kernels not built")]

import oskar_b200 as ob  # noqa: E402
from xcorr_cases import XcorrCase  # noqa: E402

FIELDS = ("jones", "I", "Q", "U", "V", "l", "m", "n", "a", "b", "c", "st_u",
          "st_v", "st_w", "st_x", "st_y")


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _ours(c, d, vis, stream=0):
    s = suffix(c.real)
    common = (c.uv_min, min(c.uv_max, 3.0e38), c.inv_wavelength,
              c.frac_bandwidth, c.time_avg, c.gha0, c.dec0, vis, stream)
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


def _ref(c, d, vis):
    ptr = {k: v.data_ptr() for k, v in d.items()}
    reference_cuda_xcorr(c.real, c.matrix, c.gaussian, c.casa, c.num_src,
                         c.num_st, c.offset_out, ptr["jones"], ptr["I"],
                         ptr["Q"], ptr["U"], ptr["V"], ptr["l"], ptr["m"],
                         ptr["n"], ptr["a"], ptr["b"], ptr["c"], ptr["st_u"],
                         ptr["st_v"], ptr["st_w"], ptr["st_x"], ptr["st_y"],
                         c.uv_min, min(c.uv_max, 3.0e38), c.inv_wavelength,
                         c.frac_bandwidth, c.time_avg, c.gha0, c.dec0,
                         vis.data_ptr())


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return max(np.max(np.abs(a - b)) / np.max(np.abs(b)),
               np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("matrix", [True, False])
@pytest.mark.parametrize("gaussian", [False, True])
@pytest.mark.parametrize("bw,ts", [(0.0, 0.0), (10e3, 0.0), (0.0, 10.0),
                                   (10e3, 10.0)])
@pytest.mark.parametrize("casa", [0, 1])
def test_parity_with_reference_cuda(real, matrix, gaussian, bw, ts, casa):
    """Same visibilities as the reference's CUDA kernel: FP64 to 1e-12;
    FP32 to 2e-5 (the reference's FP32 kernel sums in single precision, this
    library's FP32 path per 8-source chunk with FP64 chunk sums)."""
    c = XcorrCase(37, 301, real=real, matrix=matrix, gaussian=gaussian,
                  bandwidth_hz=bw, time_avg=ts, casa=casa, offset_out=2)
    d = {k: dev(getattr(c, k)) for k in FIELDS}
    v_ours, v_ref = dev(c.vis0), dev(c.vis0)
    _ours(c, d, v_ours)
    _ref(c, d, v_ref)
    torch.cuda.synchronize()
    got, ref = v_ours.cpu().numpy(), v_ref.cpu().numpy()
    assert _rel(got - c.vis0, ref - c.vis0) <= (1e-12 if real == np.float64
                                                else 2e-5)


def _time(fn, reps=3):
    fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


@pytest.mark.parametrize("real,gaussian,bw,ts", [
    (np.float64, False, 0.0, 0.0), (np.float32, False, 0.0, 0.0),
    (np.float64, True, 1e5, 10.0), (np.float32, True, 1e5, 10.0)])
def test_speed_against_reference_cuda(real, gaussian, bw, ts):
    """512 stations x 8,000 sources, one (dump, channel), physical ranges:
    both kernels on the legacy stream, CUDA events, after one untimed
    call; the results must agree. Speeds are recorded, not asserted."""
    c = XcorrCase(512, 8000, real=real, gaussian=gaussian, bandwidth_hz=bw,
                  time_avg=ts, ranges="physical", seed=9)
    d = {k: dev(getattr(c, k)) for k in FIELDS}
    v_ours = torch.zeros(8 * c.num_vis, dtype=d["I"].dtype, device="cuda")
    v_ref = torch.zeros_like(v_ours)
    ms_ours = _time(lambda: _ours(c, d, v_ours))
    ms_ref = _time(lambda: _ref(c, d, v_ref))
    work = c.num_st * (c.num_st - 1) // 2 * c.num_src
    assert _rel(v_ours.cpu().numpy(), v_ref.cpu().numpy()) <= (
        1e-12 if real == np.float64 else 1e-4)
    rec = {"case": "512 stations x 8000 sources, %s, %s, bandwidth %g Hz, "
                   "time average %g s" % ("FP64" if real == np.float64
                                          else "FP32",
                                          "Gaussian" if gaussian else
                                          "point", bw, ts),
           "ours_ms": ms_ours, "reference_cuda_ms": ms_ref,
           "ours_g_src_bl_per_s": work / (ms_ours * 1e-3) / 1e9,
           "reference_cuda_g_src_bl_per_s": work / (ms_ref * 1e-3) / 1e9,
           "speedup": ms_ref / ms_ours}
    print(json.dumps(rec))
    out = os.environ.get("OSKB_REPORT_DIR")
    if out:
        path = os.path.join(out, "ref_cuda_timing.json")
        old = json.load(open(path)) if os.path.exists(path) else []
        old.append(rec)
        json.dump(old, open(path, "w"), indent=1)


# ---- station-beam DFT against the reference's GPU weighted-DFT kernels
# (math/define_dftw_m2m.h, define_dftw_c2c.h; oracle/ref_cuda_shim.cu)

def _dft_case(real, num_in, num_out, seed, matrix, is_3d, n_types=None):
    rng = np.random.default_rng(seed)
    c = {}
    c["w"] = rng.normal(size=2 * num_in).astype(real)
    c["xi"], c["yi"] = (rng.uniform(-20, 20, num_in).astype(real)
                        for _ in range(2))
    c["zi"] = rng.uniform(-1, 1, num_in).astype(real)
    az = rng.uniform(0, 2 * np.pi, num_out)
    el = rng.uniform(0, np.pi / 2, num_out)
    c["xo"] = (np.cos(el) * np.sin(az)).astype(real)
    c["yo"] = (np.cos(el) * np.cos(az)).astype(real)
    c["zo"] = np.sin(el).astype(real)
    nd = n_types if n_types else num_in
    c["idx"] = (rng.integers(0, n_types, num_in).astype(np.int32)
                if n_types else None)
    c["data"] = rng.normal(size=nd * num_out * (8 if matrix else 2)).astype(
        real)
    c["k"] = real(2 * np.pi * 150e6 / 299792458.0)
    return c


def _dft_run(c, real, matrix, is_3d, num_in, num_out, ev, ref, reps=0):
    d = {k: (dev(v) if v is not None else None) for k, v in c.items()
         if k != "k"}
    out = torch.zeros(num_out * (8 if matrix else 2), dtype=d["w"].dtype,
                      device="cuda")
    norm = real(1.0 / num_in)
    zi = d["zi"] if is_3d else None
    zo = d["zo"] if is_3d else None
    if ref:
        lib = reference_cuda()
        fn = getattr(lib, "ref_cuda_dftw_" + ("double" if real == np.float64
                                              else "float"))
        fp = ctypes.c_double if real == np.float64 else ctypes.c_float
        P = lambda t: ctypes.c_void_p(t.data_ptr() if t is not None else 0)
        call = lambda: fn(ctypes.c_int(int(matrix)), ctypes.c_int(is_3d),
                          ctypes.c_int(num_in), fp(c["k"]), P(d["w"]),
                          P(d["xi"]), P(d["yi"]), P(zi), ctypes.c_int(0),
                          ctypes.c_int(num_out), P(d["xo"]), P(d["yo"]),
                          P(zo), P(d["idx"]), P(d["data"]),
                          ctypes.c_int(ev[0]), ctypes.c_int(ev[1]),
                          ctypes.c_int(0), P(out), fp(norm), None)
    else:
        call = lambda: ob.call("oskb_dftw_" + suffix(real), int(matrix),
                               num_in, float(c["k"]), d["w"], d["xi"],
                               d["yi"], zi, 0, num_out, d["xo"], d["yo"],
                               zo, d["idx"], d["data"], ev[0], ev[1], 0, out,
                               float(norm), 0)
    if reps:
        return out, _time(call, reps)
    call()
    torch.cuda.synchronize()
    return out.cpu().numpy(), None


import ctypes  # noqa: E402


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("matrix,is_3d,n_types,ev", [
    (True, 1, 1, (1, 1)), (True, 0, None, (1, 1)), (True, 1, 3, (1, 0)),
    (True, 1, None, (0, 1)), (False, 1, None, (1, 1)), (False, 0, 2, (1, 1))])
def test_dftw_parity_with_reference_cuda(real, matrix, is_3d, n_types, ev):
    num_in, num_out = 300, 1031
    c = _dft_case(real, num_in, num_out, 3, matrix, is_3d, n_types)
    ours, _ = _dft_run(c, real, matrix, is_3d, num_in, num_out, ev, False)
    ref, _ = _dft_run(c, real, matrix, is_3d, num_in, num_out, ev, True)
    assert _rel(ours, ref) <= (1e-12 if real == np.float64 else 2e-5)


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_dftw_speed_against_reference_cuda(real):
    """One station of the aperture-array configuration (256 dipoles, one
    element type, 12,001 directions, 3-D, 2x2 data), as oskar_dftw runs it
    per station; speeds recorded, not asserted."""
    num_in, num_out = 256, 12001
    c = _dft_case(real, num_in, num_out, 8, True, 1, 1)
    o1, ms_ours = _dft_run(c, real, True, 1, num_in, num_out, (1, 1), False,
                           reps=5)
    o2, ms_ref = _dft_run(c, real, True, 1, num_in, num_out, (1, 1), True,
                          reps=5)
    assert _rel(o1.cpu().numpy(), o2.cpu().numpy()) <= (
        1e-12 if real == np.float64 else 2e-5)
    work = num_in * num_out
    rec = {"case": "weighted DFT m2m 3-D, 256 elements x 12001 directions, "
                   "%s" % ("FP64" if real == np.float64 else "FP32"),
           "ours_ms": ms_ours, "reference_cuda_ms": ms_ref,
           "ours_g_element_directions_per_s": work / (ms_ours * 1e-3) / 1e9,
           "reference_cuda_g_element_directions_per_s":
               work / (ms_ref * 1e-3) / 1e9,
           "speedup": ms_ref / ms_ours}
    print(json.dumps(rec))
    out = os.environ.get("OSKB_REPORT_DIR")
    if out:
        path = os.path.join(out, "ref_cuda_timing.json")
        old = json.load(open(path)) if os.path.exists(path) else []
        old.append(rec)
        json.dump(old, open(path, "w"), indent=1)


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_cross_power_against_reference_cuda(real):
    """Beam-pattern cross power, 512 stations x 16,384 directions (a 128 x
    128 beam image), 2x2 Jones: the reference's CUDA kernel (pair loop,
    O(N^2) per direction) against the prefix-sum pass; parity (FP64 1e-12;
    FP32 against the FP64 result, 2e-5) and speed recorded."""
    nst, nsrc = 512, 16384
    rng = np.random.default_rng(17)
    lobe = np.exp(-np.linspace(0, 6, nsrc) ** 2)
    J = rng.normal(0, 0.05, (nst, nsrc, 8))
    J[..., 0] += lobe
    J[..., 6] += lobe
    J = np.ascontiguousarray(J.ravel().astype(real))
    stokes = (1.0, 0.1, -0.05, 0.02)
    norm = 2.0 / (nst * (nst - 1))
    dJ = dev(J)
    ours = torch.zeros(nsrc * 8, dtype=dJ.dtype, device="cuda")
    refo = torch.zeros(nsrc * 8, dtype=dJ.dtype, device="cuda")
    lib = reference_cuda()
    fn = getattr(lib, "ref_cuda_cross_power_" + ("double" if real ==
                                                  np.float64 else "float"))
    fp = ctypes.c_double if real == np.float64 else ctypes.c_float
    call_ref = lambda: fn(ctypes.c_int(nsrc), ctypes.c_int(nst),
                          ctypes.c_void_p(dJ.data_ptr()),
                          *[fp(v) for v in stokes], fp(norm), ctypes.c_int(0),
                          ctypes.c_void_p(refo.data_ptr()), None)
    call_ours = lambda: ob.call("oskb_evaluate_cross_power_" + suffix(real),
                                1, nsrc, nst, dJ, *stokes, 0, ours, 0)
    ms_ours = _time(call_ours, 5)
    ms_ref = _time(call_ref, 2)
    o, r = ours.cpu().numpy(), refo.cpu().numpy()
    if real == np.float64:
        assert _rel(o, r) <= 1e-12
    else:
        truth = torch.zeros(nsrc * 8, dtype=torch.float64, device="cuda")
        ob.call("oskb_evaluate_cross_power_d", 1, nsrc, nst,
                dev(J.astype(np.float64)), *stokes, 0, truth, 0)
        t = truth.cpu().numpy()
        assert _rel(o, t) <= 2e-5
        print("FP32 error against FP64: ours %.2e, reference kernel %.2e"
              % (_rel(o, t), _rel(r, t)))
    rec = {"case": "beam-pattern cross power, 512 stations x 16384 "
                   "directions, %s" % ("FP64" if real == np.float64
                                       else "FP32"),
           "ours_ms": ms_ours, "reference_cuda_ms": ms_ref,
           "speedup": ms_ref / ms_ours}
    print(json.dumps(rec))
    out = os.environ.get("OSKB_REPORT_DIR")
    if out:
        path = os.path.join(out, "ref_cuda_timing.json")
        old = json.load(open(path)) if os.path.exists(path) else []
        old.append(rec)
        json.dump(old, open(path, "w"), indent=1)
