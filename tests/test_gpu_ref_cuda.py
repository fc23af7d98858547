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
