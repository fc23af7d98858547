"""The batched block correlator (one persistent launch per block of dumps x
channels, Jones K and the join formed in the staging) against the oracle
run the reference's way: K, join and correlate per dump, chunk and channel.

Tolerances (max and L2, relative to the largest visibility): FP64 1e-12;
FP32 1e-4. In FP32 the Jones K phase is formed in single precision, as the
reference's FP32 path forms it (define_evaluate_jones_K.h:53-70): at the
|phase| ~ 400 rad of these 3 km baselines one rounding is ~3e-5 rad, so
two valid evaluation orders (fused multiply-add on the GPU, separate
multiply and add in the oracle) differ at 1e-5 in the visibilities."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(),
                                 reason="needs a CUDA device")]

import oskar_b200 as ob  # noqa: E402
from block_cases import BlockCase  # noqa: E402
from oracle_lib import suffix  # noqa: E402

TOL = {np.float64: 1e-12, np.float32: 1e-4}


def dev(a):
    return None if a is None else torch.from_numpy(
        np.ascontiguousarray(a)).cuda()


def rel(got, ref):
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    scale = np.max(np.abs(ref))
    return max(np.max(np.abs(got - ref)) / scale,
               np.linalg.norm(got - ref) / np.linalg.norm(ref))


def run_block(c, vis0=None):
    real = c.real
    vis = dev(np.zeros(c.num_times * c.num_channels * c.nbl * 8, real)
              if vis0 is None else vis0)
    gauss = any(c.gaussian)
    ob.call("oskb_correlate_block_direct_" + suffix(real), c.casa,
            c.num_src, c.num_st, c.num_times, c.num_channels, dev(c.E),
            int(c.beam_per_dump), dev(c.I), dev(c.Q), dev(c.U), dev(c.V),
            dev(c.l), dev(c.m), dev(c.n),
            dev(c.a) if gauss else None, dev(c.b) if gauss else None,
            dev(c.c) if gauss else None, dev(c.uvw), dev(c.st_x),
            dev(c.st_y), dev(c.inv_wl), c.bw, c.tavg, dev(c.gha0), c.dec0,
            c.uv_min_m, c.uv_max_m, 0, c.filter_min, c.filter_max, vis,
            ob.stream_ptr())
    torch.cuda.synchronize()
    return vis.cpu().numpy()


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("bw,tavg", [(0.0, 0.0), (1e5, 0.0), (0.0, 10.0),
                                     (1e5, 10.0)])
@pytest.mark.parametrize("casa", [0, 1])
def test_block_vs_oracle(real, bw, tavg, casa):
    c = BlockCase(real=real, bandwidth_hz=bw, time_avg=tavg, casa=casa)
    assert rel(run_block(c), c.oracle_vis()) <= TOL[real]


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_block_all_points_no_beam(real):
    """Point chunks only (a, b, c not passed) and identity E (J = K)."""
    c = BlockCase(real=real, gaussian=(0, 0, 0, 0), beam=False,
                  num_times=2, num_channels=3)
    assert rel(run_block(c), c.oracle_vis()) <= TOL[real]


def test_block_beam_per_dump_filters_and_accumulate():
    """E per dump, uv filter in metres, a flux filter, and accumulation
    onto existing visibilities."""
    c = BlockCase(beam_per_dump=True, uv_min_m=500.0, uv_max_m=3000.0,
                  filter_min=0.5, filter_max=2.5, num_st=70,
                  chunks=(300, 17, 45), gaussian=(1, 0, 1))
    rng = np.random.default_rng(3)
    vis0 = rng.normal(size=c.num_times * c.num_channels * c.nbl * 8)
    got = run_block(c, vis0)
    ref = c.oracle_vis() + vis0
    assert rel(got, ref) <= 1e-12
    # some baselines filtered: exactly the initial values there
    same = np.all((got == vis0).reshape(-1, 8), axis=1)
    assert same.any() and not same.all()


@pytest.mark.parametrize("sched", ["2,0", "2,1", "4,0", "8,1", "0,0",
                                   "0,1", "1,1"])
def test_block_schedules_bit_identical(sched, monkeypatch):
    """Every launch schedule gives the same bits (each visibility is summed
    over the sources in the same order whatever the grid or item order)."""
    c = BlockCase(num_st=100, chunks=(200, 33), gaussian=(1, 0))
    monkeypatch.setenv("OSKB_BLOCK_SCHEDULE", "2,1")
    ref = run_block(c)
    monkeypatch.setenv("OSKB_BLOCK_SCHEDULE", sched)
    assert np.array_equal(run_block(c), ref)


def test_block_autotuner_reports_choice(monkeypatch):
    monkeypatch.delenv("OSKB_BLOCK_SCHEDULE", raising=False)
    monkeypatch.setenv("OSKB_AUTOTUNE", "1")
    c = BlockCase(num_st=64, chunks=(150, 50), gaussian=(0, 1),
                  num_channels=5, seed=99)
    got = run_block(c)
    assert rel(got, c.oracle_vis()) <= 1e-12
    import ctypes
    buf = ctypes.create_string_buffer(8192)
    n = ob.call("oskb_block_tune_report", ctypes.addressof(buf), 8192,
                check=False)
    text = buf.value.decode()
    assert n > 0 and "stations=64" in text and "channels=5" in text


def test_block_empty_and_invalid():
    c = BlockCase(num_times=1, num_channels=1)
    vis = dev(np.zeros(c.nbl * 8))
    # nothing to do: status 0, untouched
    st = ob.call("oskb_correlate_block_direct_d", 0, 0, c.num_st, 1, 1,
                 None, 0, None, None, None, None, None, None, None, None,
                 None, None, None, None, None, None, 0.0, 0.0, None, 0.0,
                 0.0, 1e30, 0, 0.0, 1e30, vis, ob.stream_ptr(), check=False)
    assert st == 0
    # missing arrays with work to do: invalid argument
    st = ob.call("oskb_correlate_block_direct_d", 0, 5, c.num_st, 1, 1,
                 None, 0, None, None, None, None, None, None, None, None,
                 None, None, None, None, None, None, 0.0, 0.0, None, 0.0,
                 0.0, 1e30, 0, 0.0, 1e30, vis, ob.stream_ptr(), check=False)
    assert st == -3
    torch.cuda.synchronize()
    assert not vis.cpu().numpy().any()


def _host_view(ptr, count, real):
    import ctypes
    ctype = ctypes.c_double if real == np.float64 else ctypes.c_float
    buf = (ctype * count).from_address(ptr)
    return np.frombuffer(buf, dtype=real)


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_block_plan_graph_replay(real):
    """The block plan: first block eager and captured, second block a graph
    replay with new uvw and hour angles; both equal the oracle."""
    import ctypes
    lib = ob.load()
    c = BlockCase(real=real, num_st=50, chunks=(90, 30), gaussian=(1, 0))
    st = ctypes.c_int(0)
    plan = lib.oskb_block_plan_create(
        8 if real == np.float64 else 4, c.casa, c.num_st, c.num_src,
        c.num_times, c.num_channels, 1, 1, 0,
        c.freqs.ctypes.data, c.bw, c.tavg, c.dec0, c.uv_min_m, c.uv_max_m,
        0, c.filter_min, c.filter_max, ctypes.addressof(st))
    assert st.value == 0 and plan
    try:
        assert ob.call("oskb_block_plan_set_sky", plan, c.I, c.Q, c.U, c.V,
                       c.l, c.m, c.n, c.a, c.b, c.c) == 0
        assert ob.call("oskb_block_plan_set_stations", plan, c.st_x,
                       c.st_y) == 0
        assert ob.call("oskb_block_plan_set_beam", plan, c.E) == 0
        nvis = c.num_times * c.num_channels * c.nbl * 8
        uvw = _host_view(lib.oskb_block_plan_host_uvw(plan), c.uvw.size,
                         real)
        gha0 = _host_view(lib.oskb_block_plan_host_gha0(plan), c.num_times,
                          np.float64)
        vis = _host_view(lib.oskb_block_plan_host_vis(plan), nvis, real)
        tol = TOL[real]
        for block in range(3):
            if block:
                rng = np.random.default_rng(100 + block)
                c.uvw = rng.uniform(-3e3, 3e3, c.uvw.shape).astype(real)
                c.gha0 = rng.uniform(-1, 1, c.num_times)
            uvw[:] = c.uvw.ravel()
            gha0[:] = c.gha0
            assert ob.call("oskb_block_plan_execute", plan) == 0
            assert ob.call("oskb_block_plan_synchronize", plan) == 0
            assert rel(vis.copy(), c.oracle_vis()) <= tol, block
        assert lib.oskb_block_plan_graph_launches(plan) == 2
    finally:
        lib.oskb_block_plan_free(plan)


def _spectral_case(real, **kw):
    from sky_cases import SkyTable, random_sky
    c = BlockCase(real=real, **kw)
    c.freqs = np.array([60e6, 95e6, 140e6, 210e6])[:c.num_channels]
    c.inv_wl = c.freqs / 299792458.0
    sky = SkyTable(random_sky(c.num_src, 41), real)
    c.set_spectral(sky)
    return c, sky


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_block_spectral_brightness(real):
    """Brightness per channel, scaled on the device for the whole band in
    one launch, correlated in one block launch; a flux filter that sources
    cross between channels. Oracle: scale, K, join, correlate per dump,
    chunk and channel, as the reference's block loop does."""
    c, sky = _spectral_case(real, num_channels=4, bandwidth_hz=1e5,
                            time_avg=10.0, filter_min=0.8, filter_max=6.0)
    I = c.flux_c["I"]
    crossing = np.any((I > 0.8) & (I <= 6.0), 0) & \
        ~np.all((I > 0.8) & (I <= 6.0), 0)
    assert crossing.sum() > 5
    # no channel's I within rounding of a filter bound (FP32 would flip it)
    assert np.min(np.abs(I / 0.8 - 1)) > 1e-4
    assert np.min(np.abs(I / 6.0 - 1)) > 1e-4
    C, S = c.num_channels, c.num_src
    tt = torch.float64 if real == np.float64 else torch.float32
    flux = [torch.zeros(C * S, dtype=tt, device="cuda") for _ in range(4)]
    ob.call("oskb_sky_scale_flux_channels_" + suffix(real), S, sky.capacity,
            sky.num_columns, C, dev(c.freqs), dev(sky.table),
            dev(sky.num_valid), np.array(sky.cols, np.int32), S, *flux,
            ob.stream_ptr())
    vis = dev(np.zeros(c.num_times * C * c.nbl * 8, real))
    ob.call("oskb_correlate_block_direct_spectral_" + suffix(real), c.casa,
            S, c.num_st, c.num_times, C, dev(c.E), 0, *flux, S, dev(c.l),
            dev(c.m), dev(c.n), dev(c.a), dev(c.b), dev(c.c), dev(c.uvw),
            dev(c.st_x), dev(c.st_y), dev(c.inv_wl), c.bw, c.tavg,
            dev(c.gha0), c.dec0, c.uv_min_m, c.uv_max_m, 0, c.filter_min,
            c.filter_max, vis, ob.stream_ptr())
    torch.cuda.synchronize()
    assert rel(vis.cpu().numpy(), c.oracle_vis()) <= TOL[real]
    st = ob.call("oskb_correlate_block_direct_spectral_" + suffix(real),
                 c.casa, S, c.num_st, c.num_times, C, dev(c.E), 0, *flux,
                 S - 1, dev(c.l), dev(c.m), dev(c.n), dev(c.a), dev(c.b),
                 dev(c.c), dev(c.uvw), dev(c.st_x), dev(c.st_y),
                 dev(c.inv_wl), c.bw, c.tavg, dev(c.gha0), c.dec0,
                 c.uv_min_m, c.uv_max_m, 0, c.filter_min, c.filter_max, vis,
                 ob.stream_ptr(), check=False)
    assert st == -3  # stride shorter than a channel's sources


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_block_plan_spectral_sky(real):
    """The block plan with a spectral sky: scaled once when set, then every
    block (eager, then graph replays) correlates per-channel brightness."""
    import ctypes
    lib = ob.load()
    c, sky = _spectral_case(real, num_st=45, chunks=(80, 40),
                            gaussian=(1, 0), num_channels=3)
    st = ctypes.c_int(0)
    plan = lib.oskb_block_plan_create(
        8 if real == np.float64 else 4, c.casa, c.num_st, c.num_src,
        c.num_times, c.num_channels, 1, 1, 0,
        c.freqs.ctypes.data, c.bw, c.tavg, c.dec0, c.uv_min_m, c.uv_max_m,
        0, c.filter_min, c.filter_max, ctypes.addressof(st))
    assert st.value == 0 and plan
    try:
        cols = np.array(sky.cols, np.int32)
        assert ob.call("oskb_block_plan_set_spectral_sky", plan,
                       sky.capacity, sky.num_columns, sky.table,
                       sky.num_valid, cols) == 0
        assert ob.call("oskb_block_plan_set_sky", plan, None, None, None,
                       None, c.l, c.m, c.n, c.a, c.b, c.c) == 0
        assert ob.call("oskb_block_plan_set_stations", plan, c.st_x,
                       c.st_y) == 0
        assert ob.call("oskb_block_plan_set_beam", plan, c.E) == 0
        nvis = c.num_times * c.num_channels * c.nbl * 8
        uvw = _host_view(lib.oskb_block_plan_host_uvw(plan), c.uvw.size,
                         real)
        gha0 = _host_view(lib.oskb_block_plan_host_gha0(plan), c.num_times,
                          np.float64)
        vis = _host_view(lib.oskb_block_plan_host_vis(plan), nvis, real)
        for block in range(3):
            if block:
                rng = np.random.default_rng(200 + block)
                c.uvw = rng.uniform(-3e3, 3e3, c.uvw.shape).astype(real)
                c.gha0 = rng.uniform(-1, 1, c.num_times)
            uvw[:] = c.uvw.ravel()
            gha0[:] = c.gha0
            assert ob.call("oskb_block_plan_execute", plan) == 0
            assert ob.call("oskb_block_plan_synchronize", plan) == 0
            assert rel(vis.copy(), c.oracle_vis()) <= TOL[real], block
        assert lib.oskb_block_plan_graph_launches(plan) == 2
    finally:
        lib.oskb_block_plan_free(plan)


def test_block_c4_shape_sampled():
    """The batched-smearing configuration's shape with its sky scaled down
    200 times: 256 stations, 32 chunks whose sizes are drawn log-uniform on
    [500, 50,000] and divided by 200 (Gaussian chunks as the reference
    flags them), 64 channels of 100 kHz, 2 dumps, bandwidth and time
    smearing, FP64, one launch for the whole block; the oracle computes
    channels 0, 21, 42 and 63 of both dumps, which must agree to 1e-12 of
    the block's largest visibility in those channels."""
    rng = np.random.default_rng(4)
    sizes = np.maximum(3, (np.exp(rng.uniform(np.log(500), np.log(50_000),
                                              32)) / 200).astype(int))
    gauss = (rng.uniform(0, 1, 32) < 0.9).astype(int)
    c = BlockCase(num_st=256, chunks=tuple(int(x) for x in sizes),
                  gaussian=tuple(int(g) for g in gauss), num_times=2,
                  num_channels=64, seed=44)
    c.freqs = 100e6 + 1e5 * np.arange(64)
    c.inv_wl = c.freqs / 299792458.0
    got = run_block(c).reshape(2, 64, -1)
    chans = (0, 21, 42, 63)
    ref = c.oracle_vis(channels=chans).reshape(2, 64, -1)
    for ch in chans:
        assert rel(got[:, ch], ref[:, ch]) <= 1e-12, ch
