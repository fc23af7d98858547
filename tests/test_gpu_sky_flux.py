"""Sky flux scaling with frequency and the per-station Jones terms (cable
phase errors, station gains) on the GPU, against the oracle, plus the
known answers of the reference's flux-scaling tests
(oskar/sky/test/Test_Sky_scale_flux_with_frequency.cpp)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(),
                                 reason="needs a CUDA device")]

import oskar_b200 as ob  # noqa: E402
from oskar_b200 import oskar_api as oa  # noqa: E402
from oskar_b200._lib import load  # noqa: E402
from oracle_lib import oracle, suffix  # noqa: E402
from sky_cases import (SkyTable, call_scale, mixed_types_expected,  # noqa
                       mixed_types_sky, random_sky, spectral_index_expected,
                       spectral_index_sky)

# Relative to max(|value|, 1). FP64: libm differences only. FP32: float
# arithmetic is ill-conditioned for parts of the random sky: a Faraday angle
# rm lambda^2 of up to ~300 rad at 40 MHz, and Gaussian-line exponents
# (f - f0)^2 / 2 sigma^2 of up to ~100, turn one float rounding into ~2e-4
# (the FP32 oracle differs from the FP64 oracle by as much), so the FP32
# bound is 5e-4 on every value and 2e-6 on the median.
REL = {np.float64: 1e-12, np.float32: 5e-4}
MEDIAN = {np.float64: 1e-13, np.float32: 2e-6}
ERR_INVALID_ARGUMENT, ERR_TYPE_MISMATCH = -3, -9  # oskar/oskar_global.h


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def tt(real):
    return torch.float64 if real == np.float64 else torch.float32


def gpu_scale(sky, real, freq):
    n = sky.num_sources
    out = [torch.full((max(n, 1),), -7.0, dtype=tt(real), device="cuda")
           for _ in range(4)]
    ob.call("oskb_sky_scale_flux_with_frequency_" + suffix(real), n,
            sky.capacity, sky.num_columns, float(freq), dev(sky.table),
            dev(sky.num_valid), *sky.cols, *out, ob.stream_ptr())
    torch.cuda.synchronize()
    return [o.cpu().numpy()[:n] for o in out]


def check(got, ref, real):
    for g, r in zip(got, ref):
        g = np.asarray(g, np.float64)
        r = np.asarray(r, np.float64)
        err = np.abs(g - r) / np.maximum(np.abs(r), 1.0)
        assert np.all(err <= REL[real]), float(np.max(err))
        assert np.median(err) <= MEDIAN[real], float(np.median(err))


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("freq", [40e6, 101e6, 150e6, 250e6])
def test_scale_flux_random_sky(real, freq):
    sky = SkyTable(random_sky(3000, 23), real)
    check(gpu_scale(sky, real, freq), call_scale(oracle(), real, sky, freq),
          real)


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_scale_flux_channels_one_launch(real):
    """The band entry: every channel in one launch, [channel][source] with a
    padded stride, equal to one single-frequency call per channel."""
    sky = SkyTable(random_sky(1500, 29), real)
    freqs = np.linspace(95e6, 135e6, 7)
    n, stride = sky.num_sources, sky.num_sources + 5
    out = [torch.zeros(len(freqs) * stride, dtype=tt(real), device="cuda")
           for _ in range(4)]
    cols = np.array(sky.cols, np.int32)
    ob.call("oskb_sky_scale_flux_channels_" + suffix(real), n, sky.capacity,
            sky.num_columns, len(freqs), dev(freqs), dev(sky.table),
            dev(sky.num_valid), cols, stride, *out, ob.stream_ptr())
    torch.cuda.synchronize()
    got = [o.cpu().numpy().reshape(len(freqs), stride) for o in out]
    for c, f in enumerate(freqs):
        f_arg = float(np.float32(f)) if real == np.float32 else f
        ref = call_scale(oracle(), real, sky, f_arg)
        check([g[c, :n] for g in got], ref, real)
        assert np.all(got[0][c, n:] == 0)


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_reference_known_answers(real):
    """The mixed-spectral-type and spectral-index tests of the reference,
    with its tolerances (Test_Sky_scale_flux_with_frequency.cpp:36, 217)."""
    tol_mixed = 5e-5 if real == np.float32 else 1e-12
    tol_spx = 2e-5 if real == np.float32 else 3e-14
    sky = SkyTable(mixed_types_sky(), real)
    for i in range(0, 100, 3):
        f = 95e6 + i * 100e3
        got = gpu_scale(sky, real, f)[0]
        np.testing.assert_allclose(got, mixed_types_expected(f), rtol=0,
                                   atol=tol_mixed)
    n = 10000
    sky = SkyTable(spectral_index_sky(n), real)
    for f in (100e6, 60e6, 5e6):
        np.testing.assert_allclose(np.array(gpu_scale(sky, real, f)),
                                   spectral_index_expected(n, f), rtol=0,
                                   atol=tol_spx)


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_rotation_measure_round_trip(real):
    srcs = [{"I": [10.0], "Q": [1.0], "U": [0.0], "V": [0.1], "RM": [0.5],
             "REF_HZ": [100e6]} for _ in range(100)]
    sky = SkyTable(srcs, real)
    _, q, u, _ = gpu_scale(sky, real, 99e6)
    assert np.all(q != 1.0) and np.all(u != 0.0)
    _, q, u, _ = gpu_scale(sky, real, 100e6)
    tol = 5e-5 if real == np.float32 else 1e-12
    np.testing.assert_allclose(q, 1.0, atol=tol, rtol=0)
    np.testing.assert_allclose(u, 0.0, atol=tol, rtol=0)


def test_scale_flux_errors_and_empty():
    sky = SkyTable(random_sky(10, 1), np.float64)
    out = [torch.zeros(10, dtype=torch.float64, device="cuda")
           for _ in range(4)]
    cols = list(sky.cols)
    cols[0] = -1  # no Stokes I column
    st = ob.call("oskb_sky_scale_flux_with_frequency_d", 10, sky.capacity,
                 sky.num_columns, 1e8, dev(sky.table), dev(sky.num_valid),
                 *cols, *out, ob.stream_ptr(), check=False)
    assert st == ERR_INVALID_ARGUMENT
    st = ob.call("oskb_sky_scale_flux_with_frequency_d", 0, sky.capacity,
                 sky.num_columns, 1e8, None, None, *sky.cols, None, None,
                 None, None, ob.stream_ptr(), check=False)
    assert st == 0
    st = ob.call("oskb_sky_scale_flux_with_frequency_d", 10, 5,
                 sky.num_columns, 1e8, dev(sky.table), dev(sky.num_valid),
                 *sky.cols, *out, ob.stream_ptr(), check=False)
    assert st == ERR_INVALID_ARGUMENT  # capacity < sources


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("matrix", [True, False])
@pytest.mark.parametrize("ex,ey", [(1, 1), (1, 0), (0, 1)])
def test_cable_length_errors_and_gains(real, matrix, ex, ey):
    rng = np.random.default_rng(7)
    nst, nsrc = 37, 1029
    width = 8 if matrix else 2
    J = rng.normal(size=nst * nsrc * width).astype(real)
    dx = rng.uniform(-3, 3, nst).astype(real) if ex else None
    dy = rng.uniform(-3, 3, nst).astype(real) if ey else None
    k = real(2 * np.pi * 150e6 / 299792458.0)
    s = suffix(real)
    dJ = dev(J)
    ob.call("oskb_jones_apply_cable_length_errors_" + s, int(matrix), nsrc,
            nst, float(k), None if dx is None else dev(dx),
            None if dy is None else dev(dy), dJ, ob.stream_ptr())
    ref = J.copy()
    oracle().call("cable_length_errors_" + s, real, int(matrix), nsrc, nst,
                  k, dx, dy, ref)
    torch.cuda.synchronize()
    got = dJ.cpu().numpy()
    tol = 1e-14 if real == np.float64 else 2e-6
    assert np.max(np.abs(got - ref)) <= tol * np.max(np.abs(ref))
    G = rng.normal(size=nst * width).astype(real)
    ob.call("oskb_jones_apply_station_gains_" + s, int(matrix), nsrc, nst,
            dev(G), dJ, ob.stream_ptr())
    oracle().call("station_gains_" + s, real, int(matrix), nsrc, nst, G, ref)
    torch.cuda.synchronize()
    got = dJ.cpu().numpy()
    assert np.max(np.abs(got - ref)) <= 4 * tol * np.max(np.abs(ref))


@pytest.mark.parametrize("prec", [oa.OSKAR_DOUBLE, oa.OSKAR_SINGLE])
def test_oskar_named_gains_and_cable_errors(prec):
    """oskar_jones_apply_cable_length_errors / _station_gains on oskar_Jones
    containers, as the reference's simulator calls them
    (oskar_interferometer_run_block.c:287-304)."""
    lib = load()
    real = np.float64 if prec == oa.OSKAR_DOUBLE else np.float32
    mtype = prec | oa.OSKAR_COMPLEX | oa.OSKAR_MATRIX
    rng = np.random.default_rng(9)
    nst, nsrc = 11, 300
    J = rng.normal(size=nst * nsrc * 8).astype(real)
    j = oa.jones_from_numpy(J, mtype, nst, nsrc, oa.OSKAR_GPU)
    ex = oa.mem_from_numpy(rng.uniform(-2, 2, nst).astype(real), prec)
    G = rng.normal(size=nst * 8).astype(real)
    g = oa.mem_from_numpy(G, mtype)
    st = oa.ctypes.c_int(0)
    lib.oskar_jones_apply_cable_length_errors(j, oa.ctypes.c_double(120e6),
                                              ex, None, oa.status_ptr(st))
    assert st.value == 0
    lib.oskar_jones_apply_station_gains(j, g, oa.status_ptr(st))
    assert st.value == 0
    got = oa.mem_to_numpy(lib.oskar_jones_mem(j))
    ref = J.copy()
    k = real(2 * np.pi * 120e6 / 299792458.0)
    oracle().call("cable_length_errors_" + suffix(real), real, 1, nsrc, nst,
                  k, oa.mem_to_numpy(ex), None, ref)
    oracle().call("station_gains_" + suffix(real), real, 1, nsrc, nst, G,
                  ref)
    tol = 1e-14 if real == np.float64 else 4e-6
    assert np.max(np.abs(got - ref)) <= tol * np.max(np.abs(ref))
    # mismatched gain type: an error, nothing launched
    g2 = oa.mem_from_numpy(G[: 2 * nst].copy(),
                           prec | oa.OSKAR_COMPLEX)
    lib.oskar_jones_apply_station_gains(j, g2, oa.status_ptr(st))
    assert st.value == ERR_TYPE_MISMATCH
    oa.free_jones(j)
    oa.free_mem(ex, g, g2)
