"""Pins the CPU oracle against the reference's own CPU kernels.

oracle/_ref/liboskar_ref.so is the reference's code compiled from its sources
(oracle/Makefile, target "ref"); the oracle must agree with it on every
function and variant the hot path uses. Both run on the same seeded inputs.
"""
import itertools

import numpy as np
import pytest

from oracle_lib import oracle, reference, reference_xcorr, suffix
from xcorr_cases import XcorrCase
from beam_cases import enu_dirs as _enu_dirs, beam_case, oracle_beam

pytestmark = pytest.mark.skipif(reference() is None,
                                reason="reference sources not present")

TOL = {np.float64: 1e-13, np.float32: 2e-5}


def _close(a, b, real):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = np.max(np.abs(b)) + 1e-300
    return np.max(np.abs(a - b)) / scale <= TOL[real]


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("matrix", [True, False])
@pytest.mark.parametrize("gaussian", [False, True])
@pytest.mark.parametrize("bw,ts", [(0.0, 0.0), (10e3, 0.0), (0.0, 10.0),
                                   (10e3, 10.0)])
@pytest.mark.parametrize("casa", [0, 1])
def test_xcorr(real, matrix, gaussian, bw, ts, casa):
    c = XcorrCase(19, 277, real=real, matrix=matrix, gaussian=gaussian,
                  bandwidth_hz=bw, time_avg=ts, casa=casa, offset_out=3)
    v_orc, v_ref = c.vis0.copy(), c.vis0.copy()
    oracle().call("xcorr_" + ("matrix_" if matrix else "scalar_")
                  + suffix(real), real, casa, int(gaussian),
                  *c.oracle_args(v_orc))
    reference_xcorr(real, matrix, gaussian, casa, *c.oracle_args(v_ref))
    assert _close(v_orc, v_ref, real)
    assert not np.array_equal(v_orc, c.vis0)


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_xcorr_uv_filter(real):
    c = XcorrCase(12, 50, real=real, uv_min=0.5, uv_max=1.2)
    v_orc, v_ref = c.vis0.copy(), c.vis0.copy()
    oracle().call("xcorr_matrix_" + suffix(real), real, 0, 0,
                  *c.oracle_args(v_orc))
    reference_xcorr(real, True, False, 0, *c.oracle_args(v_ref))
    assert _close(v_orc, v_ref, real)
    # some baselines filtered out, some kept
    changed = np.any((v_orc != c.vis0).reshape(-1, 8), axis=1)
    assert changed.any() and not changed.all()


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("matrix", [True, False])
def test_acorr(real, matrix):
    c = XcorrCase(9, 101, real=real, matrix=matrix)
    nc = 8 if matrix else 2
    v0 = np.random.default_rng(5).uniform(-1, 1, 12 * nc).astype(real)
    v_orc, v_ref = v0.copy(), v0.copy()
    if matrix:
        args = (c.num_src, c.num_st, 2, c.jones, c.I, c.Q, c.U, c.V)
    else:
        args = (c.num_src, c.num_st, 2, c.jones, c.I)
    name = "acorr_" + ("matrix_" if matrix else "scalar_") + suffix(real)
    oracle().call(name, real, *args, v_orc)
    reference().call(name, real, *args, v_ref)
    assert _close(v_orc, v_ref, real)


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("ignore_w", [0, 1])
def test_jones_k(real, ignore_w):
    rng = np.random.default_rng(3)
    ns, nst = 1000, 100
    l, m, n = (rng.uniform(0.1, 0.9, ns).astype(real) for _ in range(3))
    u, v, w = (rng.uniform(-1e3, 1e3, nst).astype(real) for _ in range(3))
    f = rng.uniform(0, 2, ns).astype(real)
    k = 2 * np.pi * 100e6 / 299792458.0
    out_o = np.zeros(2 * ns * nst, real)
    out_r = np.zeros(2 * ns * nst, real)
    args = (ns, l, m, n, nst, u, v, w, k, f, 0.5, 1.5, ignore_w)
    oracle().call("jones_k_" + suffix(real), real, *args, out_o)
    reference().call("jones_k_" + suffix(real), real, *args, out_r)
    assert _close(out_o, out_r, real)
    assert np.count_nonzero(out_o) < out_o.size  # the filter zeroed some


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("kind,na,nb,nc", [("cc_c", 2, 2, 2),
                                           ("cc_m", 2, 2, 8),
                                           ("cm_m", 2, 8, 8),
                                           ("mc_m", 8, 2, 8),
                                           ("mm_m", 8, 8, 8)])
def test_mem_mul(real, kind, na, nb, nc):
    rng = np.random.default_rng(4)
    n = 777
    a = rng.uniform(-2, 2, n * na).astype(real)
    b = rng.uniform(-2, 2, n * nb).astype(real)
    co, cr = np.zeros(n * nc, real), np.zeros(n * nc, real)
    oracle().call("mem_mul_%s_%s" % (kind, suffix(real)), real, n, a, b, co)
    reference().call("mem_mul_%s_%s" % (kind, suffix(real)), real, n, a, b,
                     cr)
    assert _close(co, cr, real)


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("matrix,is_3d,use_idx,ex,ey",
                         [(0, 0, 0, 1, 1), (0, 1, 1, 1, 1), (1, 0, 0, 1, 1),
                          (1, 1, 1, 1, 1), (1, 1, 1, 1, 0), (1, 0, 1, 0, 1)])
def test_dftw(real, matrix, is_3d, use_idx, ex, ey):
    rng = np.random.default_rng(6)
    n_in, n_out, n_types, off_c, off_o = 64, 301, 3, 5, 7
    k = 2 * np.pi * 100e6 / 299792458.0
    w = rng.uniform(-1, 1, 2 * n_in).astype(real)
    xi, yi, zi = (rng.uniform(-20, 20, n_in).astype(real) for _ in range(3))
    xo, yo, zo = (rng.uniform(-1, 1, n_out + off_c).astype(real)
                  for _ in range(3))
    idx = (rng.integers(0, n_types, n_in).astype(np.int32) if use_idx
           else None)
    nd = n_types if use_idx else n_in
    nc = 8 if matrix else 2
    data = rng.uniform(-1, 1, nd * n_out * nc).astype(real)
    out0 = rng.uniform(-1, 1, (n_out + off_o) * nc).astype(real)
    oo, orr = out0.copy(), out0.copy()
    args = (matrix, is_3d, n_in, k, w, xi, yi, zi if is_3d else None, off_c,
            n_out, xo, yo, zo if is_3d else None, idx, data, ex, ey, off_o)
    oracle().call("dftw_" + suffix(real), real, *args, oo, 1.0 / n_in)
    reference().call("dftw_" + suffix(real), real, *args, orr, 1.0 / n_in)
    assert _close(oo, orr, real)


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_element_weights_and_uvw(real):
    rng = np.random.default_rng(7)
    n = 256
    x, y, z, cab = (rng.uniform(-20, 20, n).astype(real) for _ in range(4))
    k = 2 * np.pi * 110e6 / 299792458.0
    wo, wr = np.zeros(2 * n, real), np.zeros(2 * n, real)
    args = (n, x, y, z, cab, k, 0.3, -0.2, 0.93)
    oracle().call("element_weights_dft_" + suffix(real), real, *args, wo)
    reference().call("element_weights_dft_" + suffix(real), real, *args, wr)
    assert _close(wo, wr, real)
    outs = [[np.zeros(n + 2, real) for _ in range(3)] for _ in range(2)]
    for ign, (lib, o) in itertools.product([0, 1], zip(
            [oracle(), reference()], outs)):
        lib.call("ecef_to_station_uvw_" + suffix(real), real, n, x, y, z,
                 0.3, 0.95, -0.5, 0.86, ign, 2, *o)
        if lib is reference():
            for a, b in zip(outs[0], outs[1]):
                assert _close(a, b, real)


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("pole", [0, 1])
def test_enu_to_theta_phi(real, pole):
    rng = np.random.default_rng(11)
    n, off = 500, 3
    x, y, z = _enu_dirs(rng, n + off, real)
    outs = [[np.zeros(n + 1, real) for _ in range(3)] for _ in range(2)]
    for lib, o in zip([oracle(), reference()], outs):
        lib.call("enu_to_theta_phi_" + suffix(real), real, off, n, x, y, z,
                 pole, -0.7, 1.2, *o)
    for a, b in zip(*outs):
        assert _close(a, b, real)


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("swap", [0, 1])
def test_dipole_pattern(real, swap):
    rng = np.random.default_rng(12)
    n = 700
    th = rng.uniform(0, np.pi / 2, n).astype(real)
    th[:3] = 0  # at the pole the pattern denominator may vanish
    px, py = (rng.uniform(0, 2 * np.pi, n).astype(real) for _ in range(2))
    px[1], py[2] = 0, np.pi / 2
    kL = 1.5 * np.pi * 150e6 / 299792458.0
    outs = [np.zeros(8 * (n + 2), real) for _ in range(2)]
    for lib, o in zip([oracle(), reference()], outs):
        lib.call("dipole_pattern_" + suffix(real), real, n, th, px, py,
                 real(kL), real(np.cos(kL)), swap, 2, o)
    assert _close(outs[0], outs[1], real)


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_normalise_blank_jones_r(real):
    rng = np.random.default_rng(13)
    n = 300
    a0 = rng.uniform(-1, 1, 8 * n).astype(real)
    a = [a0.copy(), a0.copy()]
    for lib, o in zip([oracle(), reference()], a):
        lib.call("mem_normalise_matrix_" + suffix(real), real, 5, 200, o, 77)
    assert _close(a[0], a[1], real)
    mask = rng.uniform(-1, 1, n + 4).astype(real)
    b = [a0.copy(), a0.copy()]
    for lib, o in zip([oracle(), reference()], b):
        lib.call("blank_below_horizon_" + suffix(real), real, 4, n - 2, mask,
                 2, o)
    assert np.array_equal(b[0], b[1])
    ra, dec = (rng.uniform(-1.5, 1.5, n).astype(real) for _ in range(2))
    lat, lst = -0.47, 2.1
    r = [np.zeros(8 * (n + 1), real) for _ in range(2)]
    for lib, o in zip([oracle(), reference()], r):
        lib.call("jones_r_" + suffix(real), real, n, ra, dec,
                 real(np.cos(lat)), real(np.sin(lat)), real(lst), 1, o)
    assert _close(r[0], r[1], real)


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("flags", [(1, 1, 1, 0, 1), (0, 1, 1, 1, 0),
                                   (1, 0, 0, 0, 1), (0, 0, 1, 0, 0)])
def test_station_beam_composition(real, flags):
    """The oracle's composite station beam equals the same chain built from
    the reference's own kernels, step by step."""
    norm_el, norm_arr, norm_fin, swap, is_3d = flags
    c = beam_case(real, num_dir=301)
    got = oracle_beam(c, real, flags)
    ref, s = reference(), suffix(real)
    nd = len(c["dirs"][0])
    npt = nd + norm_fin
    X, Y, Z = (np.ascontiguousarray(np.append(d, real(v)), dtype=real)
               [:npt].copy() for d, v in zip(c["dirs"], c["norm"]))
    th, p1, p2 = (np.zeros(npt + 1, real) for _ in range(3))
    dphi1 = np.pi / 2 - (c["orient"][0] + np.pi / 2)
    dphi2 = np.pi / 2 - c["orient"][1]
    ref.call("enu_to_theta_phi_" + s, real, 0, npt, X, Y, Z, norm_el,
             real(dphi1), real(dphi2), th, p1, p2)
    kL = c["L"] * (np.pi * c["freq"] / 299792458.0)
    sig = np.zeros(8 * (npt + 1), real)
    ref.call("dipole_pattern_" + s, real, npt + norm_el, th, p1, p2,
             real(kL), real(np.cos(kL)), swap, 0, sig)
    if norm_el:
        ref.call("mem_normalise_matrix_" + s, real, 0, npt, sig, npt)
    k = 2 * np.pi * c["freq"] / 299792458.0
    w = np.zeros(2 * len(c["el"][0]), real)
    ref.call("element_weights_dft_" + s, real, len(w) // 2, *c["meas"],
             c["cable"], real(k), *(real(v) for v in c["b"]), w)
    out = np.zeros(8 * npt, real)
    ref.call("dftw_" + s, real, 1, is_3d, len(w) // 2, real(k), w, *c["el"],
             0, npt, X, Y, Z if is_3d else None,
             np.zeros(len(w) // 2, np.int32), sig, 1, 1, 0, out,
             real(1.0 / (len(w) // 2)) if norm_arr else real(1))
    ref.call("blank_below_horizon_" + s, real, 0, npt, Z, 0, out)
    if norm_fin:
        ref.call("mem_normalise_matrix_" + s, real, 0, npt, out, npt - 1)
    assert np.array_equal(got, out[:8 * nd]) or _close(got, out[:8 * nd],
                                                        real)
    assert np.count_nonzero(got) > 0


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_direction_conversions_and_horizon(real):
    rng = np.random.default_rng(16)
    n = 500
    lon = rng.uniform(0, 2 * np.pi, n).astype(real)
    lat = rng.uniform(-1.5, 1.5, n).astype(real)
    c0, s0 = real(np.cos(-0.5)), real(np.sin(-0.5))
    for three_d in (True, False):
        outs = [[np.zeros(n, real) for _ in range(3)] for _ in range(2)]
        for lib, o in zip([oracle(), reference()], outs):
            lib.call("lon_lat_to_relative_directions_" + suffix(real), real,
                     n, lon, lat, real(0.3), c0, s0, o[0], o[1],
                     o[2] if three_d else None)
        for a, b in zip(*outs):
            assert _close(a, b, real) or not b.any()
    outs = [[np.zeros(n + 3, real) for _ in range(3)] for _ in range(2)]
    for lib, o in zip([oracle(), reference()], outs):
        lib.call("ra_dec_to_enu_directions_" + suffix(real), real, n, lon,
                 lat, real(1.7), real(np.sin(-0.47)), real(np.cos(-0.47)), 3,
                 *o)
    for a, b in zip(*outs):
        assert _close(a, b, real)
    l, m, nn = (rng.uniform(-1, 1, n).astype(real) for _ in range(3))
    masks = [np.zeros(n, np.int32), np.zeros(n, np.int32)]
    for lib, mk in zip([oracle(), reference()], masks):
        for mul in ((0.3, -0.2, 0.9), (-0.8, 0.1, 0.2)):
            lib.call("update_horizon_mask_" + suffix(real), real, n, l, m, nn,
                     *(real(x) for x in mul), mk)
    assert np.array_equal(masks[0], masks[1])
    assert 0 < masks[0].sum() < n


@pytest.mark.parametrize("casa", [0, 1])
def test_baseline_uvw_known_answer(casa):
    """The reference's baseline order (p < q, q fastest) and sign
    (convert/src/oskar_convert_station_uvw_to_baseline_uvw.c:18-28)."""
    u = np.array([0.0, 1.0, 3.0, 7.0]); v = 2 * u; w = -u
    out = [np.zeros(8) for _ in range(3)]
    oracle().call("station_uvw_to_baseline_uvw_d", np.float64, casa, 4, 0,
                  u, v, w, 2, *out)
    f = -1 if casa else 1
    pairs = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]
    assert np.array_equal(out[0][2:], [f * (u[q] - u[p]) for p, q in pairs])
    assert np.array_equal(out[1][2:], [f * (v[q] - v[p]) for p, q in pairs])
    assert np.array_equal(out[2][2:], [f * (w[q] - w[p]) for p, q in pairs])


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("freq", [40e6, 101e6, 150e6, 102.4e6, 250e6])
def test_sky_scale_flux(real, freq):
    """Every spectral and polarisation model, NaN coefficients included,
    against the reference's flux-scaling kernel."""
    from sky_cases import SkyTable, call_scale, random_sky
    sky = SkyTable(random_sky(700, 17), real)
    got = call_scale(oracle(), real, sky, freq)
    ref = call_scale(reference(), real, sky, freq)
    tol = 1e-15 if real == np.float64 else 1e-6
    for g, r in zip(got, ref):
        np.testing.assert_allclose(g, r, rtol=tol, atol=tol * 10)


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_sky_scale_flux_sparse_table(real):
    """A table with only I, reference frequency and spectral index columns
    (every other column index is -1)."""
    from sky_cases import SkyTable, call_scale
    rng = np.random.default_rng(3)
    srcs = [{"I": [float(rng.uniform(1, 5))],
             "REF_HZ": [float(rng.uniform(80e6, 120e6))],
             "SPX": list(rng.uniform(-1, 0.5, 1 + s % 3))}
            for s in range(300)]
    sky = SkyTable(srcs, real)
    assert sky.cols.count(-1) == 11
    got = call_scale(oracle(), real, sky, 110e6)
    ref = call_scale(reference(), real, sky, 110e6)
    for g, r in zip(got, ref):
        np.testing.assert_allclose(g, r, rtol=1e-6, atol=0)


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("matrix", [True, False])
@pytest.mark.parametrize("ex,ey", [(1, 1), (1, 0), (0, 1)])
def test_cable_length_errors_and_gains(real, matrix, ex, ey):
    rng = np.random.default_rng(5)
    nst, nsrc = 13, 71
    width = 8 if matrix else 2
    J = rng.normal(size=nst * nsrc * width).astype(real)
    dx = rng.uniform(-2, 2, nst).astype(real) if ex else None
    dy = rng.uniform(-2, 2, nst).astype(real) if ey else None
    k = real(2 * np.pi * 150e6 / 299792458.0)
    a, b = J.copy(), J.copy()
    oracle().call("cable_length_errors_" + suffix(real), real, int(matrix),
                  nsrc, nst, k, dx, dy, a)
    reference().call("cable_length_errors_" + suffix(real), real,
                     int(matrix), nsrc, nst, k, dx, dy, b)
    assert _close(a, b, real)
    if ex or matrix:
        assert not np.array_equal(a, J)
    G = rng.normal(size=nst * width).astype(real)
    oracle().call("station_gains_" + suffix(real), real, int(matrix), nsrc,
                  nst, G, a)
    reference().call("station_gains_" + suffix(real), real, int(matrix),
                     nsrc, nst, G, b)
    assert _close(a, b, real)


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 255, 4096])
def test_random_gaussian(real, n):
    """The oracle's Philox4x32-10 + Box-Muller fill against the reference's
    own CPU fill (mem/src/oskar_mem_random_gaussian.c with its vendored
    Random123), bit for bit, including the ragged last quad."""
    for seed, c1, c2, c3 in [(1, 0, 0, 0), (42, 7, 3, 0x12345678),
                             (0xFFFFFFF0, 123456, 65535, 0xDEADBEEF)]:
        a = np.zeros(n, real)
        b = np.ones(n, real)
        oracle().call("random_gaussian_" + suffix(real), real, n, a, seed,
                      c1, c2, c3, 2.5)
        reference().call("random_gaussian_" + suffix(real), real, n, b,
                         seed, c1, c2, c3, 2.5)
        assert np.array_equal(a, b)
    big = np.zeros(200_000, real)
    oracle().call("random_gaussian_" + suffix(real), real, len(big), big, 3,
                  1, 2, 3, 1.0)
    assert abs(big.mean()) < 0.01 and abs(big.std() - 1) < 0.01


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_element_weights_errors(real):
    """Time-variable element gain/phase errors
    (oskar_evaluate_element_weights_errors.c:19-110): oracle against the
    reference's CPU chain, bit for bit, for several stations and times."""
    rng = np.random.default_rng(8)
    n = 257
    gain = rng.uniform(0.9, 1.1, n).astype(real)
    gain_err = rng.uniform(0, 0.1, n).astype(real)
    phase = rng.uniform(-0.2, 0.2, n).astype(real)
    phase_err = rng.uniform(0, 0.05, n).astype(real)
    for seed, t, st in [(1, 0, 0), (99, 5, 17), (2**31 + 5, 1000, 511)]:
        a = np.zeros(2 * n, real)
        b = np.ones(2 * n, real)
        oracle().call("element_weights_errors_" + suffix(real), real, n,
                      gain, gain_err, phase, phase_err, seed, t, st, a)
        reference().call("element_weights_errors_" + suffix(real), real, n,
                         gain, gain_err, phase, phase_err, seed, t, st, b)
        assert np.array_equal(a, b)
        amp = np.hypot(a[0::2], a[1::2])
        assert np.all(np.abs(amp - gain) <= 6 * gain_err + 1e-6)


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("matrix", [True, False])
def test_beam_pattern_powers(real, matrix):
    """Beam-pattern auto and cross power: oracle against the reference's
    own CPU kernels (define_evaluate_{auto,cross}_power.h)."""
    rng = np.random.default_rng(21)
    nst, nsrc, w = 23, 97, 8 if matrix else 2
    J = rng.normal(size=nst * nsrc * w).astype(real)
    stokes = (1.0, 0.2, -0.1, 0.05)
    for name, args in (("auto_power_", (int(matrix), nst * nsrc, 0, J,
                                        *stokes, 3)),
                       ("cross_power_", (int(matrix), nsrc, nst, J, *stokes,
                                         2.0 / (nst * (nst - 1)), 3))):
        n_out = (nst * nsrc if name == "auto_power_" else nsrc) + 3
        a, b = np.zeros(n_out * w, real), np.zeros(n_out * w, real)
        oracle().call(name + suffix(real), real, *args, a)
        reference().call(name + suffix(real), real, *args, b)
        assert _close(a, b, real)
