"""The beam-pattern driver (oskar_b200/beam_pattern.py) on the GPU against
the oracle composed the way the reference's application runs a chunk
(oskar_beam_pattern_run.c:276-500): pixel directions rotated to ENU at the
dump's sidereal time, each active station's beam by the oracle's station
beam chain (pinned to the reference's kernels in tests/test_oracle_pin.py),
normalised to the beam direction, then the auto and cross power of the
oracle for an unpolarised unit source and for the test source. The
rotation itself is checked against the reference's CPU function.
Tolerances: FP64 1e-12, FP32 2e-5 of the largest value (max and L2)."""
import ctypes
import math
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(),
                                 reason="needs a CUDA device")]

from oskar_b200 import beam_pattern as bpm  # noqa: E402
import oskar_b200 as ob  # noqa: E402
from oracle_lib import oracle, suffix  # noqa: E402

TOL = {np.float64: 1e-12, np.float32: 2e-5}
HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(os.path.dirname(HERE), "oracle", "_ref",
                       "liboskar_refcpu.so")


def rel(got, ref):
    got, ref = np.asarray(got), np.asarray(ref)
    d = np.abs(got - ref)
    return max(d.max() / np.abs(ref).max(),
               np.linalg.norm(got - ref) / np.linalg.norm(ref))


def rel_to_enu(l, m, n, ha0, dec0, lat):
    """The rotation of define_convert_relative_directions_to_enu_directions.h
    in numpy (FP64)."""
    sh, ch = math.sin(ha0), math.cos(ha0)
    sd, cd = math.sin(dec0), math.cos(dec0)
    sl, cl = math.sin(lat), math.cos(lat)
    x = l * ch + m * sh * sd - n * sh * cd
    t = sl * ch
    y = -l * sl * sh + m * (cl * cd + t * sd) + n * (cl * sd - t * cd)
    t = cl * ch
    z = l * cl * sh + m * (sl * cd - t * sd) + n * (sl * sd + t * cd)
    return x, y, z


def transit_mjd(lon_deg, ra_deg, ha_deg=-15.0, near=58000.0):
    """An MJD near `near` when the hour angle of ra_deg from lon_deg is
    ha_deg (so the field is well above the horizon)."""
    best, best_d = near, 1e9
    for k in range(2000):
        mjd = near + k / 2000.0
        lst = bpm.mjd_to_gast(mjd) + math.radians(lon_deg)
        d = abs(math.remainder(lst - math.radians(ra_deg) -
                               math.radians(ha_deg), 2 * math.pi))
        if d < best_d:
            best, best_d = mjd, d
    return best


def stations(rng, ns=4, ne=16):
    g = np.arange(4) * 1.6 - 2.4
    gx, gy = np.meshgrid(g, g)
    ex = np.stack([gx.ravel() + rng.normal(0, 0.1, ne) for _ in range(ns)])
    ey = np.stack([gy.ravel() + rng.normal(0, 0.1, ne) for _ in range(ns)])
    ez = rng.uniform(-0.05, 0.05, (ns, ne))
    return ex, ey, ez


def test_rel_to_enu_matches_reference():
    """The device rotation against the reference's CPU
    oskar_convert_relative_directions_to_enu_directions (oskar_Mem
    arguments, from its CPU library)."""
    if not os.path.exists(REF_LIB):
        pytest.skip("reference library not built")
    lib = ctypes.CDLL(REF_LIB, mode=ctypes.RTLD_GLOBAL)
    P, I = ctypes.c_void_p, ctypes.c_int
    lib.oskar_mem_create.restype = P
    lib.oskar_mem_create.argtypes = [I, I, ctypes.c_size_t,
                                     ctypes.POINTER(I)]
    lib.oskar_mem_void.restype = P
    lib.oskar_mem_void.argtypes = [P]
    f = lib.oskar_convert_relative_directions_to_enu_directions
    f.restype = None
    f.argtypes = [I, I, I, I, P, P, P, ctypes.c_double, ctypes.c_double,
                  ctypes.c_double, I, P, P, P, ctypes.POINTER(I)]
    rng = np.random.default_rng(3)
    n = 5000
    l, m = rng.uniform(-0.5, 0.5, n), rng.uniform(-0.5, 0.5, n)
    nn = np.sqrt(1 - l * l - m * m)
    st = I(0)
    mems = [lib.oskar_mem_create(8, 0, n, ctypes.byref(st))
            for _ in range(6)]
    for mem, a in zip(mems[:3], (l, m, nn)):
        ctypes.memmove(lib.oskar_mem_void(mem), a.ctypes.data, 8 * n)
    ha0, dec0, lat = 0.7, -0.5, -0.47
    f(0, 0, 0, n, *mems[:3], ha0, dec0, lat, 0, *mems[3:], ctypes.byref(st))
    assert st.value == 0
    ref = [np.ctypeslib.as_array(ctypes.cast(lib.oskar_mem_void(mem),
           ctypes.POINTER(ctypes.c_double)), (n,)).copy()
           for mem in mems[3:]]
    dev = lambda a: torch.from_numpy(a).cuda()
    out = [torch.empty(n, dtype=torch.float64, device="cuda")
           for _ in range(3)]
    ob.call("oskb_convert_relative_directions_to_enu_directions_d", n,
            dev(l), dev(m), dev(nn), ha0, dec0, lat, *out, ob.stream_ptr())
    torch.cuda.synchronize()
    for o, r in zip(out, ref):
        assert np.max(np.abs(o.cpu().numpy() - r)) <= 1e-15
    # the numpy restatement used below is the same rotation
    for a, r in zip(rel_to_enu(l, m, nn, ha0, dec0, lat), ref):
        assert np.max(np.abs(a - r)) <= 1e-15


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_beam_pattern_matches_oracle(real):
    rng = np.random.default_rng(7)
    ex, ey, ez = stations(rng)
    ox = rng.uniform(0, 10, 4)
    oy = ox + rng.uniform(-5, 5, 4)
    b = bpm.BeamPattern(116.76, -26.82, ex, ey, ez, 20.0, -30.0,
                        orientation_x_deg=ox, orientation_y_deg=oy,
                        dipole_length_m=1.4,
                        precision="double" if real == np.float64 else
                        "single")
    b.set_image(24, 20, 30.0, 25.0)
    b.set_observation(transit_mjd(116.76, 20.0), 1800.0, 2, 110e6, 15e6, 2)
    ids = [2, 0, 3]
    b.set_station_ids(ids)
    src = (2.0, 0.3, -0.2, 0.1)
    b.set_test_source(*src)
    out = b.run()
    l, m, n = b.pixel_grid()
    npix = l.size
    s = suffix(real)
    for t in range(2):
        lst = bpm.mjd_to_gast(b.time_mjd(t)) + b.lon
        ha0 = lst - b.ra0
        dirs = [np.ascontiguousarray(a, real)
                for a in rel_to_enu(l, m, n, ha0, b.dec0, b.lat)]
        bxyz = rel_to_enu(0.0, 0.0, 1.0, ha0, b.dec0, b.lat)
        if real == np.float32:
            bxyz = [float(np.float32(v)) for v in bxyz]
        for c in range(2):
            f = 110e6 + 15e6 * c
            J = np.zeros((len(ids), npix * 8), real)
            for k, st in enumerate(ids):
                oracle().call("station_beam_aa_" + s, np.float64, 16,
                              *[np.ascontiguousarray(a[st], real)
                                for a in (ex, ey, ez)], None, None, None,
                              np.zeros(16, real), math.radians(ox[st]),
                              math.radians(oy[st]), 1.4, 1, 1, 1, 0, 1, f,
                              *bxyz, *bxyz, npix, *dirs, J[k])
            Jc = J.reshape(len(ids), npix, 8)
            got = out["jones"][t, c].reshape(len(ids), npix, 4)
            ref = Jc[..., 0::2] + 1j * Jc[..., 1::2]
            assert rel(got, ref) <= TOL[real], ("jones", t, c)
            for kk, stokes in enumerate(((1.0, 0.0, 0.0, 0.0), src)):
                ap = np.zeros(len(ids) * npix * 8, real)
                oracle().call("auto_power_" + s, real, 1, len(ids) * npix, 0,
                              J.ravel(), *[real(v) for v in stokes], 0, ap)
                apc = ap.reshape(len(ids), npix, 8)
                got = out["auto_power"][kk, t, c].reshape(len(ids), npix, 4)
                assert rel(got, apc[..., 0::2] + 1j * apc[..., 1::2]) <= \
                    TOL[real], ("auto", kk, t, c)
                cp = np.zeros(npix * 8, real)
                nst = len(ids)
                oracle().call("cross_power_" + s, real, 1, npix, nst,
                              J.ravel(), *[real(v) for v in stokes],
                              real(2.0 / (nst * (nst - 1))), 0, cp)
                cpc = cp.reshape(npix, 8)
                got = out["cross_power"][kk, t, c].reshape(npix, 4)
                assert rel(got, cpc[..., 0::2] + 1j * cpc[..., 1::2]) <= \
                    TOL[real], ("cross", kk, t, c)
    # a beam pattern peaks at the pointing: the central pixels' station
    # beams are ~1 after the normalisation, the edges well below
    amp = bpm.amplitude(out["jones"][0, 0, 0, :, 0, 0]).reshape(20, 24)
    assert amp[9:11, 11:13].max() > 0.9 and amp[0, 0] < 0.5


def test_beam_pattern_fits_cube(tmp_path):
    """Auto-power Stokes I images averaged over time, written and read
    back."""
    rng = np.random.default_rng(8)
    ex, ey, ez = stations(rng, ns=2)
    b = bpm.BeamPattern(116.76, -26.82, ex, ey, ez, 20.0, -30.0)
    b.set_image(16, 12, 20.0, 15.0)
    b.set_observation(transit_mjd(116.76, 20.0), 600.0, 3, 100e6, 5e6, 2)
    out = b.run(jones=False, cross_power=False)
    stokes_i = bpm.linear_to_stokes(out["auto_power"][0], 0)  # t, c, st, pix
    img = bpm.average(stokes_i, axis=0)[:, 0].real.reshape(2, 12, 16)
    path = tmp_path / "auto_power_I.fits"
    bpm.write_fits(str(path), img[None], b)
    hdr, data = bpm.read_fits(str(path))
    assert data.shape == (1, 2, 12, 16)
    assert np.array_equal(data[0], img)
    assert img.max() > 0.8 and np.all(img >= 0.0)
