"""Host-side pieces of the beam-pattern driver (oskar_b200/beam_pattern.py),
no GPU needed: the beam-image pixel grid of the C ABI against the
reference's own oskar_evaluate_image_lmn_grid_d and the fast GAST against
oskar_convert_mjd_to_gast_fast (both from oracle/_ref/liboskar_refcpu.so,
the reference's CPU library built from its sources), the image products
(Stokes, IXR) on known answers, and the FITS writer read back."""
import ctypes
import math
import os

import numpy as np
import pytest

from oskar_b200 import beam_pattern as bp
from oskar_b200._lib import call

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(os.path.dirname(HERE), "oracle", "_ref",
                       "liboskar_refcpu.so")


def ref_lib():
    if not os.path.exists(REF_LIB):
        pytest.skip("reference library not built")
    return ctypes.CDLL(REF_LIB, mode=ctypes.RTLD_GLOBAL)


@pytest.mark.parametrize("w,h,fov", [(64, 48, (3.0, 2.0)), (7, 9, (40.0, 90.0)),
                                     (33, 33, (180.0, 180.0)), (1, 1, (5, 5))])
@pytest.mark.parametrize("centred", [1, 0])
def test_image_grid_matches_reference(w, h, fov, centred):
    lib = ref_lib()
    f = lib.oskar_evaluate_image_lmn_grid_d
    f.restype = None
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double,
                  ctypes.c_double, ctypes.c_int] + [ctypes.c_void_p] * 3
    ref = [np.zeros(w * h) for _ in range(3)]
    f(w, h, math.radians(fov[0]), math.radians(fov[1]), centred,
      *[a.ctypes.data for a in ref])
    got = [np.zeros(w * h) for _ in range(3)]
    assert call("oskb_evaluate_image_lmn_grid", w, h, math.radians(fov[0]),
                math.radians(fov[1]), centred, *got, check=False) == 0
    for g, r in zip(got, ref):
        assert np.array_equal(np.isnan(g), np.isnan(r))
        assert np.array_equal(g[~np.isnan(g)], r[~np.isnan(r)])


def test_gast_matches_reference():
    lib = ref_lib()
    f = lib.oskar_convert_mjd_to_gast_fast
    f.restype = ctypes.c_double
    f.argtypes = [ctypes.c_double]
    for mjd in np.linspace(40000.0, 70000.0, 101):
        assert abs(bp.mjd_to_gast(mjd) - f(mjd)) <= 1e-12


def test_products_known_answers():
    # unpolarised power: XX = YY = 1 -> I = 1, Q = U = V = 0
    p = np.array([[1.0, 0.0], [0.0, 1.0]], complex)
    assert [bp.linear_to_stokes(p, k) for k in range(4)] == [1, 0, 0, 0]
    # XY = 1 + 0.5i, YX = 1 - 0.5i -> U = 1, V = -0.5i (1i) = 0.5
    p = np.array([[0.0, 1 + 0.5j], [1 - 0.5j, 0.0]])
    assert bp.linear_to_stokes(p, 2) == 1.0
    assert abs(bp.linear_to_stokes(p, 3) - 0.5) < 1e-15
    # cond(diag(1, 0.5)) = 2 -> IXR = 9; the identity is capped
    assert abs(bp.ixr(np.diag([1.0, 0.5]).astype(complex)) - 9.0) < 1e-12
    assert bp.ixr(np.eye(2, dtype=complex)) == 1e8


def test_fits_round_trip(tmp_path):
    class P:
        ra0, dec0 = math.radians(20.0), math.radians(-30.0)
        fov = (4.0, 3.0)
        freq_start_hz, freq_inc_hz = 100e6, 1e6
        mjd_start, inc_sec = 51544.5, 60.0
    rng = np.random.default_rng(1)
    cube = rng.normal(size=(2, 3, 5, 7))
    path = tmp_path / "beam.fits"
    bp.write_fits(str(path), cube, P)
    assert os.path.getsize(path) % 2880 == 0
    hdr, data = bp.read_fits(str(path))
    assert np.array_equal(data, cube)
    assert hdr["NAXIS1"] == 7 and hdr["NAXIS4"] == 2
    assert hdr["CTYPE1"] == "RA---SIN" and hdr["CTYPE2"] == "DEC--SIN"
    assert abs(hdr["CRVAL1"] - 20.0) < 1e-12
    cell = math.degrees(math.asin(2 * math.sin(math.radians(2.0)) / 7))
    assert abs(hdr["CDELT1"] + cell) < 1e-12
    assert hdr["CRPIX2"] == 3.0
