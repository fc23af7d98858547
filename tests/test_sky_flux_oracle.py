"""The oracle's flux scaling against the known answers of the reference's
own tests (oskar/sky/test/Test_Sky_scale_flux_with_frequency.cpp): the ten
mixed spectral models, the spectral-index sky and the rotation-measure
round trip, with the reference test's tolerances."""
import numpy as np
import pytest

from oracle_lib import oracle
from sky_cases import (SkyTable, call_scale, mixed_types_expected,
                       mixed_types_sky, spectral_index_expected,
                       spectral_index_sky)

# Test_Sky_scale_flux_with_frequency.cpp:217 (FP32, FP64), :36
TOL_MIXED = {np.float32: 5e-5, np.float64: 1e-12}
TOL_SPX = {np.float32: 2e-5, np.float64: 3e-14}


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_mixed_spectral_types(real):
    sky = SkyTable(mixed_types_sky(), real)
    for i in range(100):
        f = 95e6 + i * 100e3
        got = call_scale(oracle(), real, sky, f)[0]
        np.testing.assert_allclose(got, mixed_types_expected(f), rtol=0,
                                   atol=TOL_MIXED[real])
        assert got[0] == 1.0


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_spectral_index(real):
    n = 2000
    sky = SkyTable(spectral_index_sky(n), real)
    for f in (100e6, 80e6, 60e6, 40e6, 20e6, 5e6):
        got = np.array(call_scale(oracle(), real, sky, f))
        want = spectral_index_expected(n, f)
        np.testing.assert_allclose(got, want, rtol=0, atol=TOL_SPX[real])


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_rotation_measure_round_trip(real):
    """Test_Sky_scale_flux_with_frequency.cpp:406-470: Faraday rotation
    moves Q and U away from the reference frequency and back at it."""
    srcs = [{"I": [10.0], "Q": [1.0], "U": [0.0], "V": [0.1], "RM": [0.5],
             "REF_HZ": [100e6]} for _ in range(100)]
    sky = SkyTable(srcs, real)
    _, q, u, _ = call_scale(oracle(), real, sky, 99e6)
    assert np.all(q != 1.0) and np.all(u != 0.0)
    _, q, u, _ = call_scale(oracle(), real, sky, 100e6)
    tol = TOL_MIXED[real]
    np.testing.assert_allclose(q, 1.0, atol=tol, rtol=0)
    np.testing.assert_allclose(u, 0.0, atol=tol, rtol=0)


def test_no_reference_frequency_keeps_flux():
    """A source whose nearest reference frequency is 0 keeps its values."""
    sky = SkyTable([{"I": [2.0], "Q": [0.5], "U": [0.25], "V": [0.1],
                     "REF_HZ": [0.0], "SPX": [-0.7]}], np.float64)
    got = call_scale(oracle(), np.float64, sky, 150e6)
    assert [g[0] for g in got] == [2.0, 0.5, 0.25, 0.1]
