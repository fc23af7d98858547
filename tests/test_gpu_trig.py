"""The table-driven FP64 phase factors of the weighted DFT and station-beam
element loops (oskb_phase_factors_d: e^{i pi u / 64} for a phase u given
in table steps) against long-double cos/sin of the same phase and against
CUDA's own sin/cos (torch on the device) where the phase in radians is
exact enough to compare: at most 4e-16 absolute error (about two ulp of 1)
over the phase ranges the loops see and beyond, on and between the
table's nodes, at the edges of the range the table covers and for
non-finite phases."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(),
                                 reason="needs a CUDA device")]

import oskar_b200 as ob  # noqa: E402

BOUND = 4e-16
PI_LD = np.arccos(np.longdouble(-1))


def phase_factors(u):
    d = torch.from_numpy(np.ascontiguousarray(u, np.float64)).cuda()
    out = torch.empty(2 * len(u), dtype=torch.float64, device="cuda")
    assert ob.call("oskb_phase_factors_d", len(u), d, out,
                   ob.stream_ptr()) == 0
    torch.cuda.synchronize()
    o = out.cpu().numpy()
    return o[0::2], o[1::2]


def exact(u):
    """cos, sin of pi u / 64 in long double, u reduced mod 128 exactly
    first (fmod of a double by a power of two is exact)."""
    r = np.fmod(np.asarray(u, np.float64), 128.0).astype(np.longdouble)
    x = r * PI_LD / 64
    return np.cos(x).astype(np.float64), np.sin(x).astype(np.float64)


def check(u, bound=BOUND):
    c, s = phase_factors(u)
    ce, se = exact(u)
    assert np.max(np.abs(c - ce)) <= bound
    assert np.max(np.abs(s - se)) <= bound
    return c, s


@pytest.mark.parametrize("scale", [1.0, 64.0, 1e3, 1e5, 1e7, 4e9])
def test_phase_factors_random(scale):
    rng = np.random.default_rng(int(scale) % 997 + 1)
    check(rng.uniform(-scale, scale, 300_001))


def test_phase_factors_against_cuda_sincos():
    """|phase| < pi: pi u / 64 rounds to within 2.2e-16 rad, so CUDA's
    sin/cos of the rounded radians may differ by that much more."""
    rng = np.random.default_rng(5)
    u = rng.uniform(-64, 64, 200_001)
    c, s = phase_factors(u)
    ph = torch.from_numpy(u * (np.pi / 64)).cuda()
    assert np.max(np.abs(c - torch.cos(ph).cpu().numpy())) <= 2 * BOUND
    assert np.max(np.abs(s - torch.sin(ph).cpu().numpy())) <= 2 * BOUND


def test_phase_factors_special_points():
    n = np.arange(-5000, 5001, dtype=np.float64)
    u = np.concatenate([
        n, n + 0.5, n - 0.5,                 # nodes and half-way points
        np.nextafter(n + 0.5, 0), np.nextafter(n - 0.5, 0),
        [0.0, -0.0, 1e-300, -1e-300, 5e-324],
        # either side of the covered range -2^32 <= round(u) < 2^32
        [2.0**32 - 0.75, 2.0**32 - 0.5, 2.0**32, 2.0**32 + 1,
         -(2.0**32) - 0.25, -(2.0**32) - 0.5, -(2.0**32) - 1],
        [2.0**51, -(2.0**52), 3e15, 1e300],  # library sincospi
    ])
    c, s = check(u)
    assert np.max(np.abs(c * c + s * s - 1.0)) <= 6e-16
    zero = 5 * len(n)
    assert c[zero] == 1.0 and s[zero] == 0.0     # e^{i 0} = 1 exactly


def test_phase_factors_non_finite():
    c, s = phase_factors(np.array([np.inf, -np.inf, np.nan, 1.0]))
    assert np.all(np.isnan(c[:3])) and np.all(np.isnan(s[:3]))
    assert abs(c[3] - np.cos(np.pi / 64)) <= BOUND


def test_phase_factors_arguments():
    lib = ob.load()
    assert lib.oskb_phase_factors_d(0, None, None, None) == 0
    assert lib.oskb_phase_factors_d(-1, None, None, None) != 0
