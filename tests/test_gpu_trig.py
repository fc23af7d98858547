"""The table-driven FP64 phase factors of the weighted DFT and station-beam
element loops (oskb_phase_factors_d) against numpy's sin/cos and CUDA's own
sin/cos (torch on the device) on the same phases: at most 4e-16 absolute
error (about two ulp of 1) over the phase ranges the loops see and beyond,
exact multiples of the table step, the edges of the reduction window and
non-finite phases."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(),
                                 reason="needs a CUDA device")]

import oskar_b200 as ob  # noqa: E402

BOUND = 4e-16


def phase_factors(ph):
    d = torch.from_numpy(np.ascontiguousarray(ph, np.float64)).cuda()
    out = torch.empty(2 * len(ph), dtype=torch.float64, device="cuda")
    assert ob.call("oskb_phase_factors_d", len(ph), d, out,
                   ob.stream_ptr()) == 0
    torch.cuda.synchronize()
    o = out.cpu().numpy()
    return o[0::2], o[1::2], d


@pytest.mark.parametrize("scale", [1.0, np.pi, 100.0, 1e3, 1e5, 1e7, 1e10])
def test_phase_factors_random(scale):
    rng = np.random.default_rng(int(scale) % 1000 + 1)
    ph = rng.uniform(-scale, scale, 300_001)
    c, s, d = phase_factors(ph)
    assert np.max(np.abs(c - np.cos(ph))) <= BOUND
    assert np.max(np.abs(s - np.sin(ph))) <= BOUND
    # CUDA's sin/cos on the same device arrays
    assert np.max(np.abs(c - torch.cos(d).cpu().numpy())) <= BOUND
    assert np.max(np.abs(s - torch.sin(d).cpu().numpy())) <= BOUND


def test_phase_factors_special_points():
    step = np.pi / 64
    n = np.arange(-5000, 5001, dtype=np.float64)
    ph = np.concatenate([
        n * step,                          # on the table's nodes
        n * step + step / 2,               # half-way between nodes
        n * step - step / 2,
        np.nextafter(n * step + step / 2, 0),
        [0.0, -0.0, 1e-300, -1e-300, 5e-324],
        [2.0**40 * 0.999999, -(2.0**40) * 0.999999],  # inside the window
        [2.0**40, -(2.0**40), 3e12, -7e15],           # library sincos
    ])
    c, s, _ = phase_factors(ph)
    assert np.max(np.abs(c - np.cos(ph))) <= BOUND
    assert np.max(np.abs(s - np.sin(ph))) <= BOUND
    # |e^{i ph}| stays 1 to rounding
    assert np.max(np.abs(c * c + s * s - 1.0)) <= 6e-16
    # the zero phase gives exactly 1 + 0i
    assert c[-11] == 1.0 and s[-11] == 0.0


def test_phase_factors_non_finite():
    c, s, _ = phase_factors(np.array([np.inf, -np.inf, np.nan, 1.0]))
    assert np.all(np.isnan(c[:3])) and np.all(np.isnan(s[:3]))
    assert abs(c[3] - np.cos(1.0)) <= BOUND


def test_phase_factors_arguments():
    lib = ob.load()
    assert lib.oskb_phase_factors_d(0, None, None, None) == 0
    assert lib.oskb_phase_factors_d(-1, None, None, None) != 0
