"""Beam-pattern auto and cross power on the GPU against the oracle, which
is pinned against the reference's CPU kernels
(tests/test_oracle_pin.py::test_beam_pattern_powers). The cross power
runs as one pass with prefix sums, the oracle as the reference's loop over
station pairs, so the sums are ordered differently. Tolerances: FP64
1e-12, FP32 2e-5 of the largest value (max and L2)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(),
                                 reason="needs a CUDA device")]

import oskar_b200 as ob  # noqa: E402
from oracle_lib import oracle, suffix  # noqa: E402

TOL = {np.float64: 1e-12, np.float32: 2e-5}


def rel(got, ref):
    got, ref = np.asarray(got, np.float64), np.asarray(ref, np.float64)
    return max(np.max(np.abs(got - ref)) / np.max(np.abs(ref)),
               np.linalg.norm(got - ref) / np.linalg.norm(ref))


def beams(real, nst, nsrc, matrix, seed):
    """Station beams with a common main lobe, so the cross power has the
    dynamic range of a beam pattern."""
    rng = np.random.default_rng(seed)
    w = 8 if matrix else 2
    lobe = np.exp(-np.linspace(0, 6, nsrc) ** 2)
    J = rng.normal(0, 0.05, (nst, nsrc, w))
    J[..., 0] += lobe
    if matrix:
        J[..., 6] += lobe
    return np.ascontiguousarray(J.ravel().astype(real))


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("matrix", [True, False])
@pytest.mark.parametrize("nst,nsrc", [(2, 1), (3, 100), (64, 4097),
                                      (512, 3000)])
def test_cross_power(real, matrix, nst, nsrc):
    """FP32 is checked against the FP64 oracle on the same (FP32-valued)
    inputs: the reference's own FP32 pair loop is off the FP64 result by
    5.3e-5 at 512 stations here, the prefix-sum order by ~1e-6."""
    J = beams(real, nst, nsrc, matrix, nst)
    w = 8 if matrix else 2
    stokes = (1.0, 0.1, -0.05, 0.02)
    ref = np.zeros((nsrc + 5) * w)
    oracle().call("cross_power_d", np.float64, int(matrix), nsrc, nst,
                  J.astype(np.float64), *stokes, 2.0 / (nst * (nst - 1)), 5,
                  ref)
    out = torch.zeros((nsrc + 5) * w, dtype=torch.float64 if real ==
                      np.float64 else torch.float32, device="cuda")
    ob.call("oskb_evaluate_cross_power_" + suffix(real), int(matrix), nsrc,
            nst, torch.from_numpy(J).cuda(), *stokes, 5, out,
            ob.stream_ptr())
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert not got[:5 * w].any()
    assert rel(got, ref) <= TOL[real], rel(got, ref)


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("matrix", [True, False])
def test_auto_power(real, matrix):
    J = beams(real, 7, 1001, matrix, 3)
    w = 8 if matrix else 2
    n = 7 * 1001 - 4
    stokes = (2.0, -0.3, 0.2, 0.1)
    ref = np.zeros((n + 2) * w, real)
    oracle().call("auto_power_" + suffix(real), real, int(matrix), n, 4, J,
                  *stokes, 2, ref)
    out = torch.zeros((n + 2) * w, dtype=torch.float64 if real ==
                      np.float64 else torch.float32, device="cuda")
    ob.call("oskb_evaluate_auto_power_" + suffix(real), int(matrix), n, 4,
            torch.from_numpy(J).cuda(), *stokes, 2, out, ob.stream_ptr())
    torch.cuda.synchronize()
    assert rel(out.cpu().numpy(), ref) <= TOL[real]


def test_power_arguments():
    lib = ob.load()
    assert lib.oskb_evaluate_cross_power_d(1, 0, 5, None, 1.0, 0.0, 0.0,
                                           0.0, 0, None, None) == 0
    assert lib.oskb_evaluate_cross_power_d(1, 4, 5, None, 1.0, 0.0, 0.0,
                                           0.0, 0, None, None) != 0
    assert lib.oskb_evaluate_auto_power_d(1, -1, 0, None, 1.0, 0.0, 0.0,
                                          0.0, 0, None, None) != 0
