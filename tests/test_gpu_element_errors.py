"""Element weight factors on the GPU against the CPU oracle, whose random
fill and error kernel are pinned bit for bit against the reference's own
CPU code (tests/test_oracle_pin.py::test_random_gaussian,
::test_element_weights_errors):

  - oskb_evaluate_element_weights_errors: time-variable gain and phase
    errors of one station (Philox4x32-10 + Box-Muller on the device);
  - oskb_station_element_weight_factors: errors x apodisation for many
    stations in one launch, per-station and shared error tables;
  - oskb_station_beam_aa_weighted: the fused station beam with those
    factors on the element weights, against the oracle's station beam
    composed as oskar_station_evaluate_element_weights applies them.

The device draws its Gaussian angle with sincospi as the reference's GPU
path does, the oracle with sin(pi x) as its CPU path does; they agree to
rounding. Tolerances: FP64 1e-12, FP32 2e-5 of the largest value."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(),
                                 reason="needs a CUDA device")]

import oskar_b200 as ob  # noqa: E402
from beam_cases import beam_case  # noqa: E402
from oracle_lib import oracle, suffix  # noqa: E402

TOL = {np.float64: 1e-12, np.float32: 2e-5}


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def rel(got, ref):
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    return max(np.max(np.abs(got - ref)) / np.max(np.abs(ref)),
               np.linalg.norm(got - ref) / np.linalg.norm(ref))


def tables(real, n, seed):
    rng = np.random.default_rng(seed)
    return [rng.uniform(0.9, 1.1, n).astype(real),
            rng.uniform(0.0, 0.1, n).astype(real),
            rng.uniform(-0.2, 0.2, n).astype(real),
            rng.uniform(0.0, 0.05, n).astype(real)]


def oracle_errors(real, tab, seed, t, station_id):
    out = np.zeros(2 * len(tab[0]), real)
    oracle().call("element_weights_errors_" + suffix(real), real,
                  len(tab[0]), *tab, seed, t, station_id, out)
    return out


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("n", [1, 2, 3, 256, 1001])
def test_element_weights_errors(real, n):
    tab = tables(real, n, n)
    for seed, t, st in [(1, 0, 0), (77, 9, 130), (2**31 + 3, 4000, 511)]:
        out = torch.zeros(2 * n, dtype=torch.float64 if real == np.float64
                          else torch.float32, device="cuda")
        ob.call("oskb_evaluate_element_weights_errors_" + suffix(real), n,
                *[dev(a) for a in tab], seed, t, st, out, ob.stream_ptr())
        torch.cuda.synchronize()
        assert rel(out.cpu().numpy(), oracle_errors(real, tab, seed, t,
                                                    st)) <= TOL[real]


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("per_station", [0, 1])
@pytest.mark.parametrize("errors,apod", [(1, 1), (1, 0), (0, 1), (0, 0)])
def test_station_weight_factors(real, per_station, errors, apod):
    nst, n, first, seed, t = 5, 97, 12, 1234, 3
    rng = np.random.default_rng(3)
    tabs = [tables(real, n, 10 + s) for s in range(nst)] if per_station \
        else [tables(real, n, 10)] * nst
    apod_w = rng.normal(1, 0.1, (nst, 2 * n)).astype(real)
    ref = np.zeros((nst, 2 * n), real)
    for s in range(nst):
        e = (oracle_errors(real, tabs[s], seed, t, first + s) if errors
             else np.tile(np.array([1, 0], real), n))
        if apod:
            a = apod_w[s, 0::2] + 1j * apod_w[s, 1::2]
            z = (e[0::2] + 1j * e[1::2]) * a
            e = np.stack([z.real, z.imag], 1).ravel().astype(real)
        ref[s] = e
    if errors:
        dtab = ([dev(np.concatenate([tb[i] for tb in tabs])) for i in range(4)]
                if per_station else [dev(a) for a in tabs[0]])
    else:
        dtab = [None] * 4
    out = torch.full((nst * 2 * n,), 7.0, dtype=torch.float64 if real ==
                     np.float64 else torch.float32, device="cuda")
    ob.call("oskb_station_element_weight_factors_" + suffix(real), nst, n,
            first, seed, t, *dtab, per_station,
            dev(apod_w) if apod else None, out, ob.stream_ptr())
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(nst, 2 * n)
    assert rel(got, ref) <= TOL[real]


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("flags", [(1, 1, 1, 0, 1), (0, 1, 0, 1, 0)])
def test_station_beam_with_weight_factors(real, flags):
    """Three stations in one launch, each with its own errors (station ids
    7, 8, 9) and apodisation; the factors visibly change the beam."""
    norm_el, norm_arr, norm_fin, swap, is_3d = flags
    cases = [beam_case(real, seed=50 + s, num_el=256, num_dir=777,
                       is_3d=is_3d) for s in range(3)]
    nst, n = len(cases), 256
    rng = np.random.default_rng(4)
    tab = tables(real, n, 21)
    apod = rng.normal(1, 0.2, (nst, 2 * n)).astype(real)
    factors = torch.zeros(nst * 2 * n, dtype=torch.float64 if real ==
                          np.float64 else torch.float32, device="cuda")
    ob.call("oskb_station_element_weight_factors_" + suffix(real), nst, n, 7,
            99, 2, *[dev(a) for a in tab], 0, dev(apod), factors,
            ob.stream_ptr())
    f_host = factors.cpu().numpy().reshape(nst, 2 * n)
    cat = lambda key, i: dev(np.concatenate([c[key][i] for c in cases]))
    dirs = [dev(cases[0]["dirs"][i]) for i in range(3)]
    out = torch.zeros(nst * 777 * 8, dtype=factors.dtype, device="cuda")
    ob.call("oskb_station_beam_aa_weighted_" + suffix(real), nst, n,
            *[cat("el", i) for i in range(3)],
            *[cat("meas", i) for i in range(3)],
            dev(np.concatenate([c["cable"] for c in cases])), factors,
            dev(np.array([c["orient"][0] for c in cases])),
            dev(np.array([c["orient"][1] for c in cases])), cases[0]["L"],
            norm_el, norm_arr, norm_fin, swap, is_3d, cases[0]["freq"],
            dev(np.stack([c["b"] for c in cases])),
            dev(np.stack([c["norm"] for c in cases])), 777, *dirs, 0, out,
            ob.stream_ptr())
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(nst, -1)
    for s, c in enumerate(cases):
        ref = np.zeros(8 * 777, real)
        plain = np.zeros(8 * 777, real)
        for wf, dst in ((f_host[s].copy(), ref), (None, plain)):
            oracle().call("station_beam_aa_weighted_" + suffix(real),
                          np.float64, n, *c["el"], *c["meas"], c["cable"],
                          wf, *c["orient"], c["L"], norm_el, norm_arr,
                          norm_fin, swap, is_3d, c["freq"], *c["b"],
                          *c["norm"], 777, *cases[0]["dirs"], dst)
        assert rel(got[s], ref) <= TOL[real], (s, rel(got[s], ref))
        assert rel(plain, ref) > 1e-3


def test_weight_factor_arguments():
    lib = ob.load()
    # errors requested without their tables
    assert lib.oskb_station_element_weight_factors_d(
        2, 4, 0, 1, 0, 1, None, None, None, 0, None, 1, None) != 0
    assert lib.oskb_station_element_weight_factors_d(
        0, 4, 0, 1, 0, None, None, None, None, 0, None, None, None) == 0
    assert lib.oskb_evaluate_element_weights_errors_d(
        4, None, None, None, None, 1, 0, 0, None, None) != 0
