"""GPU parity of the fused station beam (Jones E) and of Jones R against the
CPU oracle, whose composite station beam is pinned step by step against the
reference's own kernels (tests/test_oracle_pin.py).

Three stations with different layouts, element orientations and pointings
are evaluated in one launch and compared with the oracle station by station.
Tolerances: FP64 1e-12 of the largest beam value (max and L2 relative);
FP32 2e-5.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(),
                                 reason="needs a CUDA device")]

import oskar_b200 as ob  # noqa: E402
from beam_cases import beam_case, oracle_beam  # noqa: E402
from oracle_lib import oracle, suffix  # noqa: E402

TOL = {np.float64: 1e-12, np.float32: 2e-5}


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def rel(got, ref):
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    return max(np.max(np.abs(got - ref)) / np.max(np.abs(ref)),
               np.linalg.norm(got - ref) / np.linalg.norm(ref))


def stations(real, num_st=3, num_el=256, num_dir=1001, is_3d=1):
    cases = [beam_case(real, seed=30 + s, num_el=num_el, num_dir=num_dir,
                       is_3d=is_3d) for s in range(num_st)]
    for s, c in enumerate(cases):
        c["orient"] = (0.1 * s, 0.1 * s + np.pi / 2)
        c["dirs"] = cases[0]["dirs"]  # shared directions unless per-station
    return cases


def run_gpu(cases, real, flags, per_station_dirs=False):
    norm_el, norm_arr, norm_fin, swap, is_3d = flags
    st = len(cases)
    cat = lambda key, i: dev(np.concatenate([c[key][i] for c in cases]))
    el = [cat("el", i) for i in range(3)]
    me = [cat("meas", i) for i in range(3)]
    cable = dev(np.concatenate([c["cable"] for c in cases]))
    ox = dev(np.array([c["orient"][0] for c in cases]))
    oy = dev(np.array([c["orient"][1] for c in cases]))
    b = dev(np.stack([c["b"] for c in cases]))
    nrm = dev(np.stack([c["norm"] for c in cases]))
    nd = len(cases[0]["dirs"][0])
    if per_station_dirs:
        dirs = [cat("dirs", i) for i in range(3)]
    else:
        dirs = [dev(cases[0]["dirs"][i]) for i in range(3)]
    out = torch.zeros(st * nd * 8, dtype=torch.float64 if real == np.float64
                      else torch.float32, device="cuda")
    ob.call("oskb_station_beam_aa_" + suffix(real), st, len(cases[0]["cable"]),
            *el, *me, cable, ox, oy, cases[0]["L"], norm_el, norm_arr,
            norm_fin, swap, is_3d, cases[0]["freq"], b, nrm, nd, *dirs,
            int(per_station_dirs), out, ob.stream_ptr())
    torch.cuda.synchronize()
    return out.cpu().numpy().reshape(st, nd * 8)


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("flags", [(1, 1, 1, 0, 1), (0, 1, 1, 1, 0),
                                   (1, 0, 0, 0, 1), (0, 0, 1, 0, 0)])
def test_station_beam_vs_oracle(real, flags):
    cases = stations(real, is_3d=flags[4])
    cases[2]["b"] = np.array([-0.5, 0.1, np.sqrt(1 - 0.26)])
    cases[2]["norm"] = cases[2]["b"].copy()
    got = run_gpu(cases, real, flags)
    for s, c in enumerate(cases):
        ref = oracle_beam(c, real, flags)
        assert rel(got[s], ref) <= TOL[real], (s, rel(got[s], ref))
        blank = c["dirs"][2] < 0
        assert not got[s].reshape(-1, 8)[blank].any()


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_station_beam_per_station_directions(real):
    """Per-station direction cosines ([station][direction])."""
    cases = [beam_case(real, seed=40 + s, num_el=200, num_dir=513)
             for s in range(2)]
    flags = (1, 1, 1, 0, 1)
    got = run_gpu(cases, real, flags, per_station_dirs=True)
    for s, c in enumerate(cases):
        assert rel(got[s], oracle_beam(c, real, flags)) <= TOL[real]


def test_station_beam_pointing_below_horizon_is_zero():
    cases = stations(np.float64, num_st=2, num_dir=300)
    cases[1]["b"] = np.array([0.0, 0.6, -0.8])
    got = run_gpu(cases, np.float64, (1, 1, 1, 0, 1))
    assert got[0].any() and not got[1].any()


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_jones_r_vs_oracle(real):
    rng = np.random.default_rng(15)
    ns, nst = 2000, 4
    ra = rng.uniform(-np.pi, np.pi, ns).astype(real)
    dec = rng.uniform(-1.5, 1.5, ns).astype(real)
    lat = rng.uniform(-0.8, 0.8, nst)
    lst = rng.uniform(0, 2 * np.pi, nst)
    out = torch.zeros(nst * ns * 8, dtype=torch.float64 if real == np.float64
                      else torch.float32, device="cuda")
    ob.call("oskb_evaluate_jones_R_" + suffix(real), ns, dev(ra), dev(dec),
            nst, dev(lat), dev(lst), out, ob.stream_ptr())
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(nst, -1)
    for s in range(nst):
        ref = np.zeros(8 * ns, real)
        oracle().call("jones_r_" + suffix(real), real, ns, ra, dec,
                      real(np.cos(lat[s])), real(np.sin(lat[s])),
                      real(lst[s]), 0, ref)
        assert rel(got[s], ref) <= (1e-13 if real == np.float64 else 2e-5)


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("num_types", [1, 2, 3, 4])
@pytest.mark.parametrize("flags", [(1, 1, 1, 0, 1), (0, 0, 1, 1, 0)])
@pytest.mark.parametrize("model", ["dipoles", "isotropic+tapers"])
def test_station_beam_element_types(real, num_types, flags, model):
    """Stations with several element types, each a dipole length and an
    orientation of its own: one launch for three stations, each with its
    own type map, orientations and weight factors, against the oracle
    composed as the reference does it (a pattern per type, then the
    weighted DFT with data index = element type;
    oskar_evaluate_station_beam_aperture_array.c:158-202)."""
    norm_el, norm_arr, norm_fin, swap, is_3d = flags
    cases = stations(real, is_3d=is_3d, num_el=200, num_dir=613)
    nst, n, nd = len(cases), 200, 613
    rng = np.random.default_rng(num_types)
    types = rng.integers(0, num_types, (nst, n)).astype(np.int32)
    lengths = np.array([1.5, 1.1, 2.0, 0.7][:num_types])
    kinds = tapers = taper_par = None
    if model == "isotropic+tapers":
        # type 1 isotropic; cosine taper on type 0, Gaussian on the rest
        kinds = np.array([0, 1, 0, 0][:num_types], np.int32)
        tapers = np.array([1, 2, 2, 0][:num_types], np.int32)
        taper_par = np.array([1.7, 1.2, 0.8, 0.0][:num_types])
    wf = rng.normal(1, 0.1, (nst, 2 * n)).astype(real)
    ori_x = rng.uniform(0, np.pi, (nst, num_types))
    ori_y = ori_x + np.pi / 2 + rng.normal(0, 0.05, (nst, num_types))
    cat = lambda key, i: dev(np.concatenate([c[key][i] for c in cases]))
    out = torch.zeros(nst * nd * 8, dtype=torch.float64 if real ==
                      np.float64 else torch.float32, device="cuda")
    ob.call("oskb_station_beam_aa_types_" + suffix(real), nst, n,
            *[cat("el", i) for i in range(3)],
            *[cat("meas", i) for i in range(3)],
            dev(np.concatenate([c["cable"] for c in cases])), dev(wf),
            num_types, dev(types), lengths, kinds, tapers, taper_par,
            dev(ori_x), dev(ori_y), norm_el,
            norm_arr, norm_fin, swap, is_3d, cases[0]["freq"],
            dev(np.stack([c["b"] for c in cases])),
            dev(np.stack([c["norm"] for c in cases])), nd,
            *[dev(cases[0]["dirs"][i]) for i in range(3)], 0, out,
            ob.stream_ptr())
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(nst, -1)
    for s, c in enumerate(cases):
        ref = np.zeros(8 * nd, real)
        oracle().call("station_beam_aa_types_" + suffix(real), np.float64,
                      n, 1, *c["el"], *c["meas"], c["cable"], wf[s].copy(),
                      num_types, types[s].copy(), lengths, kinds, tapers,
                      taper_par, ori_x[s].copy(), ori_y[s].copy(), norm_el,
                      norm_arr,
                      norm_fin, swap, 0, is_3d, c["freq"],
                      *c["b"], *c["norm"], nd, *cases[0]["dirs"], ref)
        assert rel(got[s], ref) <= TOL[real], (s, rel(got[s], ref))


def test_station_beam_element_types_limits():
    c = beam_case(np.float64, num_el=8, num_dir=5)
    args = lambda nt, lengths: (
        1, 8, *[dev(a) for a in c["el"]], None, None, None, None, None, nt,
        None, lengths, None, None, None, dev(np.array([0.0])),
        dev(np.array([1.5])), 0, 0, 0,
        0, 1, 100e6, dev(c["b"]), dev(c["norm"]), 5,
        *[dev(a) for a in c["dirs"]], 0,
        torch.zeros(40, dtype=torch.float64, device="cuda"), None)
    five = np.ones(5)
    assert ob.call("oskb_station_beam_aa_types_d", *args(5, five),
                   check=False) == -5  # OSKB_ERR_OUT_OF_RANGE
    assert ob.call("oskb_station_beam_aa_types_d", *args(0, five),
                   check=False) == -3
    assert ob.call("oskb_station_beam_aa_types_d", *args(1, None),
                   check=False) == -3
    # a Gaussian taper needs a positive FWHM; kinds and tapers in range
    bad = list(args(1, np.ones(1)))
    bad[13], bad[14], bad[15] = None, np.array([2], np.int32), np.zeros(1)
    assert ob.call("oskb_station_beam_aa_types_d", *bad, check=False) == -3
    bad[13], bad[14] = np.array([2], np.int32), None
    assert ob.call("oskb_station_beam_aa_types_d", *bad, check=False) == -3


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("num_types", [1, 2])
@pytest.mark.parametrize("flags", [(1, 1, 1, 0, 1), (0, 1, 0, 1, 0),
                                   (1, 0, 1, 1, 0)])
def test_station_beam_two_feeds(real, num_types, flags):
    """Stations whose y feed has its own element positions (true and
    measured), cable errors and weight factors: the x feed's array factor
    forms the (xx, xy) row, the y feed's the (yx, yy) row, and the final
    normalisation uses both (oskar_evaluate_station_beam_aperture_array.c:
    208-223), against the oracle's per-feed DFT with eval_x / eval_y. One
    station points below the horizon."""
    norm_el, norm_arr, norm_fin, swap, is_3d = flags
    cases = stations(real, is_3d=is_3d, num_el=150, num_dir=517)
    cases[1]["b"] = np.array([0.3, 0.2, -np.sqrt(1 - 0.13)])
    nst, n, nd = len(cases), 150, 517
    rng = np.random.default_rng(9 + num_types)
    types = rng.integers(0, num_types, (nst, n)).astype(np.int32)
    lengths = np.array([1.5, 1.1][:num_types])
    ori_x = rng.uniform(0, np.pi, (nst, num_types))
    ori_y = ori_x + np.pi / 2
    kinds = tapers = taper_par = None
    # feed y: positions moved by up to 5 cm, its own cable errors, factors
    feeds = []
    for c in cases:
        dxy = [rng.normal(0, 0.05, n).astype(real) for _ in range(3)]
        if not is_3d:
            dxy[2][:] = 0
        fy = dict(el=[c["el"][i] + dxy[i] for i in range(3)],
                  meas=[c["meas"][i] + dxy[i] for i in range(3)],
                  cable=rng.normal(0, 0.02, n).astype(real))
        feeds.append((c, fy))
    wf = rng.normal(1, 0.1, (2, nst, 2 * n)).astype(real)
    stack = lambda key, i: dev(np.concatenate(
        [c[key][i] for c, _ in feeds] + [fy[key][i] for _, fy in feeds]))
    cable = dev(np.concatenate([c["cable"] for c, _ in feeds] +
                               [fy["cable"] for _, fy in feeds]))
    out = torch.zeros(nst * nd * 8, dtype=torch.float64 if real ==
                      np.float64 else torch.float32, device="cuda")
    ob.call("oskb_station_beam_aa_feeds_" + suffix(real), 2, nst, n,
            *[stack("el", i) for i in range(3)],
            *[stack("meas", i) for i in range(3)], cable, dev(wf),
            num_types, dev(types), lengths, kinds, tapers, taper_par,
            dev(ori_x), dev(ori_y), norm_el,
            norm_arr, norm_fin, swap, is_3d, cases[0]["freq"],
            dev(np.stack([c["b"] for c in cases])),
            dev(np.stack([c["norm"] for c in cases])), nd,
            *[dev(cases[0]["dirs"][i]) for i in range(3)], 0, out,
            ob.stream_ptr())
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(nst, -1)
    assert not got[1].any()
    for s, (c, fy) in enumerate(feeds):
        if s == 1:
            continue
        ref = np.zeros(8 * nd, real)
        cat2 = lambda a, b: np.ascontiguousarray(np.concatenate([a, b]))
        oracle().call("station_beam_aa_types_" + suffix(real), np.float64,
                      n, 2, *[cat2(c["el"][i], fy["el"][i]) for i in range(3)],
                      *[cat2(c["meas"][i], fy["meas"][i]) for i in range(3)],
                      cat2(c["cable"], fy["cable"]),
                      cat2(wf[0, s], wf[1, s]), num_types, types[s].copy(),
                      lengths, None, None, None, ori_x[s].copy(),
                      ori_y[s].copy(), norm_el,
                      norm_arr, norm_fin, swap, 0, is_3d, c["freq"], *c["b"],
                      *c["norm"], nd, *cases[0]["dirs"], ref)
        assert rel(got[s], ref) <= TOL[real], (s, rel(got[s], ref))


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("num_types", [1, 3])
@pytest.mark.parametrize("flags", [(1, 1, 1, 0, 1), (0, 0, 1, 1, 0),
                                   (1, 1, 0, 0, 0)])
def test_station_beam_scalar(real, num_types, flags):
    """The scalar (Stokes-I) mode: each type's pattern amplitude times its
    array factor, complex beam, normalised by its magnitude in the
    normalisation direction; three stations, one pointing below the
    horizon, dipole and isotropic types with tapers."""
    norm_el, norm_arr, norm_fin, swap, is_3d = flags
    cases = stations(real, is_3d=is_3d, num_el=180, num_dir=401)
    cases[2]["b"] = np.array([0.1, 0.2, -np.sqrt(1 - 0.05)])
    nst, n, nd = len(cases), 180, 401
    rng = np.random.default_rng(31 + num_types)
    types = rng.integers(0, num_types, (nst, n)).astype(np.int32)
    lengths = np.array([1.5, 1.0, 2.1][:num_types])
    kinds = np.array([0, 1, 0][:num_types], np.int32)
    tapers = np.array([0, 1, 2][:num_types], np.int32)
    taper_par = np.array([0.0, 2.0, 1.0][:num_types])
    ori_x = rng.uniform(0, np.pi, (nst, num_types))
    ori_y = ori_x + np.pi / 2
    wf = rng.normal(1, 0.1, (nst, 2 * n)).astype(real)
    cat = lambda key, i: dev(np.concatenate([c[key][i] for c in cases]))
    out = torch.zeros(nst * nd * 2, dtype=torch.float64 if real ==
                      np.float64 else torch.float32, device="cuda")
    ob.call("oskb_station_beam_aa_scalar_" + suffix(real), nst, n,
            *[cat("el", i) for i in range(3)],
            *[cat("meas", i) for i in range(3)],
            dev(np.concatenate([c["cable"] for c in cases])), dev(wf),
            num_types, dev(types), lengths, kinds, tapers, taper_par,
            dev(ori_x), dev(ori_y), norm_el, norm_arr, norm_fin, swap, is_3d,
            cases[0]["freq"], dev(np.stack([c["b"] for c in cases])),
            dev(np.stack([c["norm"] for c in cases])), nd,
            *[dev(cases[0]["dirs"][i]) for i in range(3)], 0, out,
            ob.stream_ptr())
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(nst, -1)
    assert not got[2].any()
    for s, c in enumerate(cases[:2]):
        ref = np.zeros(8 * nd, real)
        oracle().call("station_beam_aa_types_" + suffix(real), np.float64,
                      n, 1, *c["el"], *c["meas"], c["cable"], wf[s].copy(),
                      num_types, types[s].copy(), lengths, kinds, tapers,
                      taper_par, ori_x[s].copy(), ori_y[s].copy(), norm_el,
                      norm_arr, norm_fin, swap, 1, is_3d, c["freq"], *c["b"],
                      *c["norm"], nd, *cases[0]["dirs"], ref)
        assert rel(got[s], ref[:2 * nd]) <= TOL[real], (s, rel(got[s],
                                                               ref[:2 * nd]))
