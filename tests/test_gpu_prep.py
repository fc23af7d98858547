"""Device sky and baseline preparation against the oracle: direction
conversions, the multi-station horizon mask and compaction (the horizon
clip), and station -> baseline (u, v, w)."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(),
                                 reason="needs a CUDA device")]

import oskar_b200 as ob  # noqa: E402
from oracle_lib import oracle, suffix  # noqa: E402

TOL = {np.float64: 1e-14, np.float32: 2e-6}


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def close(a, b, real):
    return np.max(np.abs(a - b)) <= TOL[real] * max(1.0, np.max(np.abs(b)))


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_lon_lat_and_ra_dec_conversions(real):
    rng = np.random.default_rng(1)
    n, nst = 3001, 5
    lon = rng.uniform(0, 2 * np.pi, n).astype(real)
    lat = rng.uniform(-1.5, 1.5, n).astype(real)
    s = suffix(real)
    tt = torch.float64 if real == np.float64 else torch.float32
    l, m, nn = (torch.zeros(n, dtype=tt, device="cuda") for _ in range(3))
    ob.call("oskb_convert_lon_lat_to_relative_directions_" + s, n, dev(lon),
            dev(lat), 0.3, -0.5, l, m, nn, ob.stream_ptr())
    ref = [np.zeros(n, real) for _ in range(3)]
    oracle().call("lon_lat_to_relative_directions_" + s, real, n, lon, lat,
                  real(0.3), real(np.cos(-0.5)), real(np.sin(-0.5)), *ref)
    for g, r in zip((l, m, nn), ref):
        assert close(host(g), r, real)
    lst = rng.uniform(0, 2 * np.pi, nst)
    slat = rng.uniform(-1, 1, nst)
    xyz = [torch.zeros(nst * n, dtype=tt, device="cuda") for _ in range(3)]
    ob.call("oskb_convert_ra_dec_to_enu_directions_" + s, n, dev(lon),
            dev(lat), nst, dev(lst), dev(slat), *xyz, ob.stream_ptr())
    got = [host(a).reshape(nst, n) for a in xyz]
    for st in range(nst):
        r = [np.zeros(n, real) for _ in range(3)]
        oracle().call("ra_dec_to_enu_directions_" + s, real, n, lon, lat,
                      real(lst[st]), real(np.sin(slat[st])),
                      real(np.cos(slat[st])), 0, *r)
        for g, rr in zip(got, r):
            assert close(g[st], rr, real)


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_horizon_clip(real):
    """Mask over all stations, then an order-preserving compaction of the
    sky columns, against the oracle's mask and numpy's compaction."""
    rng = np.random.default_rng(2)
    n, nst = 70001, 7
    l, m = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    nn = rng.uniform(-1, 1, n)
    ha0, lat = rng.uniform(-3, 3, nst), rng.uniform(-1.2, 1.2, nst)
    dec0 = -0.4
    cols = [np.ascontiguousarray(a, real) for a in (l, m, nn)]
    s = suffix(real)
    mask = torch.zeros(n, dtype=torch.int32, device="cuda")
    ob.call("oskb_sky_horizon_mask_" + s, n, *[dev(a) for a in cols], nst,
            ha0, lat, dec0, mask, ob.stream_ptr())
    ref_mask = np.zeros(n, np.int32)
    for st in range(nst):
        ch, sd, cd = np.cos(ha0[st]), np.sin(dec0), np.cos(dec0)
        sl, cl = np.sin(lat[st]), np.cos(lat[st])
        oracle().call("update_horizon_mask_" + s, real, n, *cols,
                      real(cl * np.sin(ha0[st])), real(sl * cd - cl * ch * sd),
                      real(sl * sd + cl * ch * cd), ref_mask)
    got_mask = host(mask)
    # Equal except where a station sees the source within rounding of its
    # horizon (fused multiply-add on the GPU, separate operations in C).
    diff = np.nonzero(got_mask != ref_mask)[0]
    if diff.size:
        near = np.zeros(n, bool)
        for st in range(nst):
            ch, sd, cd = np.cos(ha0[st]), np.sin(dec0), np.cos(dec0)
            sl, cl = np.sin(lat[st]), np.cos(lat[st])
            d = l * cl * np.sin(ha0[st]) + m * (sl * cd - cl * ch * sd) + \
                nn * (sl * sd + cl * ch * cd)
            near |= np.abs(d) < 1e-5
        assert near[diff].all() and diff.size < 10
    assert 0 < ref_mask.sum() < n
    ins = [dev(a) for a in cols]
    outs = [torch.zeros_like(a) for a in ins]
    in_arr = (ctypes.c_void_p * 3)(*[a.data_ptr() for a in ins])
    out_arr = (ctypes.c_void_p * 3)(*[a.data_ptr() for a in outs])
    num = ctypes.c_int(-1)
    ob.call("oskb_sky_compact_" + s, n, mask, 3, ctypes.addressof(in_arr),
            ctypes.addressof(out_arr), ctypes.addressof(num),
            ob.stream_ptr())
    keep = got_mask != 0
    assert num.value == keep.sum()
    for o, c in zip(outs, cols):
        assert np.array_equal(host(o)[:num.value], c[keep])


@pytest.mark.parametrize("real", [np.float64, np.float32])
@pytest.mark.parametrize("casa", [0, 1])
def test_baseline_uvw(real, casa):
    rng = np.random.default_rng(3)
    nst = 300
    uvw = [rng.uniform(-1e4, 1e4, nst + 2).astype(real) for _ in range(3)]
    nbl = nst * (nst - 1) // 2
    s = suffix(real)
    tt = torch.float64 if real == np.float64 else torch.float32
    out = [torch.zeros(nbl + 4, dtype=tt, device="cuda") for _ in range(3)]
    ob.call("oskb_convert_station_uvw_to_baseline_uvw_" + s, casa, nst, 2,
            *[dev(a) for a in uvw], 4, *out, ob.stream_ptr())
    ref = [np.zeros(nbl + 4, real) for _ in range(3)]
    oracle().call("station_uvw_to_baseline_uvw_" + s, real, casa, nst, 2,
                  *uvw, 4, *ref)
    for g, r in zip(out, ref):
        assert np.array_equal(host(g), r)
