"""End to end on the GPU, the aperture-array chain of the reference's
sim_baselines (oskar/interferometer/src/oskar_interferometer_run_block.c:
245-334) on a small seeded configuration of the 256-dipole-station kind:
station beam E per station -> parallactic rotation R -> join E R -> Jones K
-> join K (E R) -> cross-correlation, for two dumps and two channels, every
step through the C ABI, against the oracle running the same chain.
Directions (source RA/Dec to each station's ENU frame) are prepared on the
host for both sides. Tolerances: FP64 1e-12; FP32 1e-4 (single-precision
phases of the K and beam steps, as in the reference's FP32 path)."""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(),
                                 reason="needs a CUDA device")]

import oskar_b200 as ob  # noqa: E402
from oracle_lib import oracle, suffix  # noqa: E402

C0 = 299792458.0


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def enu_dirs(ra, dec, lat, lst):
    ha = lst - ra
    x = -np.cos(dec) * np.sin(ha)
    y = math.cos(lat) * np.sin(dec) - math.sin(lat) * np.cos(dec) * np.cos(ha)
    z = math.sin(lat) * np.sin(dec) + math.cos(lat) * np.cos(dec) * np.cos(ha)
    return x, y, z


def make_config(seed=2, num_st=8, num_el=64, num_src=300):
    rng = np.random.default_rng(seed)
    lat0, lon0 = math.radians(-27.0), math.radians(116.76)
    ra0, dec0 = 0.0, math.radians(-30.0)
    r = np.exp(rng.uniform(math.log(50.0), math.log(4e3), num_st))
    th = rng.uniform(0, 2 * math.pi, num_st)
    e_off, n_off = r * np.cos(th), r * np.sin(th)
    lat = lat0 + n_off / 6.371e6
    lon = lon0 + e_off / (6.371e6 * math.cos(lat0))
    # ECEF offsets for uvw (relative to the array centre)
    sl, cl, so, co = (math.sin(lat0), math.cos(lat0), math.sin(lon0),
                      math.cos(lon0))
    ecef = np.stack([-so * e_off - sl * co * n_off, co * e_off - sl * so *
                     n_off, cl * n_off])
    # elements: 64 dipoles in a 38 m disc per station, rotated per station
    rr = 19.0 * np.sqrt(rng.uniform(0, 1, (num_st, num_el)))
    tt = rng.uniform(0, 2 * math.pi, (num_st, num_el))
    el = np.stack([rr * np.cos(tt), rr * np.sin(tt),
                   np.zeros((num_st, num_el))])
    orient = rng.uniform(0, math.pi, num_st)
    # sky: 2/3 in a 10 degree field, 1/3 anywhere above the horizon later
    nf = 2 * num_src // 3
    rad = np.sqrt(rng.uniform(0, 1, nf)) * math.radians(10)
    pa = rng.uniform(0, 2 * math.pi, nf)
    dec_f = dec0 + rad * np.cos(pa)
    ra_f = ra0 + rad * np.sin(pa) / np.cos(dec_f)
    ra_o = rng.uniform(0, 2 * math.pi, num_src - nf)
    dec_o = np.arcsin(rng.uniform(-1, 0.3, num_src - nf))
    ra, dec = np.concatenate([ra_f, ra_o]), np.concatenate([dec_f, dec_o])
    I = 10 ** rng.uniform(-2, 1, num_src)
    Q = np.where(rng.uniform(size=num_src) < 0.1,
                 rng.normal(0, 0.05, num_src) * I, 0.0)
    U = np.where(rng.uniform(size=num_src) < 0.1,
                 rng.normal(0, 0.05, num_src) * I, 0.0)
    V = np.zeros(num_src)
    dra = ra - ra0
    l = np.cos(dec) * np.sin(dra)
    m = math.cos(dec0) * np.sin(dec) - math.sin(dec0) * np.cos(dec) * \
        np.cos(dra)
    n = math.sin(dec0) * np.sin(dec) + math.cos(dec0) * np.cos(dec) * \
        np.cos(dra)
    return dict(lat=lat, lon=lon, ecef=ecef, el=el, orient=orient, ra=ra,
                dec=dec, I=I, Q=Q, U=U, V=V, l=l, m=m, n=n, ra0=ra0,
                dec0=dec0, freqs=[100e6, 130e6], gast=[4.2, 4.45])


def run_chain(cfg, real, on_gpu):
    orc = oracle()
    s = suffix(real)
    N, S = cfg["lat"].size, cfg["I"].size
    num_el = cfg["el"].shape[2]
    T, C = len(cfg["gast"]), len(cfg["freqs"])
    nbl = N * (N - 1) // 2
    cast = lambda a: np.ascontiguousarray(a, dtype=real)
    sky = {k: cast(cfg[k]) for k in ("I", "Q", "U", "V", "l", "m", "n",
                                     "ra", "dec")}
    el = [cast(cfg["el"][i]) for i in range(3)]
    flags = (0, 1, 1, 0, 0)  # element, array, final normalisation, swap, 3-D
    vis = np.zeros(T * C * nbl * 8, real)
    if on_gpu:
        d = {k: dev(v) for k, v in sky.items()}
        d_el = [dev(a) for a in el]
        d_orx = dev(cfg["orient"])
        d_ory = dev(cfg["orient"] + math.pi / 2)
        d_lat = dev(cfg["lat"])
        tt = torch.float64 if real == np.float64 else torch.float32
        d_vis = torch.zeros(vis.size, dtype=tt, device="cuda")
        E = torch.empty(N * S * 8, dtype=tt, device="cuda")
        R = torch.empty_like(E)
        K = torch.empty(N * S * 2, dtype=tt, device="cuda")
        st = ob.stream_ptr()
    for t in range(T):
        gast = cfg["gast"][t]
        lst = gast + cfg["lon"]
        dirs = np.zeros((3, N, S))
        beam = np.zeros((N, 3))
        for p in range(N):
            dirs[:, p] = enu_dirs(cfg["ra"], cfg["dec"], cfg["lat"][p],
                                  lst[p])
            beam[p] = [a[0] for a in enu_dirs(
                np.array([cfg["ra0"]]), np.array([cfg["dec0"]]),
                cfg["lat"][p], lst[p])]
        uvw = [np.zeros(N) for _ in range(3)]
        ha0 = gast - cfg["ra0"]
        orc.call("ecef_to_station_uvw_d", np.float64, N, *[
            np.ascontiguousarray(a) for a in cfg["ecef"]], math.sin(ha0),
            math.cos(ha0), math.sin(cfg["dec0"]), math.cos(cfg["dec0"]), 0,
            0, *uvw)
        uvw = [cast(a) for a in uvw]
        for c, f in enumerate(cfg["freqs"]):
            k = 2 * math.pi * f / C0
            off = (t * C + c) * nbl
            if on_gpu:
                ddir = [dev(cast(dirs[i])) for i in range(3)]
                ob.call("oskb_station_beam_aa_" + s, N, num_el, *d_el, None,
                        None, None, None, d_orx, d_ory, 1.5, *flags, f,
                        dev(beam), dev(beam), S, *ddir, 1, E, st)
                ob.call("oskb_evaluate_jones_R_" + s, S, d["ra"], d["dec"],
                        N, d_lat, dev(lst), R, st)
                ob.call("oskb_mem_multiply_" + s, 5, 0, 0, 0, N * S, E, R,
                        R, st)
                du = [dev(a) for a in uvw]
                ob.call("oskb_evaluate_jones_K_" + s, S, d["l"], d["m"],
                        d["n"], N, *du, k, d["I"], 0.0, 1e30, 0, K, st)
                ob.call("oskb_mem_multiply_" + s, 3, 0, 0, 0, N * S, K, R,
                        E, st)
                ob.call("oskb_cross_correlate_" + s, 0, 0, S, N, off, E,
                        d["I"], d["Q"], d["U"], d["V"], d["l"], d["m"],
                        d["n"], None, None, None, *du, None, None, 0.0,
                        3e38, f / C0, 0.0, 0.0, 0.0, 0.0, d_vis, st)
            else:
                E = np.zeros((N, S * 8), real)
                R = np.zeros((N, S * 8), real)
                for p in range(N):
                    orc.call("station_beam_aa_" + s, np.float64, num_el,
                             cast(el[0][p]), cast(el[1][p]), cast(el[2][p]),
                             None, None, None, np.zeros(num_el, real),
                             float(cfg["orient"][p]),
                             float(cfg["orient"][p] + math.pi / 2), 1.5,
                             *flags, f, *beam[p], *beam[p], S,
                             cast(dirs[0, p]), cast(dirs[1, p]),
                             cast(dirs[2, p]), E[p])
                    Rp = np.zeros(S * 8, real)
                    orc.call("jones_r_" + s, real, S, sky["ra"], sky["dec"],
                             real(math.cos(cfg["lat"][p])),
                             real(math.sin(cfg["lat"][p])), real(lst[p]), 0,
                             Rp)
                    R[p] = Rp
                ER = np.zeros(N * S * 8, real)
                orc.call("mem_mul_mm_m_" + s, real, N * S, E.ravel(),
                         R.ravel(), ER)
                Kh = np.zeros(N * S * 2, real)
                orc.call("jones_k_" + s, real, S, sky["l"], sky["m"],
                         sky["n"], N, *uvw, real(k), sky["I"], real(0),
                         real(1e30), 0, Kh)
                J = np.zeros(N * S * 8, real)
                orc.call("mem_mul_cm_m_" + s, real, N * S, Kh, ER, J)
                z = np.zeros(N, real)
                orc.call("xcorr_matrix_" + s, real, 0, 0, S, N, off, J,
                         sky["I"], sky["Q"], sky["U"], sky["V"], sky["l"],
                         sky["m"], sky["n"], None, None, None, *uvw, z, z,
                         real(0), real(3e38), real(f / C0), real(0),
                         real(0), real(0), real(0), vis)
    if on_gpu:
        torch.cuda.synchronize()
        return d_vis.cpu().numpy()
    return vis


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_aperture_array_chain(real):
    cfg = make_config()
    got = run_chain(cfg, real, True)
    ref = run_chain(cfg, real, False)
    got64, ref64 = got.astype(np.float64), ref.astype(np.float64)
    err = max(np.max(np.abs(got64 - ref64)) / np.max(np.abs(ref64)),
              np.linalg.norm(got64 - ref64) / np.linalg.norm(ref64))
    assert err <= (1e-12 if real == np.float64 else 1e-4), err
    assert np.count_nonzero(ref) > 0.9 * ref.size
