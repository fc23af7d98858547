"""Seeded synthetic telescope and sky configurations.

No public dataset is involved: these generators stand in for OSKAR telescope
models and sky models with the shapes and value distributions of the
benchmark configurations:

  c1: 30 isotropic stations uniform in a 1 km disc, lat -27 deg, 1 channel at
      100 MHz, 10 dumps of 60 s, phase centre RA 0, Dec -30 deg; 1,000 point
      sources uniform in a 5 deg radius, Stokes I ~ S^-1.5 on [0.01, 10] Jy,
      Q = U = V = 0; no smearing.
  c3: 512 stations log-radial (50 m to 65 km); 100,000 point sources in a
      20 deg field (10 deg radius), I ~ S^-1.5 on [0.01, 10] Jy,
      |Q|, |U|, |V| <= 0.1 I (uniform); per station-source 2x2 Jones
      E = I + complex N(0, 0.1) (real and imaginary parts each N(0, 0.1)),
      fixed over time and channel; 16 channels 100-115 MHz (1 MHz apart),
      64 dumps of 10 s from MJD 51544.5; no smearing.
"""
import math

import numpy as np

C0 = 299792458.0
LAT_DEG, LON_DEG = -27.0, 116.76
RA0_DEG, DEC0_DEG = 0.0, -30.0
MJD0 = 51544.5


def gast_rad(mjd_utc):
    """Greenwich sidereal angle from the linear GMST expression (the
    constants of the IAU 1982 model's leading terms); adequate for
    synthetic inputs, which only need internal consistency."""
    d = mjd_utc - 51544.5
    gmst_deg = 280.46061837 + 360.98564736629 * d
    return math.radians(gmst_deg % 360.0)


def enu_to_ecef_offsets(e, n, u, lat_rad, lon_rad):
    """Rotates local horizon (east, north, up) offsets to ECEF offsets."""
    sl, cl = math.sin(lat_rad), math.cos(lat_rad)
    so, co = math.sin(lon_rad), math.cos(lon_rad)
    x = -so * e - sl * co * n + cl * co * u
    y = co * e - sl * so * n + cl * so * u
    z = cl * n + sl * u
    return x, y, z


def power_law_flux(rng, n, smin=0.01, smax=10.0, index=-1.5):
    """Inverse-CDF samples of p(S) ~ S^index on [smin, smax]."""
    a = index + 1.0
    u = rng.uniform(0.0, 1.0, n)
    return (smin ** a + u * (smax ** a - smin ** a)) ** (1.0 / a)


def disc_lmn(rng, n, radius_deg):
    r = np.sqrt(rng.uniform(0, 1, n)) * math.sin(math.radians(radius_deg))
    th = rng.uniform(0, 2 * math.pi, n)
    l, m = r * np.cos(th), r * np.sin(th)
    return l, m, np.sqrt(1.0 - l * l - m * m)


class Config:
    """Host-side description of one configuration (FP64 numpy arrays)."""

    def __init__(self, name, num_st, num_src, freqs_hz, num_times, dt_sec,
                 station_enu, l, m, n, I, Q, U, V, seed):
        self.name = name
        self.num_st, self.num_src = num_st, num_src
        self.freqs_hz = np.asarray(freqs_hz, np.float64)
        self.num_times, self.dt_sec = num_times, dt_sec
        self.station_enu = station_enu
        self.l, self.m, self.n = l, m, n
        self.I, self.Q, self.U, self.V = I, Q, U, V
        self.seed = seed
        lat, lon = math.radians(LAT_DEG), math.radians(LON_DEG)
        self.ecef = np.stack(enu_to_ecef_offsets(
            station_enu[0], station_enu[1], station_enu[2], lat, lon))
        self.ra0, self.dec0 = math.radians(RA0_DEG), math.radians(DEC0_DEG)

    @property
    def num_baselines(self):
        return self.num_st * (self.num_st - 1) // 2

    def gast(self, t):
        mjd = MJD0 + (t + 0.5) * self.dt_sec / 86400.0
        return gast_rad(mjd)

    def station_uvw(self, t):
        """FP64 station (u, v, w) metres at dump t (the reference evaluates
        at the dump mid-point, oskar/telescope/src/oskar_telescope_uvw.c)."""
        ha = self.gast(t) - self.ra0
        sh, ch = math.sin(ha), math.cos(ha)
        sd, cd = math.sin(self.dec0), math.cos(self.dec0)
        x, y, z = self.ecef
        tt = x * ch - y * sh
        return np.stack([x * sh + y * ch, z * cd - tt * sd, z * sd + tt * cd])

    def source_baselines(self):
        return (self.num_baselines * self.num_src * len(self.freqs_hz)
                * self.num_times)


def c1():
    rng = np.random.default_rng(1)
    num_st, num_src = 30, 1000
    r = 500.0 * np.sqrt(rng.uniform(0, 1, num_st))
    th = rng.uniform(0, 2 * math.pi, num_st)
    enu = np.stack([r * np.cos(th), r * np.sin(th), np.zeros(num_st)])
    l, m, n = disc_lmn(rng, num_src, 5.0)
    I = power_law_flux(rng, num_src)
    z = np.zeros(num_src)
    return Config("c1", num_st, num_src, [100e6], 10, 60.0, enu, l, m, n, I,
                  z, z.copy(), z.copy(), 1)


def c3(num_src=100_000, num_st=512, num_channels=16, num_times=64):
    rng = np.random.default_rng(3)
    r = np.exp(rng.uniform(math.log(50.0), math.log(65e3), num_st))
    th = rng.uniform(0, 2 * math.pi, num_st)
    enu = np.stack([r * np.cos(th), r * np.sin(th), np.zeros(num_st)])
    l, m, n = disc_lmn(rng, num_src, 10.0)
    I = power_law_flux(rng, num_src)
    Q, U, V = (I * rng.uniform(-0.1, 0.1, num_src) for _ in range(3))
    freqs = 100e6 + 1e6 * np.arange(num_channels)
    return Config("c3", num_st, num_src, freqs, num_times, 10.0, enu, l, m,
                  n, I, Q, U, V, 3)


def jones_e_device(cfg, dtype, device="cuda"):
    """E = I + complex N(0, 0.1) per station-source, generated on the device
    with a seeded torch generator: [num_st][num_src][8] reals."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(cfg.seed)
    e = torch.randn((cfg.num_st, cfg.num_src, 8), generator=g,
                    device=device, dtype=torch.float32)
    e.mul_(0.1)
    e[..., 0] += 1.0
    e[..., 6] += 1.0
    return e.to(dtype)


def jones_e_host(cfg, rng_seed=None):
    """Host (numpy, FP64) version of E for small configurations."""
    rng = np.random.default_rng(cfg.seed if rng_seed is None else rng_seed)
    e = rng.normal(0, 0.1, (cfg.num_st, cfg.num_src, 8))
    e[..., 0] += 1.0
    e[..., 6] += 1.0
    return e


def c2(num_st=128, num_el=256, num_field=10_000, num_off=2_000,
       num_channels=4, num_times=32):
    """Aperture-array stations with beams: num_st stations log-radial from
    50 m to 40 km, each with num_el dipoles uniform in a 38 m disc (its own
    layout); num_field sources in a 10 degree field plus num_off at random
    directions (above the horizon at the first dump); I power law, Q and U
    N(0, 0.05 I) on 10 % of sources; 4 channels over 100-130 MHz, 32 dumps
    of 60 s from MJD 51544.5; array at latitude -27 deg, longitude
    116.76 deg; phase centre RA 0, Dec -30 deg. Returned as a dict of FP64
    numpy arrays."""
    rng = np.random.default_rng(2)
    lat0, lon0 = math.radians(-27.0), math.radians(116.76)
    ra0, dec0 = 0.0, math.radians(-30.0)
    r = np.exp(rng.uniform(math.log(50.0), math.log(40e3), num_st))
    th = rng.uniform(0, 2 * math.pi, num_st)
    e_off, n_off = r * np.cos(th), r * np.sin(th)
    ecef = np.stack(enu_to_ecef_offsets(e_off, n_off, np.zeros(num_st),
                                        lat0, lon0))
    lat = lat0 + n_off / 6.371e6
    lon = lon0 + e_off / (6.371e6 * math.cos(lat0))
    rr = 19.0 * np.sqrt(rng.uniform(0, 1, (num_st, num_el)))
    tt = rng.uniform(0, 2 * math.pi, (num_st, num_el))
    el_x, el_y = rr * np.cos(tt), rr * np.sin(tt)
    orient = np.zeros(num_st)
    l, m, n = disc_lmn(rng, num_field, 10.0)
    # field sources: (l, m) about the phase centre -> RA, Dec
    dec_f = np.arcsin(m * math.cos(dec0) + n * math.sin(dec0))
    ra_f = ra0 + np.arctan2(l, n * math.cos(dec0) - m * math.sin(dec0))
    mjd0 = 51544.5
    gast0 = gast_rad(mjd0 + 30.0 / 86400.0)
    # off-field sources above the horizon at the array centre, first dump
    ra_o, dec_o = [], []
    while len(ra_o) < num_off:
        ra_c = rng.uniform(0, 2 * math.pi)
        dec_c = math.asin(rng.uniform(-1, 1))
        ha = gast0 + lon0 - ra_c
        el_s = (math.sin(lat0) * math.sin(dec_c) +
                math.cos(lat0) * math.cos(dec_c) * math.cos(ha))
        if el_s > 0.05:
            ra_o.append(ra_c)
            dec_o.append(dec_c)
    ra = np.concatenate([ra_f, np.array(ra_o)])
    dec = np.concatenate([dec_f, np.array(dec_o)])
    dra = ra - ra0
    l = np.cos(dec) * np.sin(dra)
    m = math.cos(dec0) * np.sin(dec) - math.sin(dec0) * np.cos(dec) * \
        np.cos(dra)
    n = math.sin(dec0) * np.sin(dec) + math.cos(dec0) * np.cos(dec) * \
        np.cos(dra)
    ns = num_field + num_off
    I = power_law_flux(rng, ns)
    pol = rng.uniform(0, 1, ns) < 0.1
    Q = np.where(pol, rng.normal(0, 0.05, ns) * I, 0.0)
    U = np.where(pol, rng.normal(0, 0.05, ns) * I, 0.0)
    V = np.zeros(ns)
    freqs = np.linspace(100e6, 130e6, num_channels)
    gast = np.array([gast_rad(mjd0 + (t + 0.5) * 60.0 / 86400.0)
                     for t in range(num_times)])
    return dict(num_st=num_st, num_el=num_el, num_src=ns, lat=lat, lon=lon,
                ecef=ecef, el_x=el_x, el_y=el_y, orient=orient, ra=ra,
                dec=dec, l=l, m=m, n=n, I=I, Q=Q, U=U, V=V, freqs=freqs,
                gast=gast, ra0=ra0, dec0=dec0, num_times=num_times)
