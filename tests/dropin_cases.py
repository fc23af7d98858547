"""Simulation cases for the drop-in oskar_interferometer_run_block tests,
written as the inputs of tests/ref_sim.py (reference API calls)."""
import math

import numpy as np

from oskar_b200 import workloads


def lm_to_radec(l, m, ra0, dec0):
    """Sky directions of direction cosines (l, m) about (ra0, dec0) (the
    inverse orthographic projection)."""
    n = np.sqrt(1.0 - l * l - m * m)
    dec = np.arcsin(n * math.sin(dec0) + m * math.cos(dec0))
    ra = ra0 + np.arctan2(l, n * math.cos(dec0) - m * math.sin(dec0))
    return ra, dec


def c1_case(precision="double", **over):
    """C1: 30 isotropic stations in a 1 km disc at lat -27 deg, 1,000 point
    sources (S^-1.5 on [0.01, 10] Jy, Q = U = V = 0) in a 5 deg field about
    RA 0, Dec -30 deg, 1 channel at 100 MHz, 10 dumps of 60 s, full
    polarisation, no smearing."""
    cfg = workloads.c1()
    ra, dec = lm_to_radec(cfg.l, cfg.m, cfg.ra0, cfg.dec0)
    n = cfg.num_src
    z = [0.0] * n
    case = {
        "precision": precision, "pol_mode": "Full",
        "lon_deg": workloads.LON_DEG, "lat_deg": workloads.LAT_DEG,
        "station_x": cfg.station_enu[0].tolist(),
        "station_y": cfg.station_enu[1].tolist(),
        "station_type": "Isotropic beam",
        "channel_bandwidth_hz": 0.0, "time_average_sec": 0.0,
        "uv_filter": [0.0, -1.0, "Wavelengths"],
        "ra_rad": ra.tolist(), "dec_rad": dec.tolist(),
        "I": cfg.I.tolist(), "Q": list(z), "U": list(z), "V": list(z),
        "ref_freq_hz": list(z), "spectral_index": list(z),
        "rotation_measure": list(z), "major_rad": list(z),
        "minor_rad": list(z), "pa_rad": list(z),
        "phase_centre_ra_rad": cfg.ra0, "phase_centre_dec_rad": cfg.dec0,
        "freq_start_hz": 100e6, "freq_inc_hz": 0.0, "num_channels": 1,
        "mjd_start": workloads.MJD0, "inc_sec": 60.0, "num_times": 10,
        "num_devices": 1, "max_times_per_block": 10,
        "max_sources_per_chunk": 16384, "horizon_clip": 1,
        "correlation_type": "Cross-correlations", "casa": 0,
        "source_min_jy": -1e300, "source_max_jy": 1e300,
    }
    case.update(over)
    return case


def c1_extended_case(precision="double", **over):
    """C1 widened to every stage the drop-in runs: full-Stokes fluxes with a
    spectral index and rotation measure over 3 channels, 30 % Gaussian
    sources, bandwidth and time-average smearing, auto-correlations, a uv
    filter, 2 sky chunks, blocks of 4 dumps and 2 device threads."""
    c = c1_case(precision)
    rng = np.random.default_rng(11)
    n = len(c["I"])
    I = np.asarray(c["I"])
    c["Q"] = (I * rng.uniform(-0.1, 0.1, n)).tolist()
    c["U"] = (I * rng.uniform(-0.1, 0.1, n)).tolist()
    c["V"] = (I * rng.uniform(-0.1, 0.1, n)).tolist()
    c["ref_freq_hz"] = [100e6] * n
    c["spectral_index"] = rng.uniform(-1.0, 0.5, n).tolist()
    c["rotation_measure"] = rng.uniform(-5.0, 5.0, n).tolist()
    gauss = rng.uniform(0, 1, n) < 0.3
    arcsec = math.pi / 180.0 / 3600.0
    maj = np.where(gauss, rng.uniform(1, 60, n) * arcsec, 0.0)
    mnr = np.where(gauss, rng.uniform(0.3, 1.0, n) * maj, 0.0)
    c["major_rad"] = maj.tolist()
    c["minor_rad"] = mnr.tolist()
    c["pa_rad"] = np.where(gauss, rng.uniform(0, math.pi, n), 0.0).tolist()
    c.update({"num_channels": 3, "freq_inc_hz": 5e6,
              "channel_bandwidth_hz": 1e5, "time_average_sec": 10.0,
              "uv_filter": [1.0, 250.0, "Wavelengths"],
              "correlation_type": "Both", "max_sources_per_chunk": 600,
              "max_times_per_block": 4, "num_devices": 2})
    c.update(over)
    return c


def c2_small_case(precision="double", per_station=True, **over):
    """C2 scaled down: aperture-array stations (48 dipoles each at random
    positions in a 38 m disc; one layout per station, or one shared by all)
    placed log-radially out to 5 km, 400 point sources in a 10 deg field plus
    80 at random directions, 10 % of them with Stokes Q and U, 3 channels
    over 100-130 MHz, 4 dumps of 300 s, full polarisation. Sources below the
    horizon are blanked by the station beams, so the horizon clip does not
    change the result."""
    rng = np.random.default_rng(22)
    nst, nel, nsrc, noff = 12, 48, 400, 80
    r = np.exp(rng.uniform(math.log(50.0), math.log(5e3), nst))
    th = rng.uniform(0, 2 * math.pi, nst)

    def layout():
        rr = 19.0 * np.sqrt(rng.uniform(0, 1, nel))
        tt = rng.uniform(0, 2 * math.pi, nel)
        return (rr * np.cos(tt)).tolist(), (rr * np.sin(tt)).tolist()
    lays = [layout() for _ in range(nst if per_station else 1)]
    ra0, dec0 = 0.0, math.radians(-30.0)
    l, m, _ = workloads.disc_lmn(rng, nsrc, 10.0)
    ra, dec = lm_to_radec(l, m, ra0, dec0)
    ra = np.concatenate([ra, rng.uniform(0, 2 * math.pi, noff)])
    dec = np.concatenate([dec, np.arcsin(rng.uniform(-1, 1, noff))])
    n = nsrc + noff
    I = workloads.power_law_flux(rng, n)
    pol = rng.uniform(0, 1, n) < 0.1
    Q = np.where(pol, rng.normal(0, 0.05, n) * I, 0.0)
    U = np.where(pol, rng.normal(0, 0.05, n) * I, 0.0)
    z = [0.0] * n
    case = {
        "precision": precision, "pol_mode": "Full",
        "lon_deg": workloads.LON_DEG, "lat_deg": workloads.LAT_DEG,
        "station_x": (r * np.cos(th)).tolist(),
        "station_y": (r * np.sin(th)).tolist(),
        "station_type": "Aperture array",
        "station_per_folder": 1 if per_station else 0,
        "element_x": [a for a, _ in lays] if per_station else lays[0][0],
        "element_y": [b for _, b in lays] if per_station else lays[0][1],
        "channel_bandwidth_hz": 0.0, "time_average_sec": 0.0,
        "uv_filter": [0.0, -1.0, "Wavelengths"],
        "ra_rad": ra.tolist(), "dec_rad": dec.tolist(),
        "I": I.tolist(), "Q": Q.tolist(), "U": U.tolist(), "V": list(z),
        "ref_freq_hz": list(z), "spectral_index": list(z),
        "rotation_measure": list(z), "major_rad": list(z),
        "minor_rad": list(z), "pa_rad": list(z),
        "phase_centre_ra_rad": ra0, "phase_centre_dec_rad": dec0,
        "freq_start_hz": 100e6, "freq_inc_hz": 15e6, "num_channels": 3,
        "mjd_start": workloads.MJD0, "inc_sec": 300.0, "num_times": 4,
        "num_devices": 1, "max_times_per_block": 4,
        "max_sources_per_chunk": 16384, "horizon_clip": 0,
        "correlation_type": "Both", "casa": 0,
        "source_min_jy": -1e300, "source_max_jy": 1e300,
    }
    case.update(over)
    return case


def c3_shaped_case(precision="double", num_src=100_000, num_channels=16,
                   num_times=4, **over):
    """The C3 shape through the reference simulator: 512 isotropic stations
    log-radial to 65 km (one shared station model), the C3 sky (point
    sources in a 10 deg field, full Stokes, S^-1.5) about the C configurations'
    phase centre,
    num_channels channels of 1 MHz from 100 MHz, num_times dumps of 10 s in
    one block, sky chunks of 16,384 sources (the reference's default), no
    smearing, horizon clip off (the field is above the horizon), visibilities
    not read back (a timing case). The reference's E here is its isotropic
    station beam, not C3's random E."""
    cfg = workloads.c3(num_src=num_src, num_channels=num_channels,
                       num_times=num_times)
    ra0, dec0 = cfg.ra0, cfg.dec0
    ra, dec = lm_to_radec(cfg.l, cfg.m, ra0, dec0)
    z = [0.0] * num_src
    case = c1_case(precision)
    case.update({
        "station_x": cfg.station_enu[0].tolist(),
        "station_y": cfg.station_enu[1].tolist(),
        "ra_rad": ra.tolist(), "dec_rad": dec.tolist(),
        "I": cfg.I.tolist(), "Q": cfg.Q.tolist(), "U": cfg.U.tolist(),
        "V": cfg.V.tolist(), "ref_freq_hz": list(z),
        "spectral_index": list(z), "rotation_measure": list(z),
        "major_rad": list(z), "minor_rad": list(z), "pa_rad": list(z),
        "phase_centre_ra_rad": ra0, "phase_centre_dec_rad": dec0,
        "freq_start_hz": 100e6, "freq_inc_hz": 1e6,
        "num_channels": num_channels, "inc_sec": 10.0,
        "num_times": num_times, "max_times_per_block": num_times,
        "max_sources_per_chunk": 16384, "horizon_clip": 0,
        "read_back": False,
    })
    case.update(over)
    return case
