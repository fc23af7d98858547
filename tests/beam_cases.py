"""Seeded station-beam inputs shared by the oracle pin tests and the GPU
beam tests, and the oracle's composite station beam for them."""
import numpy as np

from oracle_lib import oracle, suffix


def enu_dirs(rng, n, real, below=0.1):
    """Unit ENU directions, a fraction of them below the horizon."""
    az = rng.uniform(0, 2 * np.pi, n)
    el = rng.uniform(-below * np.pi / 2, np.pi / 2, n)
    x, y, z = np.cos(el) * np.sin(az), np.cos(el) * np.cos(az), np.sin(el)
    return [np.ascontiguousarray(a, dtype=real) for a in (x, y, z)]


def beam_case(real, seed=14, num_el=256, num_dir=1001, is_3d=1):
    """A 38 m dipole station, directions over the sky (some below the
    horizon), beam and normalisation pointing above the horizon."""
    rng = np.random.default_rng(seed)
    r = 19.0 * np.sqrt(rng.uniform(0, 1, num_el))
    t = rng.uniform(0, 2 * np.pi, num_el)
    x, y = r * np.cos(t), r * np.sin(t)
    z = rng.uniform(-0.3, 0.3, num_el) if is_3d else np.zeros(num_el)
    meas = [a + rng.normal(0, 0.01, num_el) for a in (x, y, z)]
    cable = rng.normal(0, 0.02, num_el)
    dx, dy, dz = enu_dirs(rng, num_dir, np.float64)
    b = np.array([0.2, 0.3, 0.0])
    b[2] = np.sqrt(1 - b[0] ** 2 - b[1] ** 2)
    el = [np.ascontiguousarray(a, dtype=real) for a in (x, y, z)]
    me = [np.ascontiguousarray(a, dtype=real) for a in meas]
    dirs = [np.ascontiguousarray(a, dtype=real) for a in (dx, dy, dz)]
    return dict(el=el, meas=me, cable=cable.astype(real), dirs=dirs, b=b,
                norm=b.copy(), freq=110e6, orient=(0.3, 0.3 + np.pi / 2),
                L=1.5)


def oracle_beam(c, real, flags, use_meas=True):
    norm_el, norm_arr, norm_fin, swap, is_3d = flags
    out = np.zeros(8 * len(c["dirs"][0]), real)
    oracle().call("station_beam_aa_" + suffix(real), np.float64,
                  len(c["el"][0]), *c["el"],
                  *(c["meas"] if use_meas else (None, None, None)),
                  c["cable"], *c["orient"], c["L"], norm_el, norm_arr,
                  norm_fin, swap, is_3d, c["freq"], *c["b"], *c["norm"],
                  len(c["dirs"][0]), *c["dirs"], out)
    return out
