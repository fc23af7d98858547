"""Seeded input sets for the cross-correlation parity tests.

The value ranges follow the reference's consistency test
(oskar/correlate/test/Test_cross_correlate.cpp:50-120): Jones in [1, 5],
station (u, v, w) in [1, 5] m, ECEF offsets in [0.1, 1000] m,
I in [1, 2], Q in [0.1, 1], U in [0.1, 0.5], V in [0.1, 0.2],
l, m, n in [0.1, 0.9], Gaussian a, b, c in [1e-7, 2e-7]; gast = 1 rad,
100 MHz, CASA convention selectable.
"""
import numpy as np

FREQ_HZ = 100e6
C0 = 299792458.0


class XcorrCase:
    def __init__(self, num_st, num_src, real=np.float64, seed=2, matrix=True,
                 gaussian=False, bandwidth_hz=0.0, time_avg=0.0, casa=0,
                 uv_min=0.0, uv_max=np.finfo(np.float32).max, offset_out=0,
                 ranges="oskar_test"):
        rng = np.random.default_rng(seed)
        self.num_st, self.num_src, self.real = num_st, num_src, real
        self.matrix, self.gaussian, self.casa = matrix, gaussian, casa
        self.offset_out = offset_out
        u = lambda lo, hi, n: rng.uniform(lo, hi, n).astype(real)
        ncomp = 8 if matrix else 2
        if ranges == "oskar_test":
            self.jones = u(1, 5, num_st * num_src * ncomp)
            self.I, self.Q = u(1, 2, num_src), u(0.1, 1, num_src)
            self.U, self.V = u(0.1, 0.5, num_src), u(0.1, 0.2, num_src)
            self.l, self.m, self.n = (u(0.1, 0.9, num_src) for _ in range(3))
            self.st_u, self.st_v, self.st_w = (u(1, 5, num_st)
                                               for _ in range(3))
        else:  # physical: unit direction cosines, km-scale array
            j = rng.normal(0, 0.1, (num_st, num_src, ncomp))
            if matrix:
                j[..., 0] += 1.0
                j[..., 6] += 1.0
            else:
                j[..., 0] += 1.0
            self.jones = j.astype(real).ravel()
            self.I = u(0.01, 10, num_src)
            self.Q, self.U, self.V = (self.I * u(-0.1, 0.1, num_src)
                                      for _ in range(3))
            r = np.sqrt(rng.uniform(0, 1, num_src)) * np.radians(5)
            th = rng.uniform(0, 2 * np.pi, num_src)
            l_, m_ = r * np.cos(th), r * np.sin(th)
            self.l, self.m = l_.astype(real), m_.astype(real)
            self.n = np.sqrt(1 - l_ * l_ - m_ * m_).astype(real)
            self.st_u, self.st_v = u(-500, 500, num_st), u(-500, 500, num_st)
            self.st_w = u(-20, 20, num_st)
        self.a, self.b, self.c = (u(1e-7, 2e-7, num_src) for _ in range(3))
        self.st_x, self.st_y = u(0.1, 1000, num_st), u(0.1, 1000, num_st)
        self.freq = FREQ_HZ
        self.inv_wavelength = FREQ_HZ / C0
        self.frac_bandwidth = bandwidth_hz / FREQ_HZ
        self.time_avg = time_avg
        self.gha0 = 1.0 - 0.0  # gast - RA0, with RA0 = 0
        self.dec0 = np.radians(-30.0) if ranges != "oskar_test" else 0.5
        self.uv_min, self.uv_max = uv_min, uv_max
        nbl = num_st * (num_st - 1) // 2
        self.num_vis = nbl + offset_out
        self.vis0 = rng.uniform(-1, 1, self.num_vis * ncomp).astype(real)

    def oracle_args(self, vis):
        """Argument list of orc_xcorr_{matrix,scalar} after ``gaussian``."""
        return [self.num_src, self.num_st, self.offset_out, self.jones,
                self.I, self.Q, self.U, self.V, self.l, self.m, self.n,
                self.a, self.b, self.c, self.st_u, self.st_v, self.st_w,
                self.st_x, self.st_y, float(self.uv_min), float(self.uv_max),
                float(self.inv_wavelength), float(self.frac_bandwidth),
                float(self.time_avg), float(self.gha0), float(self.dec0),
                vis]


def rel_errors(got, ref):
    """(max, mean) relative error as the reference tests use it
    (oskar/mem/src/oskar_mem_evaluate_relative_error.c:42-62, magnitude
    based), and the stricter L2 relative error of the complex difference."""
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    l2 = np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-300)
    denom = np.maximum(np.abs(ref), 1e-300)
    per = np.abs(got - ref) / denom
    return float(per.max()), float(per.mean()), float(l2)
