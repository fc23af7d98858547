"""A seeded block of dumps x channels with a sky in uneven chunks (point
and Gaussian chunks, as the reference groups its sky), and the oracle's
result for it computed the way the reference's sim_baselines does: for each
dump, chunk and channel, Jones K, join with E, cross-correlate into the
block (oskar/interferometer/src/oskar_interferometer_run_block.c:156-336)."""
import math

import numpy as np

from oracle_lib import oracle, suffix

C0 = 299792458.0


class BlockCase:
    def __init__(self, num_st=40, chunks=(37, 5, 120, 64), gaussian=(0, 1,
                 1, 0), num_times=3, num_channels=4, real=np.float64,
                 seed=11, bandwidth_hz=1e5, time_avg=10.0, beam=True,
                 beam_per_dump=False, uv_min_m=0.0, uv_max_m=3.0e38,
                 filter_min=0.0, filter_max=3.0e38, casa=0):
        rng = np.random.default_rng(seed)
        self.real, self.casa = real, casa
        self.num_st, self.num_times, self.num_channels = (num_st, num_times,
                                                          num_channels)
        self.chunks, self.gaussian = list(chunks), list(gaussian)
        ns = self.num_src = int(sum(chunks))
        r = np.sqrt(rng.uniform(0, 1, ns)) * math.sin(math.radians(4))
        th = rng.uniform(0, 2 * math.pi, ns)
        l, m = r * np.cos(th), r * np.sin(th)
        n = np.sqrt(1 - l * l - m * m)
        I = rng.uniform(0.2, 3.0, ns)
        Q, U, V = (I * rng.uniform(-0.1, 0.1, ns) for _ in range(3))
        a, b, c = (rng.uniform(1e-8, 5e-7, ns) for _ in range(3))
        # point-source chunks carry a = b = c = 0
        s0 = 0
        for size, g in zip(chunks, gaussian):
            if not g:
                a[s0:s0 + size] = b[s0:s0 + size] = c[s0:s0 + size] = 0
            s0 += size
        cast = lambda x: np.ascontiguousarray(x, dtype=real)
        self.l, self.m, self.n, self.I, self.Q, self.U, self.V = map(
            cast, (l, m, n, I, Q, U, V))
        self.a, self.b, self.c = map(cast, (a, b, c))
        self.st_x, self.st_y = (cast(rng.uniform(-3e3, 3e3, num_st))
                                for _ in range(2))
        self.uvw = cast(rng.uniform(-3e3, 3e3, (num_times, 3, num_st)))
        self.freqs = 100e6 + 1e6 * np.arange(num_channels)
        self.inv_wl = self.freqs / C0
        self.gha0 = rng.uniform(-1, 1, num_times)
        self.dec0 = -0.45
        self.bw, self.tavg = bandwidth_hz, time_avg
        self.uv_min_m, self.uv_max_m = uv_min_m, uv_max_m
        self.filter_min, self.filter_max = filter_min, filter_max
        nE = num_times if beam_per_dump else 1
        E = rng.normal(0, 0.1, (nE, num_st, ns, 8))
        E[..., 0] += 1
        E[..., 6] += 1
        self.E = cast(E) if beam else None
        self.beam_per_dump = beam_per_dump
        self.nbl = num_st * (num_st - 1) // 2
        self.flux_c = None

    def set_spectral(self, sky):
        """Brightness per channel from a sky table (tests/sky_cases.py),
        scaled by the oracle at each channel frequency: flux_c[k] is
        [channel][source] for k in I, Q, U, V."""
        from sky_cases import call_scale
        assert sky.num_sources == self.num_src
        per = [call_scale(oracle(), self.real, sky, f) for f in self.freqs]
        self.flux_c = {k: np.ascontiguousarray(np.stack([p[j] for p in per]))
                       for j, k in enumerate("IQUV")}

    def oracle_vis(self, channels=None):
        """The block's visibilities [dump][channel][baseline][2x2] from the
        oracle; with `channels`, only those channels are computed (the
        others stay 0)."""
        real, s = self.real, suffix(self.real)
        T, C, N, nbl = self.num_times, self.num_channels, self.num_st, \
            self.nbl
        vis = np.zeros(T * C * nbl * 8, real)
        chans = range(C) if channels is None else channels
        orc = oracle()
        s0 = 0
        for size, g in zip(self.chunks, self.gaussian):
            sl = slice(s0, s0 + size)
            ch = {k: np.ascontiguousarray(getattr(self, k)[sl]) for k in
                  "lmnIQUVabc"}
            for t in range(T):
                u, v, w = (np.ascontiguousarray(self.uvw[t, k])
                           for k in range(3))
                if self.E is not None:
                    Et = self.E[t if self.beam_per_dump else 0][:, sl]
                    Et = np.ascontiguousarray(Et)
                for c in chans:
                    f = self.freqs[c]
                    if self.flux_c is not None:
                        for k in "IQUV":
                            ch[k] = np.ascontiguousarray(self.flux_c[k][c,
                                                                        sl])
                    K = np.zeros(2 * N * size, real)
                    orc.call("jones_k_" + s, real, size, ch["l"], ch["m"],
                             ch["n"], N, u, v, w, real(2 * math.pi * f / C0),
                             ch["I"], real(self.filter_min),
                             real(min(self.filter_max, 3e38)), 0, K)
                    if self.E is not None:
                        J = np.zeros(8 * N * size, real)
                        orc.call("mem_mul_cm_m_" + s, real, N * size, K,
                                 Et, J)
                    else:
                        Kc = K.reshape(-1, 2)
                        J = np.zeros((N * size, 8), real)
                        J[:, 0:2] = Kc
                        J[:, 6:8] = Kc
                        J = J.ravel()
                    inv = self.inv_wl[c]
                    orc.call("xcorr_matrix_" + s, real, self.casa, g, size,
                             N, (t * C + c) * nbl, J, ch["I"], ch["Q"],
                             ch["U"], ch["V"], ch["l"], ch["m"], ch["n"],
                             ch["a"], ch["b"], ch["c"], u, v, w, self.st_x,
                             self.st_y, real(self.uv_min_m * inv),
                             real(min(self.uv_max_m * inv, 3e38)), real(inv),
                             real(self.bw / f), real(self.tavg),
                             real(self.gha0[t]), real(self.dec0), vis)
            s0 += size
        return vis
