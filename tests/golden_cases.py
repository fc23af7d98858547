"""Loads the golden fixtures (tests/golden/*.npz, generated from the
reference's own CPU kernels by tests/golden/make_golden.py) and replays
their inputs through a given implementation of the hot path."""
import math
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
C0 = 299792458.0


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def c1_identity_e(nst, nsrc, real=np.float64):
    E = np.zeros((nst, nsrc, 8), real)
    E[..., 0] = 1
    E[..., 6] = 1
    return E.ravel()


def rel_err(got, ref):
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    return (float(np.linalg.norm(got - ref) / np.linalg.norm(ref)),
            float(np.max(np.abs(got - ref)) / np.max(np.abs(ref))))


def c1_oracle(g, oracle, real=np.float64):
    """The c1 chain (uvw, K, join, correlate) through the CPU oracle."""
    s = "d" if real == np.float64 else "f"
    x, y, z = (np.ascontiguousarray(a, dtype=real) for a in g["ecef"])
    nst = x.size
    l, m, n, I, Q, U, V = (np.ascontiguousarray(g[k], dtype=real)
                           for k in "l m n I Q U V".split())
    nsrc = l.size
    E = c1_identity_e(nst, nsrc, real)
    freq = float(g["freq"])
    out = []
    for ha in g["ha"]:
        uvw = [np.zeros(nst, real) for _ in range(3)]
        oracle.call("ecef_to_station_uvw_" + s, real, nst, x, y, z,
                    math.sin(ha), math.cos(ha), math.sin(float(g["dec0"])),
                    math.cos(float(g["dec0"])), 0, 0, *uvw)
        K = np.zeros(2 * nst * nsrc, real)
        oracle.call("jones_k_" + s, real, nsrc, l, m, n, nst, *uvw,
                    2 * math.pi * freq / C0, I, 0.0, 3e38, 0, K)
        J = np.zeros(8 * nst * nsrc, real)
        oracle.call("mem_mul_cm_m_" + s, real, nst * nsrc, K, E, J)
        nbl = nst * (nst - 1) // 2
        vis = np.zeros(8 * nbl, real)
        z0 = np.zeros(nst, real)
        oracle.call("xcorr_matrix_" + s, real, 0, 0, nsrc, nst, 0, J, I, Q,
                    U, V, l, m, n, None, None, None, *uvw, z0, z0, 0.0, 3e38,
                    freq / C0, 0.0, 0.0, 0.0, 0.0, vis)
        out.append(vis.reshape(nbl, 8))
    return np.stack(out)
