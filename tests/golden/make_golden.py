"""Generates the golden fixtures in tests/golden/ from the reference's own
CPU kernels (oracle/_ref/liboskar_ref.so, compiled from the reference
sources by `make -C oracle ref`).

    python tests/golden/make_golden.py

Fixtures (inputs and outputs in one .npz each, FP64 unless noted):
  c1_vis.npz        the 30-station, 1,000-source, 10-dump, 100 MHz
                    configuration: station (u, v, w) per dump from the
                    reference ECEF -> uvw kernel, Jones K, join with an
                    identity station beam, point-source cross-correlation.
  smear_vis.npz     19 stations x 150 Gaussian sources with bandwidth and
                    time-average smearing (matrix, and scalar mode).
  f32_vis.npz       the c1 chain of dump 0 in single precision.
  dftw.npz          weighted DFT, 2x2 (m2m) 3-D with element types, and
                    complex (c2c) 2-D.
  c1_sim.npz        the c1 configuration run end to end through the
                    reference's own simulator (oskar_interferometer_run,
                    full polarisation with Jones R, one shared isotropic
                    station model) by tests/ref_sim.py with the reference's
                    CPU library (oracle/_ref/liboskar_refcpu.so, `make -C
                    oracle ref_lib`): cross-correlations [dump][channel]
                    [baseline x 2x2 complex] read back from its .vis file.
  c1_stations_sim.npz  the same with one station model per station, so that
                    Jones R follows each station's own latitude and
                    longitude.
Only the generator reads the reference library; the fixtures are plain data.
Run with --sim-only to remake just the simulator fixtures.
"""
import json
import subprocess
import tempfile
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle_lib import reference, reference_xcorr  # noqa: E402
from oskar_b200 import workloads  # noqa: E402

C0 = 299792458.0


def c1_chain(real=np.float64, dumps=None):
    cfg = workloads.c1()
    ref = reference()
    s = "d" if real == np.float64 else "f"
    nst, nsrc = cfg.num_st, cfg.num_src
    x, y, z = (np.ascontiguousarray(a, dtype=real) for a in cfg.ecef)
    l, m, n, I, Q, U, V = (np.ascontiguousarray(a, dtype=real) for a in
                           (cfg.l, cfg.m, cfg.n, cfg.I, cfg.Q, cfg.U, cfg.V))
    freq = float(cfg.freqs_hz[0])
    E = np.zeros((nst, nsrc, 8), real)
    E[..., 0] = 1
    E[..., 6] = 1
    dumps = range(cfg.num_times) if dumps is None else dumps
    nbl = cfg.num_baselines
    out_uvw, out_vis = [], []
    for t in dumps:
        ha = cfg.gast(t) - cfg.ra0
        uvw = [np.zeros(nst, real) for _ in range(3)]
        ref.call("ecef_to_station_uvw_" + s, real, nst, x, y, z,
                 math.sin(ha), math.cos(ha), math.sin(cfg.dec0),
                 math.cos(cfg.dec0), 0, 0, *uvw)
        K = np.zeros(2 * nst * nsrc, real)
        ref.call("jones_k_" + s, real, nsrc, l, m, n, nst, *uvw,
                 2 * math.pi * freq / C0, I, 0.0, 3e38, 0, K)
        J = np.zeros(8 * nst * nsrc, real)
        ref.call("mem_mul_cm_m_" + s, real, nst * nsrc, K, E.ravel(), J)
        vis = np.zeros(8 * nbl, real)
        z0 = np.zeros(nst, real)
        reference_xcorr(real, True, False, 0, nsrc, nst, 0, J, I, Q, U, V,
                        l, m, n, None, None, None, *uvw, z0, z0, 0.0, 3e38,
                        freq / C0, 0.0, 0.0, 0.0, 0.0, vis)
        out_uvw.append(np.stack(uvw))
        out_vis.append(vis.reshape(nbl, 8))
    return dict(ecef=np.stack([x, y, z]), l=l, m=m, n=n, I=I, Q=Q, U=U, V=V,
                freq=freq, ha=np.array([cfg.gast(t) - cfg.ra0
                                        for t in dumps]),
                dec0=cfg.dec0, uvw=np.stack(out_uvw), vis=np.stack(out_vis))


def smear_case():
    rng = np.random.default_rng(21)
    nst, nsrc = 19, 150
    r = np.sqrt(rng.uniform(0, 1, nsrc)) * math.sin(math.radians(3))
    th = rng.uniform(0, 2 * math.pi, nsrc)
    l, m = r * np.cos(th), r * np.sin(th)
    n = np.sqrt(1 - l * l - m * m)
    I = rng.uniform(0.5, 3, nsrc)
    Q, U, V = (I * rng.uniform(-0.1, 0.1, nsrc) for _ in range(3))
    a, b, c = (rng.uniform(1e-7, 2e-6, nsrc) for _ in range(3))
    u, v, w = (rng.uniform(-2e3, 2e3, nst) for _ in range(3))
    x, y = (rng.uniform(-2e3, 2e3, nst) for _ in range(2))
    J = rng.normal(0, 0.3, (nst, nsrc, 8)).ravel()
    Js = rng.normal(0, 0.3, (nst, nsrc, 2)).ravel()
    freq, bw, tavg, gha0, dec0 = 150e6, 100e3, 10.0, 0.7, -0.5
    nbl = nst * (nst - 1) // 2
    vis = np.zeros(8 * nbl)
    reference_xcorr(np.float64, True, True, 0, nsrc, nst, 0, J, I, Q, U, V,
                    l, m, n, a, b, c, u, v, w, x, y, 0.0, 3e38, freq / C0,
                    bw / freq, tavg, gha0, dec0, vis)
    vis_s = np.zeros(2 * nbl)
    reference_xcorr(np.float64, False, True, 1, nsrc, nst, 0, Js, I, Q, U, V,
                    l, m, n, a, b, c, u, v, w, x, y, 0.0, 3e38, freq / C0,
                    bw / freq, tavg, gha0, dec0, vis_s)
    return dict(J=J, Js=Js, I=I, Q=Q, U=U, V=V, l=l, m=m, n=n, a=a, b=b,
                c=c, u=u, v=v, w=w, x=x, y=y, freq=freq, bw=bw, tavg=tavg,
                gha0=gha0, dec0=dec0, vis=vis, vis_scalar=vis_s)


def dftw_case():
    rng = np.random.default_rng(22)
    ref = reference()
    n_in, n_out, n_types = 96, 500, 2
    k = 2 * math.pi * 110e6 / C0
    ph = rng.uniform(0, 2 * math.pi, n_in)
    w = np.stack([np.cos(ph), np.sin(ph)], 1).ravel()
    xi, yi, zi = (rng.uniform(-19, 19, n_in) for _ in range(3))
    zi *= 0.05
    xo, yo = (rng.uniform(-0.7, 0.7, n_out) for _ in range(2))
    zo = np.sqrt(np.maximum(1 - xo * xo - yo * yo, 0))
    idx = rng.integers(0, n_types, n_in).astype(np.int32)
    data_m = rng.uniform(-1, 1, n_types * n_out * 8)
    n_c = 32  # elements of the c2c case, one data row each
    data_c = rng.uniform(-1, 1, n_c * n_out * 2)
    out_m = np.zeros(n_out * 8)
    ref.call("dftw_d", np.float64, 1, 1, n_in, k, w, xi, yi, zi, 0, n_out,
             xo, yo, zo, idx, data_m, 1, 1, 0, out_m, 1.0 / n_in)
    out_c = np.zeros(n_out * 2)
    ref.call("dftw_d", np.float64, 0, 0, n_c, k, w, xi, yi, None, 0, n_out,
             xo, yo, None, None, data_c, 1, 1, 0, out_c, 1.0)
    return dict(k=k, w=w, xi=xi, yi=yi, zi=zi, xo=xo, yo=yo, zo=zo, idx=idx,
                n_c=n_c, data_m=data_m, data_c=data_c, out_m=out_m,
                out_c=out_c)


def sim_fixtures():
    """The end-to-end fixtures from the reference simulator (its horizon
    clip off: every source of the field is above the horizon)."""
    from dropin_cases import c1_case
    ref_lib = os.path.join(ROOT, "oracle", "_ref", "liboskar_refcpu.so")
    if not os.path.exists(ref_lib):
        raise SystemExit("reference library not built: make -C oracle "
                         "REF_SRC=... ref_lib")
    cases = {"c1_sim.npz": c1_case("double", horizon_clip=0),
             "c1_stations_sim.npz": c1_case("double", horizon_clip=0,
                                            station_per_folder=1)}
    env = {k: v for k, v in os.environ.items() if k != "LD_PRELOAD"}
    with tempfile.TemporaryDirectory() as tmp:
        for name, case in cases.items():
            cj = os.path.join(tmp, "case.json")
            with open(cj, "w") as f:
                json.dump(case, f)
            out = os.path.join(HERE, name)
            # the reference's CPU run is repeated if it crashes (it was
            # seen to, now and then, in its flux scaling)
            for _ in range(4):
                r = subprocess.run([sys.executable, os.path.join(
                    os.path.dirname(HERE), "ref_sim.py"), cj, out], env=env)
                if r.returncode == 0:
                    break
            if r.returncode:
                raise SystemExit("reference simulator failed: %d"
                                 % r.returncode)
            d = dict(np.load(out))
            d.pop("run_seconds", None)
            np.savez_compressed(out, **d)


def main():
    if "--sim-only" in sys.argv:
        sim_fixtures()
        return
    if reference() is None:
        raise SystemExit("reference kernels not built: make -C oracle ref")
    np.savez_compressed(os.path.join(HERE, "c1_vis.npz"), **c1_chain())
    np.savez_compressed(os.path.join(HERE, "f32_vis.npz"),
                        **c1_chain(np.float32, dumps=[0]))
    np.savez_compressed(os.path.join(HERE, "smear_vis.npz"), **smear_case())
    np.savez_compressed(os.path.join(HERE, "dftw.npz"), **dftw_case())
    sim_fixtures()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
