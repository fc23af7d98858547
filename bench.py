"""Benchmark of the visibility hot path on the 512-station configuration.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--path tc|direct]

Workload (oskar_b200/workloads.py, c3): 512 stations, 100,000 point sources,
16 channels, 64 dumps; a STEP is one dump (time sample) of the full sky for
all 16 channels: per channel the station (u, v, w) is turned into the
interferometer phase K, joined with the station beam E (J = K E) and
correlated into 130,816 baselines x 4 polarisations. Source-baselines per
step = 130,816 x 100,000 x 16 = 2.09e11.

--path tc (default) uses the tensor-core compensated contraction with the
FP64 phase; --path direct uses the FP64 direct kernels. The reported metric
is source-baselines per second over all ranks; N > 1 shards dumps across
ranks with no data-path collective (weak scaling).

--impl reference times the reference's own CPU implementation of the same
path (its OpenMP kernels compiled from its sources into
oracle/_ref/liboskar_ref.so) on the host cores, on a bounded sample of the
workload per step (one channel, a source subset sized to a few seconds).
"""
import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "G source-baselines/s at 512 stn (TC compensated, rel err vs FP64)"
UNIT = "G source-baselines/s"


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while the
    timed region runs."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,"
             "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu_index = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu_index),
                 "--query-gpu=" + self.QUERY, "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["n/a"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- helpers
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def ref_lib():
    path = os.path.join(ROOT, "oracle", "_ref", "liboskar_ref.so")
    if not os.path.exists(path):
        return None
    return ctypes.CDLL(path)


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else \
        ctypes.c_void_p(0)


def reference_cpu_sample(cfg, num_src, t=0, ch=0):
    """Runs the reference's CPU path (Jones K, join K*E, cross-correlation,
    all FP64 OpenMP kernels compiled from the reference sources) for one
    (dump, channel) on the first num_src sources. Returns (seconds,
    source-baselines)."""
    lib = ref_lib()
    if lib is None:
        raise RuntimeError("oracle/_ref/liboskar_ref.so not built")
    rng = np.random.default_rng(11)
    nst = cfg.num_st
    E = rng.normal(0, 0.1, (nst, num_src, 8))
    E[..., 0] += 1
    E[..., 6] += 1
    uvw = cfg.station_uvw(t)
    u, v, w = (np.ascontiguousarray(x) for x in uvw)
    sl = slice(0, num_src)
    l, m, n = (np.ascontiguousarray(x[sl]) for x in (cfg.l, cfg.m, cfg.n))
    I, Q, U, V = (np.ascontiguousarray(x[sl]) for x in
                  (cfg.I, cfg.Q, cfg.U, cfg.V))
    freq = float(cfg.freqs_hz[ch])
    K = np.zeros((nst, num_src, 2))
    J = np.zeros((nst, num_src, 8))
    vis = np.zeros((cfg.num_baselines, 8))
    zeros = np.zeros(nst)
    D = ctypes.c_double
    t0 = time.perf_counter()
    lib.ref_jones_k_d(num_src, _p(l), _p(m), _p(n), nst, _p(u), _p(v),
                      _p(w), D(2 * math.pi * freq / 299792458.0), _p(I),
                      D(0.0), D(1e300), 0, _p(K))
    lib.ref_mem_mul_cm_m_d(nst * num_src, _p(K), _p(E), _p(J))
    lib.oskar_cross_correlate_point_omp_d(
        0, num_src, nst, 0, _p(J), _p(I), _p(Q), _p(U), _p(V), _p(l), _p(m),
        _p(n), _p(u), _p(v), _p(w), _p(zeros), _p(zeros), D(0.0), D(3e38),
        D(freq / 299792458.0), D(0.0), D(0.0), D(0.0), D(0.0), _p(vis))
    dt = time.perf_counter() - t0
    return dt, cfg.num_baselines * num_src


def calibrate_cpu_sample(cfg, target_sec):
    """Source count whose reference CPU sample takes about target_sec."""
    n0 = 500
    dt, _ = reference_cpu_sample(cfg, n0)
    n = int(n0 * target_sec / max(dt, 1e-3))
    return max(500, min(n, cfg.num_src))


# ---------------------------------------------------------------- reference
def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    from oskar_b200 import workloads
    cfg = workloads.c3()
    cores = cpu_cores()
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    if ref_lib() is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/liboskar_ref.so was not built"}))
        return 0
    nsrc = calibrate_cpu_sample(cfg, 4.0)
    for i in range(args.warmup):
        reference_cpu_sample(cfg, nsrc, t=i % cfg.num_times)
    tot_t, tot_w = 0.0, 0
    for i in range(args.steps):
        dt, work = reference_cpu_sample(cfg, nsrc, t=i % cfg.num_times,
                                        ch=i % len(cfg.freqs_hz))
        tot_t += dt
        tot_w += work
    value = tot_w / tot_t / 1e9
    sample = ("1 dump x 1 channel x %d of 100000 sources x 130816 baselines "
              "per step (Jones K + join + FP64 cross-correlation)" % nsrc)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot_t / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "c3: 512 stations, 100k point sources, "
                   "16 ch x 64 dumps (CPU sample)", "stations": 512,
                   "sources": 100000, "channels": 16, "dumps": 64},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }))
    return 0


# ---------------------------------------------------------------- ours
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--path", default="tc", choices=["tc", "direct"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    from oskar_b200 import benchpath
    return benchpath.run(args, ClockSampler, dist_setup, reference_cpu_sample,
                         calibrate_cpu_sample, cpu_cores, METRIC, UNIT)


if __name__ == "__main__":
    sys.exit(main())
