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

--workload c2 measures the aperture-array chain (station beams, Jones R,
joins, Jones K, correlation; 128 stations x 256 dipoles, 12,000 sources);
--workload c5 the learned station-beam surrogate against the exact beam.
Each prints its own JSON line; the default (c3) line is the headline.
--profile-case runs one small kernel case for an ncu capture.

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
def _load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            pk = json.load(f)
        return pk, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0,
            "bf16_tflops_sustained": 1400.0}, "fallback"


def _load_traffic(tile, arith=16):
    """DRAM bytes per launch of the contraction kernel (integer, or FP16
    square, wide or pair tiles) from the committed ncu summary
    (profiles/tc_gemm{_i8,,_wide,_pair}_c3_traffic.json), or None."""
    name = "tc_gemm_i8_c3_traffic.json" if arith == 8 else {
        256: "tc_gemm_wide_c3_traffic.json",
        512: "tc_gemm_pair_c3_traffic.json"}.get(
            tile, "tc_gemm_c3_traffic.json")
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None
    with open(path) as f:
        return json.load(f).get("dram_bytes_per_launch")


def run_ours(args):
    import torch
    import torch.distributed as dist
    import oskar_b200 as ob
    from oskar_b200 import workloads

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(
            seconds=300), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    cfg = workloads.c3()
    nst, nsrc, nch = cfg.num_st, cfg.num_src, len(cfg.freqs_hz)
    nbl = cfg.num_baselines
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    l, m, n, I, Q, U, V = (dev(x) for x in (cfg.l, cfg.m, cfg.n, cfg.I,
                                            cfg.Q, cfg.U, cfg.V))
    E = workloads.jones_e_device(cfg, torch.float32)
    uvw_all = dev(np.stack([cfg.station_uvw(t)
                            for t in range(cfg.num_times)]))
    inv_wl = dev(cfg.freqs_hz / 299792458.0)
    vis = torch.zeros((nch, nbl, 8), dtype=torch.float64, device="cuda")
    stream = ob.stream_ptr()
    sb_step = nbl * nsrc * nch  # source-baselines per step

    if args.path == "tc":
        ws_bytes = ob.call("oskb_correlate_block_tc_workspace_bytes", nsrc,
                           nst, nch, check=False)
        ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
        launches_per_step = 3

        def step(d):
            vis.zero_()
            ob.call("oskb_correlate_block_tc", 0, nsrc, nst, 1, nch, E, l, m,
                    n, I, Q, U, V, uvw_all[d], inv_wl, 0.0, 3e38, vis, ws,
                    ws_bytes, stream)
    else:
        Ed = E.double()
        K = torch.empty((nst, nsrc, 2), dtype=torch.float64, device="cuda")
        J = torch.empty((nst, nsrc, 8), dtype=torch.float64, device="cuda")
        z = torch.zeros(nst, dtype=torch.float64, device="cuda")
        launches_per_step = 3 * nch + 0

        def step(d):
            vis.zero_()
            u, v, w = uvw_all[d]
            for c in range(nch):
                f = float(cfg.freqs_hz[c])
                ob.call("oskb_evaluate_jones_K_d", nsrc, l, m, n, nst, u, v,
                        w, 2 * math.pi * f / 299792458.0, I, 0.0, 1e300, 0,
                        K, stream)
                ob.call("oskb_mem_multiply_d", 3, 0, 0, 0, nst * nsrc, K, Ed,
                        J, stream)
                ob.call("oskb_cross_correlate_d", 0, 0, nsrc, nst, 0, J, I,
                        Q, U, V, l, m, n, None, None, None, u, v, w, z, z,
                        0.0, 3e38, f / 299792458.0, 0.0, 0.0, 0.0, 0.0,
                        vis[c], stream)

    from oskar_b200.sharding import dump_of_step, max_over_ranks
    dump = lambda i: dump_of_step(i, world, rank, cfg.num_times)
    for i in range(args.warmup):
        step(dump(i))
    torch.cuda.synchronize()
    if args.path == "tc" and ob.load().oskb_tc_arithmetic() == 8:
        # the integer form adds the per-source amplitudes and the source
        # order to scale, operand preparation and contraction
        launches_per_step = 4
    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    if args.path == "tc":
        ob.call("oskb_tc_timing", 1)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for i in range(args.steps):
        step(dump(args.warmup + i))
    e1.record()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms_total = e0.elapsed_time(e1)
    gemm_ms, gemm_launches = None, 0
    if args.path == "tc":
        import ctypes
        t_ms, n_l = ctypes.c_double(0), ctypes.c_int(0)
        ob.call("oskb_tc_timing_read", ctypes.addressof(t_ms),
                ctypes.addressof(n_l))
        ob.call("oskb_tc_timing", 0)
        gemm_ms, gemm_launches = t_ms.value, n_l.value
    ms_max = max_over_ranks(ms_total)
    value = sb_step * args.steps * world / (ms_max * 1e-3) / 1e9

    result = None
    if rank == 0:
        peaks, peak_kind = _load_peaks()
        # ---- roofline of the dominant kernel
        if args.path == "tc":
            avg = gemm_ms / max(gemm_launches, 1)
            sb_launch = sb_step * args.steps / max(gemm_launches, 1)
            ach = 64.0 * sb_launch / (avg * 1e-3) / 1e12
            pk = peaks["bf16_tflops_sustained"]
            nrb = (nst + 31) // 32
            kp = 2 * 32 * ((nsrc + 31) // 32)
            tile = ob.load().oskb_tc_tile_columns()
            arith = ob.load().oskb_tc_arithmetic()
            issued_pk, issued_kind = pk, "measured bf16 sustained"
            if arith == 8:
                # integer form: six 8-bit limb products per K step (2 ops
                # per multiply-add) on square tiles (the bucket padding, at
                # most 15 source blocks, is not counted); the 8-bit dense
                # rate is twice the 16-bit one
                issued = nch * nrb * (nrb + 1) // 2 * 128 * 128 * kp * 2 * 6
                issued_pk = 2 * pk
                issued_kind = ("2 x measured bf16 sustained (the int8 dense "
                               "tensor rate is twice the bf16 one)")
            elif tile == 512:
                # pair tiles: 256 x 256 per CTA pair over the triangle of
                # row-block pairs
                npr = (nrb + 1) // 2
                issued = nch * npr * (npr + 1) // 2 * 256 * 256 * kp * 2 * 3
            elif tile == 256:
                # wide tiles: 128 x 256 columns per task over the triangle
                ntile = sum(min(2 * cp + 2, nrb)
                            for cp in range((nrb + 1) // 2))
                issued = nch * ntile * 128 * 256 * kp * 2 * 3
            else:
                issued = nch * nrb * (nrb + 1) // 2 * 128 * 128 * kp * 2 * 3
            issued_tf = issued / (avg * 1e-3) / 1e12
            traffic = _load_traffic(tile, arith)
            roof = {"bound": "tensor", "achieved": ach, "peak": pk,
                    "unit": "TFLOP/s", "frac": ach / pk, "traffic": traffic,
                    "kernel": "oskb::tc::gemm_i8_kernel" if arith == 8
                              else {256: "oskb::tc::gemm_wide_kernel",
                                    512: "oskb::tc::gemm_pair_kernel"}.get(
                                        tile, "oskb::tc::gemm_kernel"),
                    "tile_columns": tile,
                    "arithmetic": "int8 x3 limbs (6 products, amplitude "
                                  "buckets) -> exact s32" if arith == 8
                                  else "fp16 hi/lo x3 -> f32 -> f64",
                    "peak_kind": "%s bf16 sustained (fp16 same rate)"
                                 % peak_kind,
                    "algorithmic_flops_per_launch": 64.0 * sb_launch,
                    "issued_tflops": issued_tf,
                    "issued_frac": issued_tf / issued_pk,
                    "issued_peak_kind": issued_kind,
                    "avg_launch_ms": avg,
                    "share_of_step": gemm_ms / ms_total}
        else:
            roof = {"bound": "fp64", "achieved": None, "peak": None,
                    "unit": "TFLOP/s", "frac": None, "traffic": None}
        # ---- direct FP64 comparison and error on dump 0, channel 0
        cmp_ = compare_direct(args, cfg, ob, torch, dev, E, l, m, n, I, Q, U,
                              V, uvw_all, inv_wl, stream)
        result = {
            "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": ("int8x3 limbs->s32 exact (TC), f64 phase"
                      if roof.get("arithmetic", "").startswith("int8") else
                      "fp16x3->f32->f64 (TC), f64 phase")
                     if args.path == "tc" else "f64",
            "data": "synthetic",
            "config": {"workload": "c3: 512 stations log-radial to 65 km, "
                       "100,000 point sources (full Stokes), 2x2 E per "
                       "station-source, 16 ch x 64 dumps; step = 1 dump x "
                       "16 ch", "stations": nst, "sources": nsrc,
                       "channels": nch, "dumps": cfg.num_times,
                       "path": args.path,
                       "parallelism": "dumps sharded over %d rank(s)" % world,
                       "l2": "inputs larger than L2 (E 1.6 GB; operand "
                             "images %.1f GB per step)" % (
                                 nst * nsrc * nch * (24 if roof.get(
                                     "arithmetic", "").startswith("int8")
                                     else 32) / 1e9)},
            "gpu_launches": launches_per_step * args.steps,
            "roofline": roof, "clocks": clk,
            "direct_fp64": cmp_["direct"],
            "direct_fp64_dmma": cmp_["direct_dmma"],
            "fp64_class_tc64": cmp_["tc64"],
            "fp64_class_block": cmp_["block64"],
            "speedup_vs_direct_fp64": value / cmp_["direct"]["value"],
            "speedup_vs_direct_fp64_dmma":
                value / cmp_["direct_dmma"]["value"],
            "rel_err_vs_fp64": cmp_["err"],
        }
    # ---- end to end through the host-buffer entry point
    e2e = run_e2e(args, cfg, ob, torch, E, world, rank)
    if rank == 0:
        result["e2e"] = e2e
        if world == 1 and not args.no_cpu_baseline:
            result["cpu_baseline"] = cpu_baseline(cfg)
        print(json.dumps(result))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def compare_direct(args, cfg, ob, torch, dev, E, l, m, n, I, Q, U, V,
                   uvw_all, inv_wl, stream):
    """The FP64 direct comparison: throughput of the FP64 direct kernels on
    one (dump, channel) at the full sky (the SIMT kernel, the plain form,
    and the default FP64 tensor-pipe DMMA kernel), and the tensor-core
    result's error against the FP64 direct result on dumps 0 and last,
    channels 0, 7 and 15: L2 relative and max |err| / max |V|, the worst
    over those six (dump, channel) problems."""
    nst, nsrc, nbl = cfg.num_st, cfg.num_src, cfg.num_baselines
    nch = len(cfg.freqs_hz)
    Ed = E.double()
    K = torch.empty((nst, nsrc, 2), dtype=torch.float64, device="cuda")
    J = torch.empty((nst, nsrc, 8), dtype=torch.float64, device="cuda")
    z = torch.zeros(nst, dtype=torch.float64, device="cuda")
    vd = torch.zeros((nbl, 8), dtype=torch.float64, device="cuda")

    def join(d, c):
        u, v, w = uvw_all[d]
        f = float(cfg.freqs_hz[c])
        ob.call("oskb_evaluate_jones_K_d", nsrc, l, m, n, nst, u, v, w,
                2 * math.pi * f / 299792458.0, I, 0.0, 1e300, 0, K, stream)
        ob.call("oskb_mem_multiply_d", 3, 0, 0, 0, nst * nsrc, K, Ed, J,
                stream)

    def direct(d, c):
        u, v, w = uvw_all[d]
        f = float(cfg.freqs_hz[c])
        ob.call("oskb_cross_correlate_d", 0, 0, nsrc, nst, 0, J, I, Q, U, V,
                l, m, n, None, None, None, u, v, w, z, z, 0.0, 3e38,
                f / 299792458.0, 0.0, 0.0, 0.0, 0.0, vd, stream)

    def timed(kernel_env):
        old = os.environ.get("OSKB_XCORR_DMMA")
        os.environ["OSKB_XCORR_DMMA"] = kernel_env
        try:
            direct(0, 0)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            reps = 3
            e0.record()
            for _ in range(reps):
                direct(0, 0)
            e1.record()
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / reps
        finally:
            if old is None:
                del os.environ["OSKB_XCORR_DMMA"]
            else:
                os.environ["OSKB_XCORR_DMMA"] = old

    def tc64(d, c, out):
        u, v, w = uvw_all[d]
        f = float(cfg.freqs_hz[c])
        ob.call("oskb_cross_correlate_tc64_d", 0, nsrc, nst, 0, J, I, Q, U,
                V, u, v, 0.0, 3e38, f / 299792458.0, out, None, 0, stream)

    join(0, 0)
    ms_simt = timed("0")
    ms_dmma = timed("1")
    # the FP64-class integer tensor-core form on the same J, and its error
    # against the FP64 direct (DMMA) result
    v64 = torch.zeros((nbl, 8), dtype=torch.float64, device="cuda")
    tc64(0, 0, v64)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(3):
        tc64(0, 0, v64)
    e1.record()
    torch.cuda.synchronize()
    ms_tc64 = e0.elapsed_time(e1) / 3
    v64.zero_()
    tc64(0, 0, v64)
    vd.zero_()
    direct(0, 0)
    torch.cuda.synchronize()
    a64, b64 = v64.cpu().numpy(), vd.cpu().numpy()
    err64 = {"l2": float(np.linalg.norm(a64 - b64) / np.linalg.norm(b64)),
             "max_over_max": float(np.max(np.abs(a64 - b64)) /
                                   np.max(np.abs(b64)))}
    del v64
    # the FP64-class fused block: one step (dump 0 x all channels) from E
    # (FP64) with the phase formed in FP64, and its channel-0 error against
    # the FP64 direct (DMMA) result
    vb = torch.zeros((nch, nbl, 8), dtype=torch.float64, device="cuda")

    def block64():
        ob.call("oskb_correlate_block_tc64_d", 0, nsrc, nst, 1, nch, Ed, l,
                m, n, I, Q, U, V, uvw_all[0], inv_wl, 0.0, 3e38, vb, None, 0,
                stream)

    block64()
    torch.cuda.synchronize()
    e0.record()
    block64()
    e1.record()
    torch.cuda.synchronize()
    ms_b64 = e0.elapsed_time(e1)
    vb.zero_()
    block64()
    join(0, 0)
    vd.zero_()
    direct(0, 0)
    torch.cuda.synchronize()
    ab, bb = vb[0].cpu().numpy(), vd.cpu().numpy()
    errb = {"l2": float(np.linalg.norm(ab - bb) / np.linalg.norm(bb)),
            "max_over_max": float(np.max(np.abs(ab - bb)) /
                                  np.max(np.abs(bb)))}
    del vb
    # errors of the tensor-core block against the FP64 direct result
    worst_l2, worst_mx, cases = 0.0, 0.0, []
    dumps = (0, cfg.num_times - 1)
    chans = sorted({0, min(7, nch - 1), nch - 1})
    vt = torch.zeros((1, nbl, 8), dtype=torch.float64, device="cuda")
    for d in dumps:
        for c in chans:
            join(d, c)
            vd.zero_()
            direct(d, c)
            vt.zero_()
            ob.call("oskb_correlate_block_tc", 0, nsrc, nst, 1, 1, E, l, m,
                    n, I, Q, U, V, uvw_all[d], inv_wl[c:c + 1], 0.0, 3e38, vt,
                    None, 0, stream)
            torch.cuda.synchronize()
            a = vt[0].cpu().numpy()
            b = vd.cpu().numpy()
            l2 = float(np.linalg.norm(a - b) / np.linalg.norm(b))
            mx = float(np.max(np.abs(a - b)) / np.max(np.abs(b)))
            cases.append({"dump": d, "channel": c, "l2": l2,
                          "max_over_max": mx})
            worst_l2, worst_mx = max(worst_l2, l2), max(worst_mx, mx)
    err = {"l2": worst_l2, "max_over_max": worst_mx, "cases": cases,
           "sample": "worst over dumps %s x channels %s: all 130,816 "
                     "baselines x 4 pols each; reference = FP64 direct "
                     "kernel on the same inputs (E upcast from FP32)"
                     % (list(dumps), chans)}
    del J, K, Ed
    torch.cuda.empty_cache()
    sb = nbl * nsrc
    return {"direct": {"value": sb / (ms_simt * 1e-3) / 1e9, "unit": UNIT,
                       "kernel": "oskb xcorr_direct_kernel<double> (SIMT "
                                 "FP64, the plain direct form; "
                                 "OSKB_XCORR_DMMA=0)",
                       "ms_per_channel": ms_simt},
            "direct_dmma": {"value": sb / (ms_dmma * 1e-3) / 1e9,
                            "unit": UNIT,
                            "kernel": "oskb xcorr_dmma_kernel (FP64 on the "
                                      "tensor pipe, DMMA; the default FP64 "
                                      "point-source kernel)",
                            "ms_per_channel": ms_dmma},
            "tc64": {"value": sb / (ms_tc64 * 1e-3) / 1e9, "unit": UNIT,
                     "kernel": "oskb gemm_l6_kernel (FP64-class: 48-bit "
                               "fixed point in six 8-bit limbs on the "
                               "integer tensor cores, "
                               "oskb_cross_correlate_tc64_d)",
                     "ms_per_channel": ms_tc64,
                     "error_vs_fp64_direct": err64},
            "block64": {"value": sb * nch / (ms_b64 * 1e-3) / 1e9,
                        "unit": UNIT,
                        "kernel": "oskb prep_fused_l6_kernel + "
                                  "gemm_l6_kernel (FP64-class fused block, "
                                  "oskb_correlate_block_tc64_d, E in FP64, "
                                  "FP64 phase)",
                        "ms_per_step": ms_b64,
                        "step": "1 dump x %d channels" % nch,
                        "error_vs_fp64_direct_channel0": errb},
            "err": err}


def run_e2e(args, cfg, ob, torch, E, world, rank):
    """Source-baselines per second through the pipelined host-buffer
    entry point (oskb_tc_plan_*) with page-locked host buffers over the
    whole observation (this rank's share of the dumps): a step is one block
    of 8 dumps x 16 channels (the reference's default block length); every
    block's E and station uvw are uploaded from host memory
    and its visibilities downloaded to host memory inside the timed region,
    the upload of block b + 1 overlapping the correlation of block b. The
    sky is uploaded once per plan, before the timed region (5.6 MB)."""
    import ctypes
    nst, nsrc, nch = cfg.num_st, cfg.num_src, len(cfg.freqs_hz)
    nbl = cfg.num_baselines
    nt = 8
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    Eh = E.cpu().pin_memory()
    freqs = np.ascontiguousarray(cfg.freqs_hz, np.float64)
    visb = [torch.empty((nt, nch, nbl, 8), dtype=torch.float64).pin_memory()
            for _ in range(2)]
    # the whole observation: this rank's share of the dumps, in blocks of 8
    nblocks = max(2, -(-cfg.num_times // (nt * world)))
    uvws = [pin(np.stack([cfg.station_uvw((rank + (b * world) * nt + i)
                                          % cfg.num_times)
                          for i in range(nt)])) for b in range(nblocks)]
    lib = ob.load()
    st = ctypes.c_int(0)
    plan = lib.oskb_tc_plan_create(0, nsrc, nst, nt, nch, freqs.ctypes.data,
                                   0.0, 3e38, ctypes.addressof(st))
    if st.value or not plan:
        raise RuntimeError("oskb_tc_plan_create failed: %d" % st.value)
    sky = [np.ascontiguousarray(x) for x in (cfg.l, cfg.m, cfg.n, cfg.I,
                                             cfg.Q, cfg.U, cfg.V)]
    ob.call("oskb_tc_plan_set_sky", plan, *sky)
    # warm-up (allocates the library's workspace)
    ob.call("oskb_tc_plan_enqueue", plan, Eh, uvws[0], visb[0])
    ob.call("oskb_tc_plan_wait", plan)
    t0 = time.perf_counter()
    for b in range(nblocks):
        ob.call("oskb_tc_plan_enqueue", plan, Eh, uvws[b], visb[b % 2])
    ob.call("oskb_tc_plan_wait", plan)
    dt = time.perf_counter() - t0
    lib.oskb_tc_plan_free(plan)
    from oskar_b200.sharding import max_over_ranks
    dt = max_over_ranks(dt)
    sb = nbl * nsrc * nch * nt * nblocks * world
    h2d = Eh.numel() * 4 + nt * 3 * nst * 8
    d2h = visb[0].numel() * 8
    del Eh, visb
    return {"value": sb / dt / 1e9, "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h,
            "step": "one block of 8 dumps x 16 channels via oskb_tc_plan_* "
                    "(host buffers, page-locked; upload of the next block "
                    "overlaps the current block's correlation)",
            "blocks": nblocks, "seconds": dt}


def run_profile_case(args):
    """One small invocation of a single kernel, for ncu captures: inputs
    larger than L2 but a few GB on the device at most, two launches.
      tc_small      the tensor-core contraction (gemm_i8_kernel, the
                    default) and its operand preparation
                    (prep_fused_kernel): 512 stations x
                    20,000 sources x 1 channel, 1/80 of a bench launch;
      tc_wide_small the wide-tile contraction (gemm_wide_kernel, tile
                    shape fixed to 128 x 256): 512 stations x 2,500
                    sources x 8 channels (576 tiles), also 1/80 of a bench
                    launch;
      tc_pair_small the pair-tile contraction (gemm_pair_kernel, 256 x 256
                    tiles on CTA pairs) on the same case (288 pair tiles);
      tc_i8_small   the integer contraction (gemm_i8_kernel, the default)
                    and its operand preparation (prep_fused_i8_kernel):
                    512 stations x 10,000 sources x 4 channels (544 square
                    tiles, 1/40 of a bench launch: enough sources that the
                    amplitude buckets' chunks have their bench-size length);
      direct_small  the FP64 direct cross-correlation: 512 stations x 2,000
                    sources, 1 channel;
      tc64_small    the FP64-class integer contraction (gemm_l6_kernel) and
                    its operand preparation (prep_jones_l6_kernel): 512
                    stations x 10,000 sources, 1 channel (272 tasks of
                    128 x 64, one per tile half);
      beam_small    the fused station beam: 32 stations x 256 dipoles x
                    12,001 directions (FP64);
      block_small   the block correlator with Jones K fused: 256 stations x
                    10,000 sources (30% Gaussian) x 2 channels, bandwidth and
                    time smearing, FP64, seed 4."""
    import torch
    import oskar_b200 as ob
    from oskar_b200 import workloads
    torch.cuda.set_device(0)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    stream = ob.stream_ptr()
    case = args.profile_case
    if case in ("tc_wide_small", "tc_pair_small"):
        os.environ["OSKB_TC_TILE"] = "256" if case == "tc_wide_small" \
            else "512"
    if case in ("tc_small", "tc_wide_small", "tc_pair_small", "tc_i8_small",
                "direct_small", "tc64_small"):
        nsrc = {"tc_small": 20_000, "tc_wide_small": 2_500,
                "tc_pair_small": 2_500, "tc_i8_small": 10_000,
                "direct_small": 2_000, "tc64_small": 10_000}[case]
        nch = {"tc_wide_small": 8, "tc_pair_small": 8,
               "tc_i8_small": 4}.get(case, 1)
        cfg = workloads.c3(num_src=nsrc, num_channels=nch, num_times=1)
        nst, nbl = cfg.num_st, cfg.num_baselines
        l, m, n, I, Q, U, V = (dev(x) for x in (cfg.l, cfg.m, cfg.n, cfg.I,
                                                cfg.Q, cfg.U, cfg.V))
        E = workloads.jones_e_device(cfg, torch.float32)
        uvw = dev(cfg.station_uvw(0)[None])
        inv_wl = dev(cfg.freqs_hz / 299792458.0)
        vis = torch.zeros((nch, nbl, 8), dtype=torch.float64, device="cuda")
        if case == "tc64_small":
            f = float(cfg.freqs_hz[0])
            u, v, w = uvw[0]
            K = torch.empty((nst, nsrc, 2), dtype=torch.float64,
                            device="cuda")
            J = torch.empty((nst, nsrc, 8), dtype=torch.float64,
                            device="cuda")
            ob.call("oskb_evaluate_jones_K_d", nsrc, l, m, n, nst, u, v, w,
                    2 * math.pi * f / 299792458.0, I, 0.0, 1e300, 0, K,
                    stream)
            ob.call("oskb_mem_multiply_d", 3, 0, 0, 0, nst * nsrc, K,
                    E.double(), J, stream)
            for _ in range(2):
                ob.call("oskb_cross_correlate_tc64_d", 0, nsrc, nst, 0, J, I,
                        Q, U, V, u, v, 0.0, 3e38, f / 299792458.0, vis[0],
                        None, 0, stream)
        elif case != "direct_small":
            ws_bytes = ob.call("oskb_correlate_block_tc_workspace_bytes",
                               nsrc, nst, nch, check=False)
            ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
            for _ in range(2):
                ob.call("oskb_correlate_block_tc", 0, nsrc, nst, 1, nch, E,
                        l, m, n, I, Q, U, V, uvw, inv_wl, 0.0, 3e38, vis,
                        ws, ws_bytes, stream)
        else:
            f = float(cfg.freqs_hz[0])
            u, v, w = uvw[0]
            K = torch.empty((nst, nsrc, 2), dtype=torch.float64,
                            device="cuda")
            J = torch.empty((nst, nsrc, 8), dtype=torch.float64,
                            device="cuda")
            z = torch.zeros(nst, dtype=torch.float64, device="cuda")
            ob.call("oskb_evaluate_jones_K_d", nsrc, l, m, n, nst, u, v, w,
                    2 * math.pi * f / 299792458.0, I, 0.0, 1e300, 0, K,
                    stream)
            ob.call("oskb_mem_multiply_d", 3, 0, 0, 0, nst * nsrc, K,
                    E.double(), J, stream)
            for _ in range(2):
                ob.call("oskb_cross_correlate_d", 0, 0, nsrc, nst, 0, J, I,
                        Q, U, V, l, m, n, None, None, None, u, v, w, z, z,
                        0.0, 3e38, f / 299792458.0, 0.0, 0.0, 0.0, 0.0,
                        vis[0], stream)
    elif case == "block_small":
        rng = np.random.default_rng(4)
        nst, nsrc, nch = 256, 10_000, 2
        r = np.sqrt(rng.uniform(0, 1, nsrc)) * math.sin(math.radians(4))
        th = rng.uniform(0, 2 * math.pi, nsrc)
        l, m = r * np.cos(th), r * np.sin(th)
        n = np.sqrt(1 - l * l - m * m)
        I = rng.uniform(0.2, 3.0, nsrc)
        Q, U, V = (I * rng.uniform(-0.1, 0.1, nsrc) for _ in range(3))
        ga, gb, gc = (rng.uniform(1e-8, 5e-7, nsrc) for _ in range(3))
        for g in (ga, gb, gc):
            g[3000:] = 0  # 30% Gaussian, the rest point sources
        E = rng.normal(0, 0.1, (nst, nsrc, 8))
        E[..., 0] += 1
        E[..., 6] += 1
        uvw = rng.uniform(-3e3, 3e3, (1, 3, nst))
        sx, sy = (rng.uniform(-3e3, 3e3, nst) for _ in range(2))
        inv_wl = (100e6 + 1e6 * np.arange(nch)) / 299792458.0
        nbl = nst * (nst - 1) // 2
        vis = torch.zeros(nch * nbl * 8, dtype=torch.float64, device="cuda")
        args_ = [0, nsrc, nst, 1, nch, dev(E), 0] + [dev(a) for a in (
            I, Q, U, V, l, m, n, ga, gb, gc, uvw, sx, sy, inv_wl)] + [
            1e5, 10.0, dev(np.array([0.3])), -0.45, 0.0, 3e38, 0, 0.0, 3e38,
            vis, stream]
        os.environ["OSKB_BLOCK_SCHEDULE"] = "2,0"
        for _ in range(2):
            ob.call("oskb_correlate_block_direct_d", *args_)
    elif case == "beam_small":
        st, ne, nd = 32, 256, 12_001
        rng = np.random.default_rng(2)
        r = 19.0 * np.sqrt(rng.uniform(0, 1, (st, ne)))
        t = rng.uniform(0, 2 * math.pi, (st, ne))
        ex, ey = dev(r * np.cos(t)), dev(r * np.sin(t))
        ez = torch.zeros_like(ex)
        az = rng.uniform(0, 2 * math.pi, nd)
        el = np.arcsin(rng.uniform(0, 1, nd))
        dx, dy, dz = (dev(a) for a in (np.cos(el) * np.sin(az),
                                       np.cos(el) * np.cos(az), np.sin(el)))
        ori = dev(rng.uniform(0, 2 * math.pi, st))
        ori_y = ori + math.pi / 2
        b = dev(np.tile([0.0, 0.0, 1.0], (st, 1)))
        beam = torch.empty((st, nd, 8), dtype=torch.float64, device="cuda")
        for _ in range(2):
            ob.call("oskb_station_beam_aa_d", st, ne, ex, ey, ez, None, None,
                    None, None, ori, ori_y, 1.5, 1, 1, 1, 0, 0, 110e6, b, b,
                    nd, dx, dy, dz, 0, beam, stream)
    torch.cuda.synchronize()
    print(json.dumps({"profile_case": case, "ok": True}))
    return 0


def c2_cpu_sample(cfg, t=0, ch=0, num_beam_st=32, num_corr_src=3000):
    """The reference's own CPU kernels (OpenMP, oracle/_ref) on bounded
    samples of one (dump, channel) of the aperture-array chain: the station
    beam (element pattern, weights, weighted DFT, blanking, final
    normalisation) of num_beam_st stations for every source, and Jones K,
    the join and the cross-correlation of all stations for num_corr_src
    sources. Returns the seconds the whole (dump, channel) would take,
    scaled linearly from the two samples, and the sample description."""
    lib = ref_lib()
    if lib is None:
        raise RuntimeError("oracle/_ref/liboskar_ref.so not built")
    D = ctypes.c_double
    N, S, ne = cfg["num_st"], cfg["num_src"], cfg["num_el"]
    f = float(cfg["freqs"][ch])
    k = 2 * math.pi * f / 299792458.0
    kL = 0.5 * 299792458.0 / f * (math.pi * f / 299792458.0)
    lst = cfg["gast"][t] + cfg["lon"]
    t0 = time.perf_counter()
    for p in range(num_beam_st):
        sl, cl = math.sin(cfg["lat"][p]), math.cos(cfg["lat"][p])
        ha = lst[p] - cfg["ra"]
        x = np.ascontiguousarray(-np.cos(cfg["dec"]) * np.sin(ha))
        y = np.ascontiguousarray(cl * np.sin(cfg["dec"]) -
                                 sl * np.cos(cfg["dec"]) * np.cos(ha))
        z = np.ascontiguousarray(sl * np.sin(cfg["dec"]) +
                                 cl * np.cos(cfg["dec"]) * np.cos(ha))
        hb = lst[p] - cfg["ra0"]
        b = (-math.cos(cfg["dec0"]) * math.sin(hb),
             cl * math.sin(cfg["dec0"]) - sl * math.cos(cfg["dec0"]) *
             math.cos(hb),
             sl * math.sin(cfg["dec0"]) + cl * math.cos(cfg["dec0"]) *
             math.cos(hb))
        X = np.ascontiguousarray(np.append(x, b[0]))
        Y = np.ascontiguousarray(np.append(y, b[1]))
        Z = np.ascontiguousarray(np.append(z, b[2]))
        th, p1, p2 = (np.zeros(S + 2) for _ in range(3))
        lib.ref_enu_to_theta_phi_d(0, S + 1, _p(X), _p(Y), _p(Z), 0,
                                   D(-cfg["orient"][p]),
                                   D(math.pi / 2 - cfg["orient"][p]),
                                   _p(th), _p(p1), _p(p2))
        sig = np.zeros((S + 1) * 8)
        lib.ref_dipole_pattern_d(S + 1, _p(th), _p(p1), _p(p2), D(kL),
                                 D(math.cos(kL)), 0, 0, _p(sig))
        ex = np.ascontiguousarray(cfg["el_x"][p])
        ey = np.ascontiguousarray(cfg["el_y"][p])
        ez = np.zeros(ne)
        w = np.zeros(2 * ne)
        lib.ref_element_weights_dft_d(ne, _p(ex), _p(ey), _p(ez), _p(ez),
                                      D(k), D(b[0]), D(b[1]), D(b[2]), _p(w))
        out = np.zeros((S + 1) * 8)
        types = np.zeros(ne, np.int32)  # one element type
        lib.ref_dftw_d(1, 0, ne, D(k), _p(w), _p(ex), _p(ey), _p(None), 0,
                       S + 1, _p(X), _p(Y), _p(None), _p(types), _p(sig), 1,
                       1, 0, _p(out), D(1.0 / ne))
        lib.ref_blank_below_horizon_d(0, S + 1, _p(Z), 0, _p(out))
        lib.ref_mem_normalise_matrix_d(0, S + 1, _p(out), S)
    t_beam = time.perf_counter() - t0
    ns = num_corr_src
    rng = np.random.default_rng(12)
    E = rng.normal(0, 0.1, (N, ns, 8))
    E[..., 0] += 1
    E[..., 6] += 1
    x, y, z = (np.ascontiguousarray(a) for a in cfg["ecef"])
    ha0 = cfg["gast"][t] - cfg["ra0"]
    u, v, w = (np.zeros(N) for _ in range(3))
    lib.ref_ecef_to_station_uvw_d(N, _p(x), _p(y), _p(z), D(math.sin(ha0)),
                                  D(math.cos(ha0)), D(math.sin(cfg["dec0"])),
                                  D(math.cos(cfg["dec0"])), 0, 0, _p(u),
                                  _p(v), _p(w))
    sl_ = slice(0, ns)
    l, m, n, I, Q, U, V = (np.ascontiguousarray(cfg[c][sl_]) for c in
                           ("l", "m", "n", "I", "Q", "U", "V"))
    K = np.zeros((N, ns, 2))
    J = np.zeros((N, ns, 8))
    nbl = N * (N - 1) // 2
    vis = np.zeros((nbl, 8))
    zeros = np.zeros(N)
    t1 = time.perf_counter()
    lib.ref_jones_k_d(ns, _p(l), _p(m), _p(n), N, _p(u), _p(v), _p(w), D(k),
                      _p(I), D(0.0), D(1e300), 0, _p(K))
    lib.ref_mem_mul_cm_m_d(N * ns, _p(K), _p(E), _p(J))
    lib.oskar_cross_correlate_point_omp_d(
        0, ns, N, 0, _p(J), _p(I), _p(Q), _p(U), _p(V), _p(l), _p(m), _p(n),
        _p(u), _p(v), _p(w), _p(zeros), _p(zeros), D(0.0), D(3e38),
        D(f / 299792458.0), D(0.0), D(0.0), D(0.0), D(0.0), _p(vis))
    t_corr = time.perf_counter() - t1
    est = t_beam * N / num_beam_st + t_corr * S / ns
    return est, ("1 dump x 1 channel: station beams of %d of %d stations x "
                 "%d sources (%.1f s) and K + join + correlation of %d "
                 "stations x %d of %d sources (%.1f s), scaled linearly"
                 % (num_beam_st, N, S, t_beam, N, ns, S, t_corr))


def run_c2(args):
    """Aperture-array chain per dump: ENU directions of every source at
    every station, station beams (256 dipoles), Jones R, E R, Jones K,
    J = K (E R), cross-correlation, for 4 channels; 128 stations, 12,000
    sources, FP64. Prints one JSON line: source-baselines/s through the
    chain, the station-beam kernel's share and element-directions/s, and
    the reference's CPU kernels on the host cores beside it."""
    import torch
    import oskar_b200 as ob
    from oskar_b200 import workloads
    torch.cuda.set_device(0)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    cfg = workloads.c2()
    N, S, ne = cfg["num_st"], cfg["num_src"], cfg["num_el"]
    C = len(cfg["freqs"])
    nbl = N * (N - 1) // 2
    st = ob.stream_ptr()
    d = {k: dev(cfg[k]) for k in ("ra", "dec", "l", "m", "n", "I", "Q", "U",
                                  "V", "lat", "el_x", "el_y", "orient")}
    ex, ey, ez = (dev(cfg[k][i]) for k, i in (("ecef", 0), ("ecef", 1),
                                              ("ecef", 2)))
    el_z = torch.zeros_like(d["el_x"])
    f64 = torch.float64
    X, Y, Z = (torch.empty((N, S), dtype=f64, device="cuda")
               for _ in range(3))
    BX, BY, BZ = (torch.empty((N, 1), dtype=f64, device="cuda")
                  for _ in range(3))
    u, v, w = (torch.empty(N, dtype=f64, device="cuda") for _ in range(3))
    E = torch.empty((N, S, 8), dtype=f64, device="cuda")
    R = torch.empty_like(E)
    K = torch.empty((N, S, 2), dtype=f64, device="cuda")
    vis = torch.zeros((C, nbl, 8), dtype=f64, device="cuda")
    ra0 = dev(np.array([cfg["ra0"]]))
    dec0 = dev(np.array([cfg["dec0"]]))
    beam_events = []

    def step(t):
        lst = d["lat"].new_tensor(cfg["gast"][t] + cfg["lon"])
        ob.call("oskb_convert_ra_dec_to_enu_directions_d", S, d["ra"],
                d["dec"], N, lst, d["lat"], X, Y, Z, st)
        ob.call("oskb_convert_ra_dec_to_enu_directions_d", 1, ra0, dec0, N,
                lst, d["lat"], BX, BY, BZ, st)
        benu = torch.cat([BX, BY, BZ], 1).contiguous()
        ob.call("oskb_convert_ecef_to_station_uvw_d", N, ex, ey, ez,
                cfg["ra0"], cfg["dec0"], float(cfg["gast"][t]), 0, 0, u, v,
                w, st)
        ob.call("oskb_evaluate_jones_R_d", S, d["ra"], d["dec"], N,
                d["lat"], lst, R, st)
        vis.zero_()
        for c in range(C):
            f = float(cfg["freqs"][c])
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            ob.call("oskb_station_beam_aa_d", N, ne, d["el_x"], d["el_y"],
                    el_z, None, None, None, None, d["orient"], d["orient"],
                    0.5 * 299792458.0 / f, 0, 1, 1, 0, 0, f, benu, benu, S,
                    X, Y, Z, 1, E, st)
            e1.record()
            beam_events.append((e0, e1))
            ob.call("oskb_mem_multiply_d", 5, 0, 0, 0, N * S, E, R, E, st)
            ob.call("oskb_evaluate_jones_K_d", S, d["l"], d["m"], d["n"], N,
                    u, v, w, 2 * math.pi * f / 299792458.0, d["I"], 0.0,
                    1e300, 0, K, st)
            ob.call("oskb_mem_multiply_d", 3, 0, 0, 0, N * S, K, E, E, st)
            ob.call("oskb_cross_correlate_d", 0, 0, S, N, 0, E, d["I"],
                    d["Q"], d["U"], d["V"], d["l"], d["m"], d["n"], None,
                    None, None, u, v, w, None, None, 0.0, 3e38,
                    f / 299792458.0, 0.0, 0.0, 0.0, 0.0, vis[c], st)

    for i in range(args.warmup):
        step(i % cfg["num_times"])
    torch.cuda.synchronize()
    beam_events.clear()
    clocks = ClockSampler(0)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for i in range(args.steps):
        step((args.warmup + i) % cfg["num_times"])
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps
    beam_ms = sum(a.elapsed_time(b) for a, b in beam_events) / args.steps
    sb = nbl * S * C
    eldir = N * S * ne * C
    est, sample = c2_cpu_sample(cfg)
    cpu = sb / C / est / 1e9
    print(json.dumps({
        "workload": "c2: 128 aperture-array stations (256 dipoles each, "
                    "38 m), 12,000 sources (10,000 in a 10 deg field + "
                    "2,000 anywhere above the horizon), 4 channels "
                    "100-130 MHz, 32 dumps; step = 1 dump x 4 channels of "
                    "ENU directions -> beam -> R -> E R -> K -> J -> "
                    "cross-correlation, FP64",
        "metric": "G source-baselines/s through the aperture-array chain",
        "value": sb / (ms * 1e-3) / 1e9, "unit": "G source-baselines/s",
        "ms_per_step": ms, "steps": args.steps, "warmup": args.warmup,
        "dtype": "f64",
        "station_beam": {"ms_per_step": beam_ms,
                         "share_of_step": beam_ms / ms,
                         "G_element_directions_per_s":
                             eldir / (beam_ms * 1e-3) / 1e9},
        "cpu_baseline": {"value": cpu, "unit": "G source-baselines/s",
                         "cores": cpu_cores(), "kind": "reference",
                         "sample": sample},
        "clocks": clk,
    }))
    return 0


def c4_sky(rng, num_chunks=32):
    """Sky of the batched-smearing configuration: chunk sizes log-uniform on
    [500, 50,000] sources; 30 % of sources Gaussian (FWHM major and minor
    uniform in [1, 60] arcsec, position angle uniform in [0, pi)), the rest
    points; a chunk holding any Gaussian is a Gaussian chunk, as the
    reference groups its sky (oskar_sky_append_to_set.c:119), and its point
    sources have a = b = c = 0. Gaussian coefficients as the reference forms
    them (sky/src/oskar_sky_evaluate_gaussian_source_parameters.c:171-178:
    0.5 FWHM^2 pi^2 / (2 ln 2) along each axis, rotated by the angle)."""
    sizes = np.exp(rng.uniform(math.log(500), math.log(50_000),
                               num_chunks)).astype(int)
    ns = int(sizes.sum())
    r = np.sqrt(rng.uniform(0, 1, ns)) * math.sin(math.radians(5))
    th = rng.uniform(0, 2 * math.pi, ns)
    l, m = r * np.cos(th), r * np.sin(th)
    n = np.sqrt(1 - l * l - m * m)
    I = np.exp(rng.uniform(math.log(0.01), math.log(10.0), ns))
    Q, U, V = (I * rng.uniform(-0.1, 0.1, ns) for _ in range(3))
    gauss = rng.uniform(0, 1, ns) < 0.3
    arcsec = math.pi / 180 / 3600
    maj = rng.uniform(1, 60, ns) * arcsec
    mnr = np.minimum(maj, rng.uniform(1, 60, ns) * arcsec)
    pa = rng.uniform(0, math.pi, ns)
    k = math.pi ** 2 / (2 * math.log(2))
    imaj, imin = 0.5 * maj ** 2 * k, 0.5 * mnr ** 2 * k
    cp2, sp2, s2p = np.cos(pa) ** 2, np.sin(pa) ** 2, np.sin(2 * pa)
    a = cp2 * imin + sp2 * imaj
    b = -s2p * imin * 0.5 + s2p * imaj * 0.5
    c = sp2 * imin + cp2 * imaj
    for g in (a, b, c):
        g[~gauss] = 0.0
    return sizes, dict(l=l, m=m, n=n, I=I, Q=Q, U=U, V=V, a=a, b=b, c=c)


def run_c4(args):
    """Batched blocks with smearing at the configuration's full shape: 256
    stations (32,640 baselines), the whole sky in 32 uneven chunks
    (log-uniform 500-50,000 sources, 30 % Gaussian), 64 channels of
    100 kHz, 10 s time averaging, bandwidth and time smearing, FP64 E per
    station-source. A step is one dump x 64 channels x every chunk through
    the block plan (one CUDA graph per block: upload, clear, one persistent
    launch with K fused, download). The reference's OpenMP
    Gaussian/smearing kernel is timed on a bounded sample beside it."""
    import ctypes
    import torch
    import oskar_b200 as ob
    from oskar_b200 import workloads
    torch.cuda.set_device(0)
    rng = np.random.default_rng(4)
    st = workloads.c3(num_src=1, num_st=256, num_channels=1, num_times=16)
    sizes, sky = c4_sky(rng)
    ns = int(np.sum(sizes))
    sky = {k: np.ascontiguousarray(v) for k, v in sky.items()}
    N, C, T = st.num_st, 64, 1
    nbl = N * (N - 1) // 2
    freqs = 100e6 + 1e5 * np.arange(C)
    x, y = (np.ascontiguousarray(a) for a in st.ecef[:2])
    E = rng.standard_normal((N, ns, 8))
    E *= 0.1
    E[..., 0] += 1
    E[..., 6] += 1
    lib = ob.load()
    status = ctypes.c_int(0)
    plan = lib.oskb_block_plan_create(8, 0, N, ns, T, C, 1, 1, 0,
                                      freqs.ctypes.data, 1e5, 10.0,
                                      st.dec0, 0.0, 3e38, 0, 0.0, 3e38,
                                      ctypes.addressof(status))
    if status.value or not plan:
        raise RuntimeError("oskb_block_plan_create failed")
    ob.call("oskb_block_plan_set_sky", plan, *[sky[k] for k in
                                               "I Q U V l m n a b c".split()])
    ob.call("oskb_block_plan_set_stations", plan, x, y)
    ob.call("oskb_block_plan_set_beam", plan, E)

    def host(ptr, count, dtype=np.float64):
        buf = (ctypes.c_double * count).from_address(ptr)
        return np.frombuffer(buf, dtype=dtype)
    uvw_h = host(lib.oskb_block_plan_host_uvw(plan), T * 3 * N)
    gha_h = host(lib.oskb_block_plan_host_gha0(plan), T)

    def block(t):
        uvw_h[:] = st.station_uvw(t).ravel()
        gha_h[:] = [st.gast(t) - st.ra0]
        ob.call("oskb_block_plan_execute", plan)
        ob.call("oskb_block_plan_synchronize", plan)
    for i in range(args.warmup):
        block(i % st.num_times)
    clocks = ClockSampler(0)
    clocks.start()
    t0 = time.perf_counter()
    for i in range(args.steps):
        block((args.warmup + i) % st.num_times)
    dt = (time.perf_counter() - t0) / args.steps
    clk = clocks.stop()
    graphs = lib.oskb_block_plan_graph_launches(plan)
    buf = ctypes.create_string_buffer(4096)
    ob.call("oskb_block_tune_report", ctypes.addressof(buf), 4096,
            check=False)
    lib.oskb_block_plan_free(plan)
    work = nbl * ns * C * T
    # reference CPU: Gaussian + bandwidth + time smearing, one channel
    nc = 200
    ref = ref_lib()
    cpu = None
    if ref is not None:
        D = ctypes.c_double
        u, v, w = (np.ascontiguousarray(a) for a in st.station_uvw(0))
        J = np.ascontiguousarray(E[:, :nc].reshape(N, nc, 8))
        vis = np.zeros((nbl, 8))
        cs = {k: np.ascontiguousarray(sky[k][:nc]) for k in sky}
        t1 = time.perf_counter()
        ref.oskar_cross_correlate_gaussian_omp_d(
            0, nc, N, 0, _p(J), _p(cs["I"]), _p(cs["Q"]), _p(cs["U"]),
            _p(cs["V"]), _p(cs["l"]), _p(cs["m"]), _p(cs["n"]), _p(cs["a"]),
            _p(cs["b"]), _p(cs["c"]), _p(u), _p(v), _p(w), _p(x), _p(y),
            D(0.0), D(3e38), D(freqs[0] / 299792458.0), D(1e5 / freqs[0]),
            D(10.0), D(st.gast(0) - st.ra0), D(st.dec0), _p(vis))
        cpu = nbl * nc / (time.perf_counter() - t1) / 1e9
    print(json.dumps({
        "workload": "c4: 256 stations, %d sources in 32 uneven chunks "
                    "(log-uniform 500-50,000; 30%% Gaussian), 1 dump x %d "
                    "channels of 100 kHz per step, 10 s averaging, "
                    "bandwidth and time smearing, FP64 E per station-source"
                    % (ns, C),
        "metric": "G source-baselines/s through the block plan",
        "value": work / dt / 1e9, "unit": "G source-baselines/s",
        "ms_per_step": dt * 1e3, "steps": args.steps, "warmup": args.warmup,
        "source_baselines_per_step": work, "graph_replays": graphs,
        "schedule": buf.value.decode().strip(), "clocks": clk,
        "timing": "host wall clock around execute + synchronize of each "
                  "block (graph replay: upload of uvw and hour angle, clear, "
                  "one launch, download of 134 MB of visibilities)",
        "cpu_baseline": {"value": cpu, "unit": "G source-baselines/s",
                         "cores": cpu_cores(), "kind": "reference",
                         "sample": "oskar_cross_correlate_gaussian_omp_d "
                                   "with both smearings, 1 channel x %d "
                                   "sources x %d baselines" % (nc, nbl)},
    }))
    return 0


def run_c5(args):
    """Learned station-beam surrogate against the exact station beam, one
    step = the Jones E of every station for every source at one (dump,
    channel): 512 stations built from 3 planar layouts of 256 dipoles in a
    38 m disc, each station a layout rotated by a random angle, 200,000
    sources of which ~90% lie outside the first null of the main lobe,
    100 MHz. Prints one JSON line: exact and surrogate throughput
    (station-source beam values per second), the audit record, the beam
    error over the whole step and the visibility error it causes (FP64
    correlation of 32 stations with either beam)."""
    import torch
    import oskar_b200 as ob
    from oskar_b200.surrogate import BeamSurrogate, first_null_kappa
    torch.cuda.set_device(0)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    rng = np.random.default_rng(5)
    ns, ne, nsrc, freq = 512, 256, 200_000, 100e6
    layouts = []
    for _ in range(3):
        r = 19.0 * np.sqrt(rng.uniform(0, 1, ne))
        t = rng.uniform(0, 2 * math.pi, ne)
        layouts.append((r * np.cos(t), r * np.sin(t)))
    types = np.arange(ns) % 3
    rot = rng.uniform(0, 2 * math.pi, ns)
    # pointing: 60 deg elevation; sources: 10% within the main lobe
    b = np.array([0.0, math.cos(math.radians(60)), math.sin(math.radians(60))])
    null = first_null_kappa(38.0) / (2 * math.pi * freq / 299792458.0)
    n_in = nsrc // 10
    rr = null * np.sqrt(rng.uniform(0, 1, n_in))
    th = rng.uniform(0, 2 * math.pi, n_in)
    xi, yi = b[0] + rr * np.cos(th), b[1] + rr * np.sin(th)
    az = rng.uniform(0, 2 * math.pi, nsrc - n_in)
    el = np.arcsin(rng.uniform(0, 1, nsrc - n_in))
    xo, yo = np.cos(el) * np.sin(az), np.cos(el) * np.cos(az)
    x = np.concatenate([xi, xo]); y = np.concatenate([yi, yo])
    z = np.sqrt(np.maximum(0.0, 1 - x * x - y * y))
    outside = (np.hypot(x - b[0], y - b[1]) > null).mean()
    dirs = [torch.from_numpy(a.astype(np.float32)).cuda() for a in (x, y, z)]
    dirs_st = [d.unsqueeze(0).expand(ns, nsrc).contiguous() for d in dirs]
    bb = dev(np.tile(b, (ns, 1)))
    d_rot = dev(rot)
    # exact beam: rotated layouts per station
    ex = np.zeros((ns, ne), np.float32); ey = np.zeros_like(ex)
    for s in range(ns):
        lx, ly = layouts[types[s]]
        co, si = math.cos(rot[s]), math.sin(rot[s])
        ex[s] = co * lx - si * ly
        ey[s] = si * lx + co * ly
    d_ex, d_ey, d_ez = dev(ex), dev(ey), dev(np.zeros_like(ex))
    E_exact = torch.empty((ns, nsrc, 8), dtype=torch.float32, device="cuda")

    def exact():
        ob.call("oskb_station_beam_aa_f", ns, ne, d_ex, d_ey, d_ez, None,
                None, None, None, d_rot, d_rot, 1.5, 0, 1, 1, 0, 0, freq, bb,
                bb, nsrc, *dirs, 0, E_exact, ob.stream_ptr())

    sur = BeamSurrogate(layouts, freq, seed=5)
    t0 = time.perf_counter()
    train = sur.train(num_samples=1_000_000, steps=args.c5_steps,
                      batch=4096, lr=1e-4, report_every=1000, seed=5)
    train_s = time.perf_counter() - t0
    E_sur = torch.empty_like(E_exact)
    audit = {}

    def surrogate():
        _, a = sur.beam(types, d_rot, bb, *dirs_st, freq, audit_stride=100,
                        audit_bound=args.c5_bound, out=E_sur)
        audit.update(a)

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    ms_exact = timed(exact, 3)
    ms_sur = timed(surrogate, 3)
    d = (E_sur - E_exact).float()
    beam_max = d.abs().max().item()
    beam_rms = d.pow(2).mean().sqrt().item()
    # visibility error: 32 stations, FP64 direct correlation of either beam
    nv = 32
    rng2 = np.random.default_rng(6)
    I = 10 ** rng2.uniform(-2, 1, nsrc)
    zeros = np.zeros(nsrc)
    lmn = [dev(x), dev(y), dev(z)]
    uvw = [dev(rng2.uniform(-2e3, 2e3, nv)) for _ in range(3)]
    vis = []
    for E in (E_exact, E_sur):
        J = E[:nv].double().contiguous()
        v = torch.zeros((nv * (nv - 1) // 2, 8), dtype=torch.float64,
                        device="cuda")
        ob.call("oskb_cross_correlate_d", 0, 0, nsrc, nv, 0, J, dev(I),
                dev(zeros), dev(zeros), dev(zeros), *[a.double() for a in
                lmn], None, None, None, *uvw, None, None, 0.0, 3e38,
                freq / 299792458.0, 0.0, 0.0, 0.0, 0.0, v, ob.stream_ptr())
        vis.append(v)
    torch.cuda.synchronize()
    vd = vis[1] - vis[0]
    vis_l2 = (vd.norm() / vis[0].norm()).item()
    vis_max = (vd.abs().max() / vis[0].abs().max()).item()
    n_vals = ns * nsrc
    print(json.dumps({
        "workload": "c5: learned station-beam surrogate vs exact station "
                    "beam, 512 stations (3 layouts x 256 dipoles, rotated), "
                    "200,000 sources (%.0f%% outside the first null), "
                    "100 MHz, FP32 beams" % (100 * outside),
        "unit": "G station-source beam values/s",
        "exact": {"ms": ms_exact, "value": n_vals / ms_exact / 1e6,
                  "kernel": "oskb station_beam_kernel<float> (256-element "
                            "array factor per value)"},
        "surrogate": {"ms": ms_sur, "value": n_vals / ms_sur / 1e6,
                      "audit": audit, "audit_bound": args.c5_bound},
        "speedup": ms_exact / ms_sur,
        "beam_error_vs_exact": {"max": beam_max, "rms": beam_rms,
                                "note": "beam normalised to 1 at the "
                                        "pointing"},
        "vis_error_vs_exact": {"l2": vis_l2, "max_over_max": vis_max,
                               "sample": "32 stations x 200,000 sources, "
                                         "FP64 correlation"},
        "training": {"seconds_all_types": train_s,
                     "steps": args.c5_steps, "samples_per_type": 1_000_000,
                     "final_loss": [float(t["loss"][-1]) for t in train]},
    }))
    sur.free()
    return 0


def cpu_baseline(cfg):
    cores = cpu_cores()
    if ref_lib() is None:
        return {"value": None, "unit": UNIT, "cores": cores,
                "kind": "reference", "sample": "unavailable: "
                "oracle/_ref/liboskar_ref.so not built"}
    nsrc = calibrate_cpu_sample(cfg, 8.0)
    dt, work = reference_cpu_sample(cfg, nsrc)
    return {"value": work / dt / 1e9, "unit": UNIT, "cores": cores,
            "kind": "reference",
            "sample": "1 dump x 1 channel x %d of 100000 sources x 130816 "
                      "baselines (reference OpenMP Jones K + join + FP64 "
                      "cross-correlation, %.1f s)" % (nsrc, dt)}


def run_dry(args):
    """The multi-rank plumbing of the default workload without a GPU: gloo
    process group, each rank's dumps and host-side inputs for warm-up and
    timed steps, barriers around the timed region and the maximum of the
    ranks' times. No kernel runs, so no throughput is reported."""
    import datetime
    import torch.distributed as dist
    from oskar_b200 import workloads
    from oskar_b200.sharding import max_over_ranks, rank_dump_uvw
    world, rank, _ = dist_setup()
    if world > 1:
        dist.init_process_group("gloo", timeout=datetime.timedelta(
            seconds=60))
    cfg = workloads.c3(num_src=1000)
    rank_dump_uvw(cfg, world, rank, args.warmup)
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    uvw, dumps = rank_dump_uvw(cfg, world, rank, args.steps, args.warmup)
    dt = time.perf_counter() - t0
    if world > 1:
        dist.barrier()
    dt = max_over_ranks(dt)
    all_dumps = [None] * world
    if world > 1:
        dist.all_gather_object(all_dumps, dumps)
    else:
        all_dumps = [dumps]
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": None, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "dry_run": True,
            "scaling": "weak", "host_seconds_max_over_ranks": dt,
            "dumps_per_rank": all_dumps,
            "config": {"workload": "c3 plumbing only (no kernels)",
                       "parallelism": "dumps sharded over %d rank(s)"
                                      % world}}))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--path", default="tc", choices=["tc", "direct"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="c3",
                    choices=["c3", "c2", "c4", "c5"],
                    help="c2: the aperture-array beam chain; c5: the learned "
                         "station-beam surrogate")
    ap.add_argument("--c5-steps", type=int, default=20000)
    ap.add_argument("--c5-bound", type=float, default=1e-4)
    ap.add_argument("--profile-case", default=None,
                    choices=["tc_small", "tc_wide_small", "tc_pair_small",
                             "tc_i8_small", "tc64_small",
                             "direct_small",
                             "beam_small",
                             "block_small"],
                    help="run one small kernel case for an ncu capture")
    ap.add_argument("--dry-run", action="store_true",
                    help="CPU-only check of the multi-rank plumbing (gloo, "
                         "no kernels): rank start-up, dump sharding, the "
                         "host-side inputs of each rank's steps, barriers "
                         "and the max-over-ranks time; prints a JSON line "
                         "with n_gpus and no throughput")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU, started here when no launcher did it
        from oskar_b200.sharding import spawn_ranks
        return spawn_ranks([sys.executable, os.path.abspath(__file__)] +
                           sys.argv[1:], args.gpus)
    if args.dry_run:
        return run_dry(args)
    if args.profile_case:
        return run_profile_case(args)
    if args.workload == "c5":
        return run_c5(args)
    if args.workload == "c2":
        return run_c2(args)
    if args.workload == "c4":
        return run_c4(args)
    os.environ.setdefault("OMP_NUM_THREADS", str(cpu_cores()))
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
