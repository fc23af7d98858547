"""Runs one interferometer simulation through the reference library's own
driver and writes its visibilities to an .npz file (test infrastructure).

    python tests/ref_sim.py case.json out.npz

The reference library is oracle/_ref/liboskar_refcpu.so (the reference's CPU
library compiled from its sources by `make -C oracle ref_lib`). The
simulation goes through the reference's public C API exactly as its
applications use it: a telescope model loaded from a directory written here
(position.txt, layout.txt, one station folder), a sky model filled source by
source, oskar_interferometer_run (worker threads, work-unit claiming, block
finalisation and the .vis writer), then the .vis file read back with the
reference's reader. Started with this repository's
oskar_b200/liboskar_b200_dropin.so in LD_PRELOAD ahead of the reference
library, the same run reaches the B200 oskar_interferometer_run_block
through the reference's own calls; without it, the reference's CPU path
runs. The caller chooses, so the two runs can be compared.

case.json keys (all required):
  precision "double" | "single"; pol_mode "Full" | "Scalar";
  lon_deg, lat_deg; station_x, station_y (ENU metres); station_type
  (e.g. "Isotropic beam"); channel_bandwidth_hz, time_average_sec,
  uv_filter [min, max, "Wavelengths" | "Metres"];
  ra_rad, dec_rad, I, Q, U, V, ref_freq_hz, spectral_index,
  rotation_measure, major_rad, minor_rad, pa_rad (per source);
  phase_centre_ra_rad, phase_centre_dec_rad; freq_start_hz, freq_inc_hz,
  num_channels; mjd_start, inc_sec, num_times; num_devices,
  max_times_per_block, max_sources_per_chunk, horizon_clip,
  correlation_type ("Cross-correlations" | "Auto-correlations" | "Both"),
  casa, source_min_jy, source_max_jy. Optional: station_per_folder (one
  station model per station, station-beam duplication off), element_x and
  element_y (aperture-array element layouts), read_back (default true:
  false skips reading the .vis file back, for timing runs).
The .npz also holds run_seconds, the wall time of oskar_interferometer_run
alone (the simulator's block loop and .vis writer).
"""
import ctypes
import json
import os
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "liboskar_refcpu.so")
DROPIN_LIB = os.path.join(ROOT, "oskar_b200", "liboskar_b200_dropin.so")

OSKAR_SINGLE, OSKAR_DOUBLE, OSKAR_CPU = 4, 8, 0
OSKAR_COORDS_RADEC = 2


def _lib():
    lib = ctypes.CDLL(REF_LIB, mode=ctypes.RTLD_GLOBAL)
    P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    S = ctypes.c_char_p
    IP = ctypes.POINTER(ctypes.c_int)
    sig = {
        "oskar_telescope_create": (P, [I, I, I, IP]),
        "oskar_telescope_set_pol_mode": (None, [P, S, IP]),
        "oskar_telescope_set_allow_station_beam_duplication": (None, [P, I]),
        "oskar_telescope_load": (None, [P, S, P, IP]),
        "oskar_telescope_set_station_type": (None, [P, S, IP]),
        "oskar_telescope_set_phase_centre": (None, [P, I, D, D]),
        "oskar_telescope_set_channel_bandwidth": (None, [P, D]),
        "oskar_telescope_set_time_average": (None, [P, D]),
        "oskar_telescope_set_uv_filter": (None, [P, D, D, S, IP]),
        "oskar_sky_create": (P, [I, I, I, IP]),
        "oskar_sky_set_source": (None, [P, I, D, D, D, D, D, D, D, D, D, D,
                                        D, D, IP]),
        "oskar_interferometer_create": (P, [I, IP]),
        "oskar_interferometer_set_gpus": (None, [P, I, P, IP]),
        "oskar_interferometer_set_num_devices": (None, [P, I]),
        "oskar_interferometer_set_observation_frequency": (None, [P, D, D,
                                                                  I]),
        "oskar_interferometer_set_observation_time": (None, [P, D, D, I]),
        "oskar_interferometer_set_max_times_per_block": (None, [P, I]),
        "oskar_interferometer_set_max_sources_per_chunk": (None, [P, I]),
        "oskar_interferometer_set_horizon_clip": (None, [P, I]),
        "oskar_interferometer_set_correlation_type": (None, [P, S, IP]),
        "oskar_interferometer_set_casa_phase_convention": (None, [P, I]),
        "oskar_interferometer_set_source_flux_range": (None, [P, D, D]),
        "oskar_interferometer_set_sky_model": (None, [P, P, IP]),
        "oskar_interferometer_set_telescope_model": (None, [P, P, IP]),
        "oskar_interferometer_set_output_vis_file": (None, [P, S]),
        "oskar_interferometer_run": (None, [P, IP]),
        "oskar_interferometer_free": (None, [P, IP]),
        "oskar_binary_create": (P, [S, ctypes.c_char, IP]),
        "oskar_binary_free": (None, [P]),
        "oskar_vis_header_read": (P, [P, IP]),
        "oskar_vis_header_num_blocks": (I, [P]),
        "oskar_vis_block_create_from_header": (P, [I, P, IP]),
        "oskar_vis_block_read": (None, [P, P, P, I, IP]),
        "oskar_vis_block_num_times": (I, [P]),
        "oskar_vis_block_num_channels": (I, [P]),
        "oskar_vis_block_cross_correlations_const": (P, [P]),
        "oskar_vis_block_auto_correlations_const": (P, [P]),
        "oskar_vis_block_has_cross_correlations": (I, [P]),
        "oskar_vis_block_has_auto_correlations": (I, [P]),
        "oskar_mem_void_const": (P, [P]),
        "oskar_mem_length": (ctypes.c_size_t, [P]),
        "oskar_mem_type": (I, [P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype, f.argtypes = res, args
    return lib


def _check(st, what):
    if st.value:
        raise RuntimeError("%s: OSKAR status %d" % (what, st.value))


def write_telescope(d, case):
    with open(os.path.join(d, "position.txt"), "w") as f:
        f.write("%.17g,%.17g,0\n" % (case["lon_deg"], case["lat_deg"]))
    with open(os.path.join(d, "layout.txt"), "w") as f:
        for x, y in zip(case["station_x"], case["station_y"]):
            f.write("%.17g,%.17g\n" % (x, y))
    # one station folder shared by all stations, or one per station (each
    # station then has its own model: its own latitude and longitude for
    # Jones R, and its own beam); element layouts (ENU metres) from
    # element_x / element_y: one list for every folder, or one list per
    # folder; a single element at the centre without them
    num = len(case["station_x"]) if case.get("station_per_folder") else 1
    ex, ey = case.get("element_x"), case.get("element_y")
    for i in range(num):
        s = os.path.join(d, "station%04d" % i)
        os.makedirs(s)
        with open(os.path.join(s, "layout.txt"), "w") as f:
            if ex is None:
                f.write("0,0\n")
                continue
            xs = ex[i] if isinstance(ex[0], list) else ex
            ys = ey[i] if isinstance(ey[0], list) else ey
            for x, y in zip(xs, ys):
                f.write("%.17g,%.17g\n" % (x, y))


def mem_array(lib, mem, complex_matrix):
    n = lib.oskar_mem_length(mem)
    typ = lib.oskar_mem_type(mem)
    real = np.float64 if (typ & 0x0F) == OSKAR_DOUBLE else np.float32
    per = (8 if (typ & 0x40) else 2) if (typ & 0x20) else 1
    ptr = lib.oskar_mem_void_const(mem)
    buf = (ctypes.c_char * (n * per * np.dtype(real).itemsize)).from_address(
        ptr)
    return np.frombuffer(bytes(buf), dtype=real).copy()


def run(case, out_path):
    lib = _lib()
    st = ctypes.c_int(0)
    prec = OSKAR_DOUBLE if case["precision"] == "double" else OSKAR_SINGLE
    work = tempfile.mkdtemp(prefix="oskb_refsim_")
    tdir = os.path.join(work, "telescope")
    os.makedirs(tdir)
    write_telescope(tdir, case)
    tel = lib.oskar_telescope_create(prec, OSKAR_CPU, 0, ctypes.byref(st))
    lib.oskar_telescope_set_pol_mode(tel, case["pol_mode"].encode(),
                                     ctypes.byref(st))
    lib.oskar_telescope_set_allow_station_beam_duplication(
        tel, 0 if case.get("station_per_folder") else 1)
    lib.oskar_telescope_load(tel, tdir.encode(), None, ctypes.byref(st))
    _check(st, "telescope load")
    lib.oskar_telescope_set_station_type(tel, case["station_type"].encode(),
                                         ctypes.byref(st))
    lib.oskar_telescope_set_phase_centre(tel, OSKAR_COORDS_RADEC,
                                         case["phase_centre_ra_rad"],
                                         case["phase_centre_dec_rad"])
    lib.oskar_telescope_set_channel_bandwidth(tel,
                                              case["channel_bandwidth_hz"])
    lib.oskar_telescope_set_time_average(tel, case["time_average_sec"])
    uvf = case["uv_filter"]
    lib.oskar_telescope_set_uv_filter(tel, uvf[0], uvf[1], uvf[2].encode(),
                                      ctypes.byref(st))
    _check(st, "telescope set-up")
    nsrc = len(case["I"])
    sky = lib.oskar_sky_create(prec, OSKAR_CPU, nsrc, ctypes.byref(st))
    for i in range(nsrc):
        lib.oskar_sky_set_source(
            sky, i, case["ra_rad"][i], case["dec_rad"][i], case["I"][i],
            case["Q"][i], case["U"][i], case["V"][i], case["ref_freq_hz"][i],
            case["spectral_index"][i], case["rotation_measure"][i],
            case["major_rad"][i], case["minor_rad"][i], case["pa_rad"][i],
            ctypes.byref(st))
    _check(st, "sky set-up")
    h = lib.oskar_interferometer_create(prec, ctypes.byref(st))
    lib.oskar_interferometer_set_gpus(h, 0, None, ctypes.byref(st))
    lib.oskar_interferometer_set_num_devices(h, case["num_devices"])
    lib.oskar_interferometer_set_observation_frequency(
        h, case["freq_start_hz"], case["freq_inc_hz"], case["num_channels"])
    lib.oskar_interferometer_set_observation_time(
        h, case["mjd_start"], case["inc_sec"], case["num_times"])
    lib.oskar_interferometer_set_max_times_per_block(
        h, case["max_times_per_block"])
    lib.oskar_interferometer_set_max_sources_per_chunk(
        h, case["max_sources_per_chunk"])
    lib.oskar_interferometer_set_horizon_clip(h, case["horizon_clip"])
    lib.oskar_interferometer_set_correlation_type(
        h, case["correlation_type"].encode(), ctypes.byref(st))
    lib.oskar_interferometer_set_casa_phase_convention(h, case["casa"])
    lib.oskar_interferometer_set_source_flux_range(
        h, case["source_min_jy"], case["source_max_jy"])
    lib.oskar_interferometer_set_sky_model(h, sky, ctypes.byref(st))
    lib.oskar_interferometer_set_telescope_model(h, tel, ctypes.byref(st))
    vis_path = os.path.join(work, "out.vis")
    lib.oskar_interferometer_set_output_vis_file(h, vis_path.encode())
    _check(st, "simulator set-up")
    t0 = time.perf_counter()
    lib.oskar_interferometer_run(h, ctypes.byref(st))
    run_seconds = time.perf_counter() - t0
    _check(st, "oskar_interferometer_run")
    lib.oskar_interferometer_free(h, ctypes.byref(st))
    if not case.get("read_back", True):
        np.savez(out_path, run_seconds=np.array([run_seconds]),
                 dropin=np.array([DROPIN_LIB in
                                  os.environ.get("LD_PRELOAD", "")]))
        return
    # read the blocks back with the reference's reader
    fb = lib.oskar_binary_create(vis_path.encode(), b"r", ctypes.byref(st))
    hdr = lib.oskar_vis_header_read(fb, ctypes.byref(st))
    _check(st, "vis header read")
    blk = lib.oskar_vis_block_create_from_header(OSKAR_CPU, hdr,
                                                 ctypes.byref(st))
    cross, autos = [], []
    for b in range(lib.oskar_vis_header_num_blocks(hdr)):
        lib.oskar_vis_block_read(blk, hdr, fb, b, ctypes.byref(st))
        _check(st, "vis block read")
        nt = lib.oskar_vis_block_num_times(blk)
        nc = lib.oskar_vis_block_num_channels(blk)
        if lib.oskar_vis_block_has_cross_correlations(blk):
            cross.append(mem_array(
                lib, lib.oskar_vis_block_cross_correlations_const(blk),
                True).reshape(nt, nc, -1))
        if lib.oskar_vis_block_has_auto_correlations(blk):
            autos.append(mem_array(
                lib, lib.oskar_vis_block_auto_correlations_const(blk),
                True).reshape(nt, nc, -1))
    lib.oskar_binary_free(fb)
    out = {}
    if cross:
        out["cross"] = np.concatenate(cross, axis=0)
    if autos:
        out["autos"] = np.concatenate(autos, axis=0)
    out["dropin"] = np.array(
        [DROPIN_LIB in os.environ.get("LD_PRELOAD", "")])
    out["run_seconds"] = np.array([run_seconds])
    np.savez(out_path, **out)


if __name__ == "__main__":
    with open(sys.argv[1]) as f:
        run(json.load(f), sys.argv[2])
