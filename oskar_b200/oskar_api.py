"""Python helpers over the OSKAR-named C API (include/oskar_b200_api.h).

They create oskar_Mem / oskar_Jones / oskar_Telescope objects from numpy
arrays and read them back, so that code (and tests) can drive
oskar_cross_correlate and the other functions with the reference's
argument lists. The objects are plain C handles (integers) owned by the
caller; free them with free_mem / free_jones / free_telescope.
"""
import ctypes

import numpy as np

from ._lib import load

OSKAR_CPU, OSKAR_GPU = 0, 1
OSKAR_INT, OSKAR_SINGLE, OSKAR_DOUBLE = 0x02, 0x04, 0x08
OSKAR_COMPLEX, OSKAR_MATRIX = 0x20, 0x40
OSKAR_METRES, OSKAR_WAVELENGTHS = 0, 1
OSKAR_COORDS_RADEC, OSKAR_COORDS_AZEL = 2, 4

_NUMPY = {OSKAR_INT: np.int32, OSKAR_SINGLE: np.float32,
          OSKAR_DOUBLE: np.float64}
_REALS = {0: 1, OSKAR_COMPLEX: 2, OSKAR_COMPLEX | OSKAR_MATRIX: 8}


class OskarError(RuntimeError):
    def __init__(self, where, status):
        super().__init__("%s: OSKAR status %d" % (where, status))
        self.status = status


def status_ptr(st):
    return ctypes.addressof(st)


def check(where, st):
    if st.value != 0:
        raise OskarError(where, st.value)


def reals_per_element(type_code):
    return _REALS[type_code & (OSKAR_COMPLEX | OSKAR_MATRIX)]


def mem_from_numpy(arr, type_code, location=OSKAR_GPU):
    """New oskar_Mem of type_code holding arr (flattened, reals)."""
    lib = load()
    base = _NUMPY[type_code & 0x0F]
    arr = np.ascontiguousarray(arr, dtype=base).ravel()
    n = arr.size // reals_per_element(type_code)
    st = ctypes.c_int(0)
    cpu = lib.oskar_mem_create(type_code, OSKAR_CPU, n, status_ptr(st))
    check("oskar_mem_create", st)
    if n:
        ctypes.memmove(lib.oskar_mem_void(cpu), arr.ctypes.data, arr.nbytes)
    if location == OSKAR_CPU:
        return cpu
    gpu = lib.oskar_mem_create(type_code, location, n, status_ptr(st))
    check("oskar_mem_create", st)
    lib.oskar_mem_copy_contents(gpu, cpu, 0, 0, n, status_ptr(st))
    lib.oskar_mem_free(cpu, status_ptr(st))
    check("oskar_mem_copy_contents", st)
    return gpu


def mem_to_numpy(mem):
    """Copy of an oskar_Mem's contents (reals) as a numpy array."""
    lib = load()
    t = lib.oskar_mem_type(mem)
    n = lib.oskar_mem_length(mem)
    out = np.zeros(n * reals_per_element(t), _NUMPY[t & 0x0F])
    if n == 0:
        return out
    st = ctypes.c_int(0)
    if lib.oskar_mem_location(mem) == OSKAR_CPU:
        ctypes.memmove(out.ctypes.data, lib.oskar_mem_void(mem), out.nbytes)
        return out
    cpu = lib.oskar_mem_create(t, OSKAR_CPU, n, status_ptr(st))
    lib.oskar_mem_copy_contents(cpu, mem, 0, 0, n, status_ptr(st))
    check("oskar_mem_copy_contents", st)
    ctypes.memmove(out.ctypes.data, lib.oskar_mem_void(cpu), out.nbytes)
    lib.oskar_mem_free(cpu, status_ptr(st))
    return out


def free_mem(*mems):
    lib = load()
    st = ctypes.c_int(0)
    for m in mems:
        if m:
            lib.oskar_mem_free(m, status_ptr(st))


def jones_from_numpy(arr, type_code, num_stations, num_sources,
                     location=OSKAR_GPU):
    """New oskar_Jones [station][source] filled from arr."""
    lib = load()
    st = ctypes.c_int(0)
    j = lib.oskar_jones_create(type_code, location, num_stations,
                               num_sources, status_ptr(st))
    check("oskar_jones_create", st)
    src = mem_from_numpy(arr, type_code, OSKAR_CPU)
    lib.oskar_mem_copy_contents(lib.oskar_jones_mem(j), src, 0, 0,
                                num_stations * num_sources, status_ptr(st))
    free_mem(src)
    check("oskar_mem_copy_contents", st)
    return j


def free_jones(*js):
    lib = load()
    st = ctypes.c_int(0)
    for j in js:
        if j:
            lib.oskar_jones_free(j, status_ptr(st))


def telescope(precision, location, station_x, station_y, station_z=None):
    """oskar_Telescope with the given true ECEF station offsets (metres)."""
    lib = load()
    st = ctypes.c_int(0)
    n = len(station_x)
    t = lib.oskar_telescope_create(precision, location, n, status_ptr(st))
    check("oskar_telescope_create", st)
    cols = [station_x, station_y,
            station_z if station_z is not None else np.zeros(n)]
    for dim, col in enumerate(cols):
        src = mem_from_numpy(col, precision, OSKAR_CPU)
        lib.oskar_mem_copy_contents(
            lib.oskar_telescope_station_true_offset_ecef_metres(t, dim), src,
            0, 0, n, status_ptr(st))
        free_mem(src)
    check("oskar_mem_copy_contents", st)
    return t


def free_telescope(*ts):
    lib = load()
    st = ctypes.c_int(0)
    for t in ts:
        if t:
            lib.oskar_telescope_free(t, status_ptr(st))


def mem_array(*mems):
    """A C array of oskar_Mem* (for src_flux[4], src_dir[3], ...)."""
    return (ctypes.c_void_p * len(mems))(*mems)
