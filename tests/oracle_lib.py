"""ctypes access to the CPU oracle and to the reference's own CPU kernels.

Test infrastructure only. ``oracle()`` loads oracle/_build/liboskar_oracle.so
(the C restatement of the reference kernels); ``reference()`` loads
oracle/_ref/liboskar_ref.so (the reference's kernels compiled from its own
sources by ``make -C oracle ref``), or returns None where it was not built.
Both are plain C libraries; every array argument is a contiguous numpy array.
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "_build", "liboskar_oracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "liboskar_ref.so")

_cache = {}


def _ensure(path, target):
    """Builds a missing oracle library; the ref* targets also need the
    reference's source directory in OSKB_REF_SRC (otherwise they are left
    unbuilt and the caller skips)."""
    if not os.path.exists(path):
        cmd = ["make", "-s", "-C", os.path.join(ROOT, "oracle"), target]
        if os.environ.get("OSKB_REF_SRC"):
            cmd.insert(3, "REF_SRC=" + os.environ["OSKB_REF_SRC"])
        subprocess.run(cmd, check=False, capture_output=True)
    return os.path.exists(path)


class _Lib:
    """Wraps a library whose functions take (int | real | pointer) args."""

    def __init__(self, path, prefix):
        self.lib = ctypes.CDLL(path)
        self.prefix = prefix

    def call(self, name, real, *args):
        fn = getattr(self.lib, self.prefix + name)
        cargs = []
        for a in args:
            if a is None:
                cargs.append(ctypes.c_void_p(0))
            elif isinstance(a, np.ndarray):
                assert a.flags.c_contiguous, name
                cargs.append(ctypes.c_void_p(a.ctypes.data))
            elif isinstance(a, (bool, int, np.integer)):
                cargs.append(ctypes.c_int(int(a)))
            elif isinstance(a, (float, np.floating)):
                cargs.append(ctypes.c_double(a) if real == np.float64
                             else ctypes.c_float(a))
            else:
                raise TypeError(f"{name}: unsupported arg {type(a)}")
        fn.restype = None
        fn(*cargs)


def oracle():
    if "oracle" not in _cache:
        if not _ensure(ORACLE_SO, "all"):
            raise RuntimeError("oracle library not built: make -C oracle")
        _cache["oracle"] = _Lib(ORACLE_SO, "orc_")
    return _cache["oracle"]


def reference():
    if "ref" not in _cache:
        _cache["ref"] = (_Lib(REF_SO, "ref_")
                         if _ensure(REF_SO, "ref") else None)
    return _cache["ref"]


def reference_xcorr(real, matrix, gaussian, *args):
    """Calls the reference's exported oskar_cross_correlate_*_omp_{f,d}.

    ``args`` are the oracle's xcorr arguments after ``gaussian``:
    (num_src, num_st, offset_out, jones, I, Q, U, V, l, m, n, a, b, c,
     st_u, st_v, st_w, st_x, st_y, uv_min, uv_max, inv_wavelength,
     frac_bandwidth, time_int_sec, gha0, dec0, vis) plus ``casa`` first.
    """
    ref = reference()
    casa, rest = args[0], list(args[1:])
    s = "d" if real == np.float64 else "f"
    kind = "gaussian" if gaussian else "point"
    name = ("oskar_cross_correlate_" + ("" if matrix else "scalar_") + kind
            + "_omp_" + s)
    if not gaussian:
        del rest[11:14]  # the point kernels take no a, b, c
    if not matrix:
        del rest[5:8]  # the scalar kernels take Stokes I only
    fn = getattr(ref.lib, name)
    cargs = [ctypes.c_int(casa)]
    for a in rest:
        if a is None:
            cargs.append(ctypes.c_void_p(0))
        elif isinstance(a, np.ndarray):
            cargs.append(ctypes.c_void_p(a.ctypes.data))
        elif isinstance(a, (bool, int, np.integer)):
            cargs.append(ctypes.c_int(int(a)))
        else:
            cargs.append(ctypes.c_double(a) if real == np.float64
                         else ctypes.c_float(a))
    fn.restype = None
    fn(*cargs)


def suffix(real):
    return "d" if real == np.float64 else "f"


REF_CUDA_SO = os.path.join(ROOT, "oracle", "_ref", "liboskar_ref_cuda.so")


def reference_cuda():
    """The reference's own CUDA cross-correlation kernels compiled from its
    sources (``make -C oracle ref_cuda``), or None where not built."""
    if "ref_cuda" not in _cache:
        _cache["ref_cuda"] = (ctypes.CDLL(REF_CUDA_SO)
                              if os.path.exists(REF_CUDA_SO) else None)
    return _cache["ref_cuda"]


def reference_cuda_xcorr(real, matrix, gaussian, casa, num_src, num_st,
                         offset_out, jones, I, Q, U, V, l, m, n, a, b, c,
                         st_u, st_v, st_w, st_x, st_y, uv_min, uv_max,
                         inv_wavelength, frac_bandwidth, time_int_sec, gha0,
                         dec0, vis):
    """Calls oskar_cross_correlate_[scalar_]{point,gaussian}_cuda_{f,d}
    (correlate/oskar_cross_correlate_cuda.h, _scalar_cuda.h) with device
    pointers (ints) and host scalars; launches on the legacy stream."""
    lib = reference_cuda()
    s = "d" if real == np.float64 else "f"
    kind = "gaussian" if gaussian else "point"
    fn = getattr(lib, "oskar_cross_correlate_" + ("" if matrix else
                                                 "scalar_") + kind
                 + "_cuda_" + s)
    fp = ctypes.c_double if real == np.float64 else ctypes.c_float
    p = lambda x: ctypes.c_void_p(x)
    args = [ctypes.c_int(casa), ctypes.c_int(num_src), ctypes.c_int(num_st),
            ctypes.c_int(offset_out), p(jones), p(I)]
    if matrix:
        args += [p(Q), p(U), p(V)]
    args += [p(l), p(m), p(n)]
    if gaussian:
        args += [p(a), p(b), p(c)]
    args += [p(st_u), p(st_v), p(st_w), p(st_x), p(st_y)]
    args += [fp(x) for x in (uv_min, uv_max, inv_wavelength, frac_bandwidth,
                             time_int_sec, gha0, dec0)]
    args.append(p(vis))
    fn.restype = None
    fn(*args)
