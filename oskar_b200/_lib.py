"""Loads liboskar_b200.so and binds every C entry point declared in
include/*.h through ctypes.

The argument types come from the header prototypes themselves, so the Python
binding and the C ABI cannot drift apart. Pointer arguments accept torch
tensors (their data_ptr()), numpy arrays, raw integers or None. There is no
fallback: if the shared library is missing or fails to load, every call
raises.
"""
import ctypes
import glob
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
# OSKB_LIBRARY selects another build of the same library (same C ABI).
LIB_PATH = os.environ.get("OSKB_LIBRARY",
                          os.path.join(HERE, "liboskar_b200.so"))

_SCALARS = {
    "int": ctypes.c_int,
    "double": ctypes.c_double,
    "float": ctypes.c_float,
    "size_t": ctypes.c_size_t,
    "long long": ctypes.c_longlong,
    "unsigned int": ctypes.c_uint,
    "unsigned long long": ctypes.c_ulonglong,
}


def parse_headers(paths=None):
    """Returns {name: (restype, [argtype, ...])} for the prototypes in the
    public headers."""
    if paths is None:
        paths = sorted(glob.glob(os.path.join(ROOT, "include", "*.h")))
    protos = {}
    for path in paths:
        text = open(path).read()
        text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
        text = re.sub(r"//[^\n]*", " ", text)
        text = re.sub(r"#[^\n]*", " ", text)
        for m in re.finditer(
                r"((?:const\s+)?\w+\s*\**)\s*\b((?:oskb|oskar)_\w+)\s*"
                r"\(([^)]*)\)\s*;", text):
            ret, name, args = " ".join(m.group(1).split()), m.group(2), \
                m.group(3)
            if ret.startswith("typedef") or ret == "struct":
                continue
            argtypes = []
            args = args.strip()
            if args and args != "void":
                for a in args.split(","):
                    a = " ".join(a.split())
                    if "*" in a:
                        argtypes.append(ctypes.c_void_p)
                        continue
                    base = re.sub(r"\bconst\b", "", a).strip()
                    base = " ".join(base.split()[:-1])  # drop the name
                    if base not in _SCALARS:
                        raise ValueError("%s: unsupported type '%s'"
                                         % (name, base))
                    argtypes.append(_SCALARS[base])
            if ret.replace(" ", "") == "constchar*":
                restype = ctypes.c_char_p
            elif "*" in ret:
                restype = ctypes.c_void_p
            else:
                restype = {"int": ctypes.c_int, "void": None,
                           "size_t": ctypes.c_size_t}[ret]
            protos[name] = (restype, argtypes)
    return protos


class OskbError(RuntimeError):
    def __init__(self, name, status, detail):
        super().__init__("%s failed with OSKAR status %d%s" % (
            name, status, (": " + detail) if detail else ""))
        self.status = status


_lib = None
_protos = None


def load():
    global _lib, _protos
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            "liboskar_b200.so not built (python -m oskar_b200.build); the "
            "package has no CPU fallback")
    lib = ctypes.CDLL(LIB_PATH)
    protos = parse_headers()
    for name, (restype, argtypes) in protos.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    _lib, _protos = lib, protos
    return lib


def _ptr(x):
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if hasattr(x, "ctypes"):
        return x.ctypes.data
    raise TypeError("cannot pass %r as a pointer" % type(x))


def call(name, *args, check=True):
    """Calls an oskb_* entry point; tensors/arrays become pointers. Raises
    OskbError on a non-zero status when check is set; returns the status."""
    lib = load()
    restype, argtypes = _protos[name]
    if len(args) != len(argtypes):
        raise TypeError("%s takes %d arguments, got %d"
                        % (name, len(argtypes), len(args)))
    conv = [(_ptr(a) if t is ctypes.c_void_p else a)
            for a, t in zip(args, argtypes)]
    status = getattr(lib, name)(*conv)
    if check and name.startswith("oskb_") and restype is ctypes.c_int \
            and status != 0:
        detail = lib.oskb_last_error().decode()
        raise OskbError(name, status, detail)
    return status


def stream_ptr(stream=None):
    """The raw cudaStream_t of a torch stream (default: current stream)."""
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream
