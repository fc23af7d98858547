"""Builds liboskar_b200.so (all CUDA sources, sm_100a) in-tree, and the
drop-in liboskar_b200_dropin.so.

Usage: python -m oskar_b200.build [--verbose-ptxas]
The libraries land next to this file; objects go to oskar_b200/_build/.
Rebuilds only when a source or header is newer than a library.

liboskar_b200_dropin.so holds the same kernels and oskb_* entry points plus
csrc/dropin/ (oskar_interferometer_run_block for an unmodified reference
liboskar), and leaves out the OSKAR-named container layer of oskar_api.cu:
its oskar_mem_* and oskar_jones_* functions would otherwise take the place
of the reference's own when the drop-in is loaded ahead of liboskar. The
reference functions the drop-in calls stay undefined until that liboskar is
loaded next to it.
"""
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liboskar_b200.so")
DROPIN_LIB = os.path.join(HERE, "liboskar_b200_dropin.so")
DROPIN = os.path.join(CSRC, "dropin")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
         "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _dropin_sources():
    return sorted(glob.glob(os.path.join(DROPIN, "*.cu")))


def _deps():
    return (_sources() + _dropin_sources() +
            glob.glob(os.path.join(CSRC, "*.cuh")) +
            glob.glob(os.path.join(DROPIN, "*.h")) +
            glob.glob(os.path.join(ROOT, "include", "*.h")))


def needs_build():
    for lib in (LIB, DROPIN_LIB):
        if not os.path.exists(lib):
            return True
        t = os.path.getmtime(lib)
        if any(os.path.getmtime(f) > t for f in _deps()):
            return True
    return False


def _compile(src, verbose_ptxas):
    name = os.path.basename(src)
    if os.path.dirname(src) == DROPIN:
        name = "dropin_" + name
    obj = os.path.join(BUILD, name + ".o")
    cmd = [NVCC, *ARCH, *FLAGS, "-c", src, "-o", obj]
    if verbose_ptxas:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s%s" % (src, r.stdout,
                                                           r.stderr))
    return obj, r.stderr


def build(force=False, verbose_ptxas=False):
    if not force and not needs_build():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    srcs = _sources() + _dropin_sources()
    with cf.ThreadPoolExecutor(max_workers=8) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose_ptxas), srcs))
    if verbose_ptxas:
        for _, log in results:
            sys.stderr.write(log)
    objs = dict(zip(srcs, [o for o, _ in results]))
    main = [objs[s] for s in _sources()]
    dropin = [objs[s] for s in srcs
              if os.path.basename(s) != "oskar_api.cu"]
    for out, o in ((LIB, main), (DROPIN_LIB, dropin)):
        cmd = [NVCC, *ARCH, "-shared", "-o", out, *o]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s%s" % (r.stdout, r.stderr))
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose_ptxas="--verbose-ptxas" in sys.argv))
