"""CPU checks of the C ABI: the library loads without a GPU and exports every
entry point that include/*.h declares, with the argument types the header
gives. No kernel is launched here."""
import ctypes
import os
import subprocess

import pytest

import oskar_b200
from oskar_b200 import _lib


def test_every_declared_symbol_is_exported():
    lib = _lib.load()
    protos = _lib.parse_headers()
    assert len(protos) >= 17
    for name in protos:
        assert hasattr(lib, name), name
    assert lib.oskb_version().startswith(b"oskar_b200")


def test_nm_matches_header():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH],
                         capture_output=True, text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines()
                if " T " in ln and ln.split()[-1].startswith("oskb_")}
    declared = {k for k in _lib.parse_headers() if k.startswith("oskb_")}
    assert declared <= exported, declared - exported
    # nothing else from the library leaks out under the oskb_ prefix
    assert exported <= declared, exported - declared


def test_oskar_api_symbols_exported():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH],
                         capture_output=True, text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    declared = {k for k in _lib.parse_headers() if k.startswith("oskar_")}
    assert len(declared) >= 30
    assert declared <= exported, declared - exported


def test_header_compiles_as_c():
    inc = os.path.join(_lib.ROOT, "include")
    src = ("#include <oskar_b200.h>\n#include <oskar_b200_api.h>\n"
           "int main(void){return 0;}\n")
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I" + inc,
                        "-x", "c", "-", "-o", os.devnull], input=src,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_argument_count_checked():
    with pytest.raises(TypeError):
        oskar_b200.call("oskb_cross_correlate_d", 1, 2, 3)


def test_last_error_empty_initially():
    assert isinstance(_lib.load().oskb_last_error(), bytes)
