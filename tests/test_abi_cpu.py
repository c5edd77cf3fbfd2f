"""The C ABI library loads on a CPU-only machine and exports every entry point declared in
include/fresnel_b200.h; calls that need no GPU behave as documented."""

import ctypes
import os
import re

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "fresnel_b200.h")
LIB = os.path.join(REPO, "fresnel_b200", "libfrb200.so")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"FR_API\s+[\w\s\*]+?\b(fr_\w+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    names = declared()
    assert len(names) >= 30
    lib = ctypes.CDLL(LIB)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_calls_without_a_gpu():
    lib = ctypes.CDLL(LIB)
    lib.fr_last_error.restype = ctypes.c_char_p
    assert lib.fr_abi_version() == 1
    n = ctypes.c_int(-1)
    assert lib.fr_get_num_available_devices(ctypes.byref(n)) == 0
    assert n.value >= 0
    if n.value == 0:
        dev = ctypes.c_void_p()
        assert lib.fr_device_create(-1, ctypes.byref(dev)) == 6  # FR_ERR_UNSUPPORTED
        assert b"No GPUs" in lib.fr_last_error()
    buf = ctypes.create_string_buffer(1024)
    assert lib.fr_get_all_gpus(buf, 1024) == 0
    # null handles are rejected, not dereferenced
    assert lib.fr_tracer_render_path(None, None, None, 1, 1, 1) == 1
    assert b"must not be null" in lib.fr_last_error()
    assert lib.fr_geometry_write(None, 0, None, 0, 0) == 1
