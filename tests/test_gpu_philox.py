"""The device Philox4x32-10 against cuRAND's and against the (CPU-pinned) oracle."""

import ctypes
import os

import numpy
import pytest

from test_philox_cpu import oracle_philox

pytestmark = pytest.mark.gpu
LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "fresnel_b200",
                   "libfrb200.so")


def test_device_philox_matches_curand_and_oracle():
    lib = ctypes.CDLL(LIB)
    rng = numpy.random.default_rng(11)
    n = 4096
    inp = rng.integers(0, 2**32, (n, 6), dtype=numpy.uint64).astype(numpy.uint32)
    inp[0] = 0
    inp[1] = 0xFFFFFFFF
    ours = numpy.zeros((n, 4), numpy.uint32)
    cur = numpy.zeros((n, 4), numpy.uint32)
    P = ctypes.POINTER(ctypes.c_uint32)
    rc = lib.fr_selftest_philox(inp.ctypes.data_as(P), n, ours.ctypes.data_as(P),
                                cur.ctypes.data_as(P))
    assert rc == 0
    numpy.testing.assert_array_equal(ours, cur)
    for i in range(0, n, 97):
        numpy.testing.assert_array_equal(ours[i], oracle_philox(inp[i, :4], inp[i, 4:]))
