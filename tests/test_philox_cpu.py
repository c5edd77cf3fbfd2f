"""Philox4x32-10 and u01 (the random numbers behind every sample) on the CPU.

Random123's own known-answer vectors are not in the reference tree (its extern/random123
submodule is empty), so the oracle's generator is checked against an independent
implementation of the same published algorithm: PyTorch's header-only
at::philox_engine (ATen/core/PhiloxRNGEngine.h), compiled here.  With seed = key0 | key1<<32,
subsequence = ctr2 | ctr3<<32 and offset = ctr0 | ctr1<<32, its first four outputs are
Philox4x32-10(ctr, key).  The GPU generator is compared with the same oracle (and with cuRAND)
in tests/test_gpu_philox.py.
"""

import ctypes
import os
import subprocess
import tempfile

import numpy
import pytest

from oracle import cpu_module

TORCH_SRC = r"""
#include <ATen/core/PhiloxRNGEngine.h>
#include <cstdint>
#include <cstdio>
int main() {
    unsigned a, b, c, d, e, f;
    while (std::scanf("%u %u %u %u %u %u", &a, &b, &c, &d, &e, &f) == 6) {
        uint64_t seed = uint64_t(e) | (uint64_t(f) << 32);
        uint64_t sub = uint64_t(c) | (uint64_t(d) << 32);
        uint64_t off = uint64_t(a) | (uint64_t(b) << 32);
        at::philox_engine eng(seed, sub, off);
        unsigned r0 = eng(), r1 = eng(), r2 = eng(), r3 = eng();
        std::printf("%u %u %u %u\n", r0, r1, r2, r3);
    }
    return 0;
}
"""


def _torch_include():
    try:
        import torch
    except Exception:
        return None
    inc = os.path.join(os.path.dirname(torch.__file__), "include")
    return inc if os.path.exists(os.path.join(inc, "ATen/core/PhiloxRNGEngine.h")) else None


def oracle_philox(ctr, key):
    lib = cpu_module.load("restated")
    c = numpy.array(ctr, numpy.uint32)
    k = numpy.array(key, numpy.uint32)
    o = numpy.zeros(4, numpy.uint32)
    lib.or_philox4x32_10(cpu_module.ptr(c, cpu_module._up), cpu_module.ptr(k, cpu_module._up),
                         cpu_module.ptr(o, cpu_module._up))
    return o


@pytest.mark.skipif(_torch_include() is None, reason="PyTorch headers not available")
def test_philox_matches_independent_implementation():
    rng = numpy.random.default_rng(7)
    cases = [[0, 0, 0, 0, 0, 0], [0xFFFFFFFF] * 6, [0, 0, 5, 0x22ab5871, 12345, 2],
             [0, 3, 17, 0x8754abcd, 2073599, 1], [0, 0, 1, 0x983abc12, 0, 7]]
    cases += [list(map(int, rng.integers(0, 2**32, 6, dtype=numpy.uint64))) for _ in range(300)]
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "p.cpp")
        exe = os.path.join(d, "p")
        with open(src, "w") as f:
            f.write(TORCH_SRC)
        subprocess.run(["g++", "-O1", "-std=c++17", "-I", _torch_include(), src, "-o", exe],
                       check=True, capture_output=True)
        inp = "\n".join(" ".join(str(x) for x in c) for c in cases) + "\n"
        r = subprocess.run([exe], input=inp, capture_output=True, text=True, check=True)
    got = [list(map(int, line.split())) for line in r.stdout.strip().splitlines()]
    assert len(got) == len(cases)
    for c, g in zip(cases, got):
        assert list(oracle_philox(c[:4], c[4:])) == g, c


def test_u01_mapping():
    lib = cpu_module.load("restated")
    # Random123 u01<float>: x * 2^-32 + 2^-33 in float, range (0, 1]
    assert lib.or_u01(0) == numpy.float32(2.0**-33)
    assert lib.or_u01(0xFFFFFFFF) == 1.0
    for x in (1, 12345, 2**31, 2**32 - 257, 2**24 + 1):
        expect = numpy.float32(numpy.float32(x) * numpy.float32(2.0**-32)) + numpy.float32(2.0**-33)
        assert lib.or_u01(x) == numpy.float32(expect)
    u = numpy.array([lib.or_u01(int(x)) for x in
                     numpy.random.default_rng(0).integers(0, 2**32, 20000, dtype=numpy.uint64)])
    assert u.min() > 0 and u.max() <= 1
    assert abs(u.mean() - 0.5) < 0.01


def test_philox_avalanche():
    base = oracle_philox([0, 0, 0, 0], [0, 0])
    flips = []
    for bit in range(32):
        o = oracle_philox([1 << bit, 0, 0, 0], [0, 0])
        flips.append(sum(bin(int(a) ^ int(b)).count("1") for a, b in zip(o, base)))
    assert 40 < numpy.mean(flips) < 88  # about half of 128 output bits flip
