"""util.Array on the CPU: large whole-array writes and reads are copied as row blocks on several
threads, and must give exactly what the single numpy assignment gives; everything else keeps the
plain assignment. A stand-in buffer with map()/unmap() and __array__ replaces the backend's."""

import warnings

import numpy
import pytest

from fresnel_b200 import util


class FakeBuffer:
    """map()/unmap() like the backend's Array classes, the storage shown to numpy as is."""

    def __init__(self, shape, dtype):
        self.a = numpy.zeros(shape, dtype)
        self.mapped = False
        self.maps = 0

    def map(self):
        assert not self.mapped
        self.mapped = True
        self.maps += 1

    def unmap(self):
        assert self.mapped
        self.mapped = False

    def __array__(self, dtype=None, copy=None):
        assert self.mapped, "buffer read while unmapped"
        return self.a


class FakeGeometry:
    def __init__(self):
        self.updates = 0
        self._geometry = self

    def update(self):
        self.updates += 1


BIG = util.PARALLEL_COPY_BYTES // 12 + 1001  # rows of 3 float32: just over the threshold


def _plain_write(shape, dtype, data, slc=slice(None)):
    a = numpy.zeros(shape, dtype)
    a[slc] = data
    return a


@pytest.mark.parametrize("src_dtype", [numpy.float32, numpy.float64, numpy.int32, numpy.uint8])
def test_large_write_equals_plain_assignment(src_dtype):
    rng = numpy.random.default_rng(0)
    data = (rng.uniform(-100, 100, (BIG, 3))).astype(src_dtype)
    buf = FakeBuffer((BIG, 3), numpy.float32)
    geom = FakeGeometry()
    arr = util.Array(buf, geom)
    assert util._parallel_ok(buf.a, data)
    arr[:] = data
    assert numpy.array_equal(buf.a, _plain_write((BIG, 3), numpy.float32, data))
    assert geom.updates == 1 and not buf.mapped


def test_large_write_with_ellipsis_and_odd_row_count():
    data = numpy.arange(3 * (BIG + 7), dtype=numpy.float32).reshape(BIG + 7, 3)
    buf = FakeBuffer((BIG + 7, 3), numpy.float32)
    util.Array(buf, None)[...] = data
    assert numpy.array_equal(buf.a, data)


@pytest.mark.parametrize("case", ["broadcast", "list", "partial", "small", "view_of_self",
                                  "strided", "complex"])
def test_other_writes_keep_plain_assignment(case):
    rng = numpy.random.default_rng(1)
    shape = (BIG, 3)
    buf = FakeBuffer(shape, numpy.float32)
    buf.a[:] = rng.uniform(0, 1, shape).astype(numpy.float32)
    before = buf.a.copy()
    arr = util.Array(buf, None)
    slc = slice(None)
    if case == "broadcast":
        data = numpy.array([1.0, 2.0, 3.0])
    elif case == "list":
        data = [[0.5, 0.25, 0.125]]
    elif case == "partial":
        slc = slice(10, 2000)
        data = rng.uniform(0, 1, (1990, 3))
    elif case == "small":
        buf = FakeBuffer((50, 3), numpy.float32)
        before = buf.a.copy()
        arr = util.Array(buf, None)
        data = rng.uniform(0, 1, (50, 3))
    elif case == "view_of_self":
        data = buf.a[::-1]  # overlaps the destination: numpy buffers it
    elif case == "strided":
        data = numpy.asfortranarray(rng.uniform(0, 1, shape))
    else:
        data = (rng.uniform(0, 1, shape) + 0j)
    if case != "list":
        assert not (isinstance(data, numpy.ndarray) and util._whole(slc)
                    and util._parallel_ok(buf.a, data))
    expect = before.copy()
    src = data.copy() if isinstance(data, numpy.ndarray) else data
    with numpy.errstate(all="ignore"):
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            expect[slc] = src
            arr[slc] = data
    assert numpy.array_equal(buf.a, expect)


@pytest.mark.parametrize("shape,dtype", [((BIG, 3), numpy.float32),
                                         ((1080, 1920, 4), numpy.uint8),
                                         ((541, 960, 4), numpy.float32)])
def test_large_read_equals_copy(shape, dtype):
    rng = numpy.random.default_rng(2)
    buf = FakeBuffer(shape, dtype)
    buf.a[:] = rng.uniform(0, 200, shape).astype(dtype)
    out = util.Array(buf, None)[:]
    assert out.shape == shape and out.dtype == numpy.dtype(dtype)
    assert out.flags.c_contiguous
    assert numpy.array_equal(out, buf.a)
    assert not numpy.may_share_memory(out, buf.a)
    assert not buf.mapped
    part = util.Array(buf, None)[5:9]
    assert numpy.array_equal(part, buf.a[5:9]) and not numpy.may_share_memory(part, buf.a)


def test_copy_threads_made_again_in_a_new_process(monkeypatch):
    # a forked child has none of its parent's threads: the pool is keyed by the process id
    buf = FakeBuffer((BIG, 3), numpy.float32)
    util.Array(buf, None)[:] = numpy.ones((BIG, 3), numpy.float32)
    parent_pool = util._copy_pool()
    assert util._copy_pool() is parent_pool
    monkeypatch.setattr(util.os, "getpid", lambda: -12345)
    child_pool = util._copy_pool()
    assert child_pool is not parent_pool
    data = numpy.arange(3 * BIG, dtype=numpy.float32).reshape(BIG, 3)
    util.Array(buf, None)[:] = data
    assert numpy.array_equal(buf.a, data)
