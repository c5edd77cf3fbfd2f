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


class TrackingBuffer(FakeBuffer):
    """A backend buffer with the read-only unmap and the direct whole-array download: unmap()
    marks the host copy for upload, unmapRead() does not; readCopy() returns a copy (or None, when
    the backend has no storage to give)."""

    def __init__(self, shape, dtype, copies=True):
        super().__init__(shape, dtype)
        self.stale = False
        self.copies = copies
        self.read_copies = 0

    def unmap(self):
        super().unmap()
        self.stale = True

    def unmapRead(self):
        FakeBuffer.unmap(self)

    def readCopy(self):
        self.read_copies += 1
        return self.a.copy() if self.copies else None


@pytest.mark.parametrize("shape", [(BIG, 3), (40, 3)])
def test_reads_do_not_mark_the_host_copy_for_upload(shape):
    buf = TrackingBuffer(shape, numpy.float32, copies=False)
    arr = util.Array(buf, FakeGeometry())
    assert not buf.stale  # constructing the wrapper reads the shape only
    buf.a[:] = 7.0
    assert numpy.all(arr[:] == 7.0) and numpy.all(arr[2:5] == 7.0)
    assert not buf.stale and not buf.mapped
    arr[1] = (1.0, 2.0, 3.0)
    assert buf.stale


def test_whole_reads_take_the_direct_download():
    buf = TrackingBuffer((12, 10, 4), numpy.uint8)
    buf.a[:] = numpy.arange(480, dtype=numpy.uint8).reshape(12, 10, 4)
    arr = util.ImageArray(buf, None)
    maps = buf.maps
    out = arr[:]
    assert buf.read_copies == 1 and buf.maps == maps  # no map: the copy came from readCopy
    assert numpy.array_equal(out, buf.a) and not numpy.may_share_memory(out, buf.a)
    out = arr[...]
    assert buf.read_copies == 2 and numpy.array_equal(out, buf.a)
    part = arr[3:5]  # a part is read through the mapped buffer
    assert buf.read_copies == 2 and buf.maps == maps + 1
    assert numpy.array_equal(part, buf.a[3:5])
    none = TrackingBuffer((12, 10, 4), numpy.uint8, copies=False)
    none.a[:] = 5
    assert numpy.all(util.ImageArray(none, None)[:] == 5) and none.read_copies == 1


def _stream_copy():
    from fresnel_b200 import _gpu
    return _gpu.ArrayVec3f.streamCopy


@pytest.mark.parametrize("src_dtype,dst_dtype,shape", [
    (numpy.float32, numpy.float32, (BIG, 3)),
    (numpy.float64, numpy.float32, (BIG, 3)),
    (numpy.float64, numpy.float32, (5, 3)),      # shorter than one block of the conversion
    (numpy.uint8, numpy.uint8, (97, 13, 4)),     # an odd number of bytes
    (numpy.float32, numpy.float32, (1,)),
])
def test_stream_copy_equals_numpy_assignment(src_dtype, dst_dtype, shape):
    """The backend's copy with streaming stores gives the numpy assignment's bytes, float64
    rounding, infinities, NaN and subnormals included, at any alignment of the destination."""
    copy = _stream_copy()
    rng = numpy.random.default_rng(3)
    src = rng.uniform(-1e3, 1e3, shape).astype(src_dtype)
    if src.dtype.kind == "f":
        flat = src.reshape(-1)
        special = [numpy.inf, -numpy.inf, numpy.nan, 1e-45, -1e-44, 3.4028235e38, 1e39, -0.0,
                   1.0000000596046448]  # the last rounds to even
        with numpy.errstate(over="ignore"):
            flat[:len(special)] = numpy.array(special[:flat.size], dtype=src_dtype)
    for shift in (0, 4, 12):  # destination offsets of 0, 4 and 12 bytes from a 16-byte boundary
        storage = numpy.zeros(src.size * numpy.dtype(dst_dtype).itemsize + 64, numpy.uint8)
        base = (-storage.ctypes.data) % 16 + shift
        dst = storage[base:base + src.size * numpy.dtype(dst_dtype).itemsize].view(dst_dtype)
        dst = dst.reshape(shape)
        with numpy.errstate(over="ignore"):
            expect = numpy.zeros(shape, dst_dtype)
            expect[...] = src
        assert copy(dst, src) is True
        assert dst.tobytes() == expect.tobytes()


def test_stream_copy_declines_what_it_does_not_take():
    copy = _stream_copy()
    a = numpy.zeros((100, 3), numpy.float32)
    assert copy(a, numpy.ones((100, 3), numpy.int32)) is False          # other types
    assert copy(a, numpy.ones((99, 3), numpy.float32)) is False         # other shapes
    assert copy(a, numpy.ones((3, 100), numpy.float32).T) is False      # not C-contiguous
    assert copy(a[:60], a[40:]) is False                                # overlapping storage
    assert not a.any()


def test_large_write_through_stream_copy_equals_plain_assignment():
    class StreamingBuffer(TrackingBuffer):
        streamCopy = staticmethod(_stream_copy())
    rng = numpy.random.default_rng(4)
    for src_dtype in (numpy.float64, numpy.float32, numpy.int64):  # int64: numpy's assignment
        data = rng.uniform(-50, 50, (BIG, 3)).astype(src_dtype)
        buf = StreamingBuffer((BIG, 3), numpy.float32)
        util.Array(buf, FakeGeometry())[:] = data
        assert numpy.array_equal(buf.a, _plain_write((BIG, 3), numpy.float32, data))
        assert buf.stale and not buf.mapped
