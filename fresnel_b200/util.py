"""Buffer access helpers (fresnel/util.py)."""

import io
import os
from concurrent.futures import ThreadPoolExecutor

import numpy

try:
    import PIL.Image as PIL_Image
except ImportError:  # pragma: no cover - PIL is optional
    PIL_Image = None


# Whole-array copies of at least this many bytes between numpy and a mapped buffer are split
# into row blocks copied on several threads (numpy releases the GIL while it copies): one core
# copies some 5-10 GB/s, so a 1M-sphere scene's arrays (28 MB) would otherwise spend several
# milliseconds in a single memcpy.
PARALLEL_COPY_BYTES = 1 << 22

_pool = None
_pool_pid = None
_pool_workers = 1


def _copy_pool():
    """The copy threads of this process (made again in a forked child, which has none)."""
    global _pool, _pool_pid, _pool_workers
    if _pool is None or _pool_pid != os.getpid():
        _pool_workers = min(8, os.cpu_count() or 1)
        _pool = ThreadPoolExecutor(max_workers=_pool_workers, thread_name_prefix="fresnel-copy")
        _pool_pid = os.getpid()
    return _pool


def _whole(slc):
    return slc is Ellipsis or (isinstance(slc, slice) and slc == slice(None))


def _parallel_ok(dst, src):
    """True when ``dst[:] = src`` may be done as row blocks on several threads: the same shape,
    both C-contiguous and apart in memory, a plain numeric source, and enough bytes."""
    return (isinstance(src, numpy.ndarray) and src.shape == dst.shape and dst.ndim >= 1
            and dst.shape[0] > 1 and dst.nbytes >= PARALLEL_COPY_BYTES
            and src.dtype.kind in "biuf" and dst.dtype.kind in "biuf"
            and dst.flags.c_contiguous and src.flags.c_contiguous
            and not numpy.may_share_memory(dst, src))


def _copy_rows(dst, src, stream_copy=None):
    """``dst[:] = src`` (same shapes) as row blocks on the copy threads.  Each block is an
    ordinary numpy assignment, or ``stream_copy(dst_block, src_block)`` (the backend's copy with
    cache-bypassing stores, for a buffer uploaded next) where that takes the pair of types; either
    way the result equals the single assignment element for element."""
    pool = _copy_pool()
    n = dst.shape[0]
    step = -(-n // _pool_workers)

    def block(i):
        d, s = dst[i:i + step], src[i:i + step]
        if stream_copy is None or not stream_copy(d, s):
            d[...] = s
    futures = [pool.submit(block, i) for i in range(0, n, step)]
    for fut in futures:
        fut.result()


class Array:
    """numpy-like access to a backend buffer (fresnel/util.py:15-70).

    ``array[slice] = v`` maps the buffer, writes, unmaps (uploading to the device) and marks the
    owning geometry stale; ``array[slice]`` returns a copy and uploads nothing (a whole tracer
    output is downloaded straight into the returned array).
    """

    def __init__(self, buf, geom):
        self.buf = buf
        self.geom = geom
        self.buf.map()
        a = numpy.asarray(self.buf)
        self.shape = a.shape
        self.dtype = a.dtype
        self._unmap_read()

    def __setitem__(self, slc, data):
        self.buf.map()
        a = numpy.asarray(self.buf)
        if _whole(slc) and _parallel_ok(a, data):
            _copy_rows(a, data, getattr(self.buf, "streamCopy", None))
        else:
            a[slc] = data
        self.buf.unmap()
        if self.geom is not None:
            self.geom._geometry.update()

    def __getitem__(self, slc):
        read_copy = getattr(self.buf, "readCopy", None)
        if read_copy is not None and _whole(slc):
            # a tracer output downloaded straight into the returned array's own storage
            data = read_copy()
            if data is not None:
                return data
        self.buf.map()
        a = numpy.asarray(self.buf)
        if _whole(slc) and a.ndim >= 1 and a.shape[0] > 1 and a.nbytes >= PARALLEL_COPY_BYTES \
                and a.flags.c_contiguous and a.dtype.kind in "biuf":
            data = numpy.empty(a.shape, a.dtype)
            _copy_rows(data, a)
        else:
            data = numpy.array(a[slc], copy=True)
        self._unmap_read()
        return data

    def _unmap_read(self):
        """Unmaps after a read: the host copy is unchanged, so nothing is uploaded again (a
        backend without unmapRead treats every unmap as a write)."""
        getattr(self.buf, "unmapRead", self.buf.unmap)()


class ImageArray(Array):
    """An (H, W, 4) uint8 RGBA image with a PNG representation for notebooks."""

    def _repr_png_(self):
        if PIL_Image is None:
            raise RuntimeError("No PIL.Image module to format png")
        self.buf.map()
        f = io.BytesIO()
        PIL_Image.fromarray(numpy.asarray(self.buf), mode='RGBA').save(f, 'png')
        self._unmap_read()
        return f.getvalue()


def convex_polyhedron_from_vertices(vertices):
    """Faces of the convex hull of ``vertices`` in the form `geometry.ConvexPolyhedron` takes:
    a dict with ``face_origin``, ``face_normal``, ``face_color``, ``face_sides`` and ``radius``
    (fresnel/util.py:98-126)."""
    from ._common import find_polyhedron_faces
    return find_polyhedron_faces(vertices)
