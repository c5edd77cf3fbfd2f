"""Buffer access helpers (fresnel/util.py)."""

import io

import numpy

try:
    import PIL.Image as PIL_Image
except ImportError:  # pragma: no cover - PIL is optional
    PIL_Image = None


class Array:
    """numpy-like access to a backend buffer (fresnel/util.py:15-70).

    ``array[slice] = v`` maps the buffer, writes, unmaps (uploading to the device) and marks the
    owning geometry stale; ``array[slice]`` returns a copy.
    """

    def __init__(self, buf, geom):
        self.buf = buf
        self.geom = geom
        self.buf.map()
        a = numpy.asarray(self.buf)
        self.shape = a.shape
        self.dtype = a.dtype
        self.buf.unmap()

    def __setitem__(self, slc, data):
        self.buf.map()
        a = numpy.asarray(self.buf)
        a[slc] = data
        self.buf.unmap()
        if self.geom is not None:
            self.geom._geometry.update()

    def __getitem__(self, slc):
        self.buf.map()
        a = numpy.asarray(self.buf)
        data = numpy.array(a[slc], copy=True)
        self.buf.unmap()
        return data


class ImageArray(Array):
    """An (H, W, 4) uint8 RGBA image with a PNG representation for notebooks."""

    def _repr_png_(self):
        if PIL_Image is None:
            raise RuntimeError("No PIL.Image module to format png")
        self.buf.map()
        f = io.BytesIO()
        PIL_Image.fromarray(numpy.asarray(self.buf), mode='RGBA').save(f, 'png')
        self.buf.unmap()
        return f.getvalue()


def convex_polyhedron_from_vertices(vertices):
    """Faces of the convex hull of ``vertices`` in the form `geometry.ConvexPolyhedron` takes:
    a dict with ``face_origin``, ``face_normal``, ``face_color``, ``face_sides`` and ``radius``
    (fresnel/util.py:98-126)."""
    from ._common import find_polyhedron_faces
    return find_polyhedron_faces(vertices)
