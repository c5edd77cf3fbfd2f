"""Colour utilities (fresnel/color.py:9-62)."""

import numpy


def _channel(x):
    """sRGB transfer function inverse for one value or array, in the input's own precision."""
    if numpy.ndim(x) == 0:
        return x / 12.92 if x < 0.04045 else ((x + 0.055) / (1.055))**2.4
    out = numpy.empty(numpy.shape(x), dtype=numpy.float32)
    low = x < 0.04045
    out[low] = x[low] / 12.92
    high = numpy.logical_not(low)
    out[high] = ((x[high] + 0.055) / (1.055))**2.4
    return out


def linear(color):
    """Convert sRGB colour(s) to fresnel's linear colour space.

    Accepts shape (3,), (4,), (N, 3) or (N, 4); the alpha channel is dropped.  Returns float32
    with shape (3,) or (N, 3).  Each channel is converted in the input's precision and stored as
    float32, as the reference does.
    """
    c = numpy.ascontiguousarray(color)
    if c.shape == (3,) or c.shape == (4,):
        out = numpy.zeros(3, dtype=numpy.float32)
        for k in range(3):
            out[k] = _channel(c[k])
        return out
    if c.ndim == 2 and c.shape[1] in (3, 4):
        out = numpy.zeros((c.shape[0], 3), dtype=numpy.float32)
        for k in range(3):
            out[:, k] = _channel(c[:, k])
        return out
    raise TypeError("color must be a length 3, 4, Nx3, or Nx4 array")
