"""TEST INFRASTRUCTURE: CPU restatement of fresnel's output-side helpers, used only by tests as
the checker for the device-side versions; the product never imports it.

``histogram`` restates ``Tracer.histogram`` (fresnel/tracer.py:79-108): over the pixels of a
linear RGBA float32 image whose alpha is positive, the lightness l = 0.21 r + 0.72 g + 0.07 b
and the R, G, B channels, each raised to 1/2.2 and counted by numpy.histogram in 512 bins over
[0, 1].  Pinned against the reference's own method run on crafted images
(tests/golden/histogram.npz, made by tests/golden/make_histogram_golden.py).
"""

import numpy

N_BINS = 512


def histogram(linear):
    """(counts[512, 4] int64, upper bin edges[512]) of a (H, W, 4) float32 image
    (fresnel/tracer.py:93-108)."""
    a = numpy.asarray(linear, dtype=numpy.float32)
    img = a[a[:, :, 3] > 0]
    r, g, b = img[:, 0], img[:, 1], img[:, 2]
    lum = 0.21 * r + 0.72 * g + 0.07 * b
    cols = []
    edges = None
    for ch in (lum, r, g, b):
        counts, edges = numpy.histogram(ch**(1 / 2.2), bins=N_BINS, range=[0, 1])
        cols.append(counts)
    return numpy.stack(cols, axis=1), edges[1:]


def crafted_images(seed=0):
    """Linear RGBA test images for the histogram: random colours in [0, 1.3] with some
    transparent pixels, and one image of special values (0, 1, just above 1, negative, NaN,
    infinity, subnormal, alpha 0 / negative / NaN)."""
    rng = numpy.random.default_rng(seed)
    out = {}
    a = rng.uniform(0.0, 1.3, (48, 64, 4)).astype(numpy.float32)
    a[..., 3] = (rng.uniform(0, 1, (48, 64)) > 0.2).astype(numpy.float32)
    out["random"] = a
    b = rng.uniform(0.0, 1.0, (16, 16, 4)).astype(numpy.float32) ** 3
    b[..., 3] = 1.0
    specials = numpy.array([0.0, 1.0, numpy.nextafter(numpy.float32(1), numpy.float32(2)), -0.5,
                            numpy.nan, numpy.inf, 1e-40, -0.0, 0.5, 0.25, 2.0 ** -9,
                            2.0 ** -20, 0.999999, 3.0], dtype=numpy.float32)
    flat = b.reshape(-1, 4)
    for i, v in enumerate(specials):
        flat[i, i % 3] = v
        flat[20 + i, :3] = v
    flat[40, 3] = 0.0
    flat[41, 3] = -1.0
    flat[42, 3] = numpy.nan
    flat[43, 3] = 1e-30
    out["specials"] = b
    out["transparent"] = numpy.zeros((8, 8, 4), numpy.float32)
    return out
