"""Tracer.histogram's CPU restatement (oracle/output_path.py) against the reference's own
method run on crafted images (tests/golden/histogram.npz), and the bin edges the product
returns against numpy's."""

import os

import numpy

from fresnel_b200 import tracer
from oracle import output_path

GOLDEN = numpy.load(os.path.join(os.path.dirname(__file__), "golden", "histogram.npz"))
NAMES = ("random", "specials", "transparent")


def test_restatement_matches_reference_goldens():
    import warnings
    for name in NAMES:
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", RuntimeWarning)
            counts, edges = output_path.histogram(GOLDEN[name + "_image"])
        assert numpy.array_equal(counts, GOLDEN[name + "_counts"]), name
        assert numpy.array_equal(edges, GOLDEN[name + "_edges"]), name
    assert GOLDEN["transparent_counts"].sum() == 0


def test_product_bin_edges_are_numpys():
    assert tracer._HIST_EDGES.dtype == numpy.float32
    assert numpy.array_equal(tracer._HIST_EDGES[1:], GOLDEN["random_edges"])
    assert tracer._HIST_EDGES[0] == 0.0 and tracer._HIST_EDGES[-1] == 1.0


def test_special_values_are_binned_as_numpy_does():
    # 0 and 1 are counted (1 in the last bin; so is the float just above 1, whose power rounds
    # to 1); larger values, negatives, NaN and infinity are not; alpha <= 0 or NaN hides a pixel
    c = GOLDEN["specials_counts"]
    img = GOLDEN["specials_image"].reshape(-1, 4)
    vis = img[img[:, 3] > 0]
    r = vis[:, 0]
    above_one = numpy.nextafter(numpy.float32(1), numpy.float32(2))
    expect = numpy.count_nonzero((r >= 0) & (r <= above_one))
    assert c[:, 1].sum() == expect
    assert c[511, 1] >= numpy.count_nonzero((r == 1.0) | (r == above_one))
    assert len(vis) == len(img) - 3  # alpha 0, -1 and NaN
