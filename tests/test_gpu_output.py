"""Device-side output path: Tracer.histogram on the GPU against the reference's method
(goldens made by its own code) and the CPU restatement, and the page-locked download of the
output buffers.

The device computes numpy's float32 lightness exactly and raises each value to float32(1/2.2)
in double precision, rounded once.  numpy's float32 power is not always correctly rounded (it
differs from the correctly rounded value by an ulp for a sizeable share of inputs on common
hosts), so a value lying within an ulp of one of the 512 bin edges can land in the neighbouring
bin: each column may differ by at most TOL_REL of its counted values (plus 2), moved between
neighbouring bins.
"""

import os
import warnings

import numpy
import pytest

import fresnel_b200 as fresnel
from fresnel_b200 import workloads
from oracle import output_path

pytestmark = pytest.mark.gpu

GOLDEN = numpy.load(os.path.join(os.path.dirname(__file__), "golden", "histogram.npz"))
TOL_REL = 1e-4


def _close(got, ref):
    assert got.shape == ref.shape == (512, 4)
    for c in range(4):
        n = int(ref[:, c].sum())
        d = numpy.abs(got[:, c].astype(numpy.int64) - ref[:, c].astype(numpy.int64))
        assert d.sum() <= 2 + 2 * TOL_REL * n, f"column {c}: {d.sum()} of {n} counts differ"
        assert abs(int(got[:, c].sum()) - n) <= 1 + TOL_REL * n


@pytest.mark.parametrize("name", ["random", "specials", "transparent"])
def test_histogram_matches_reference_goldens(gpu_device, name):
    img = GOLDEN[name + "_image"]
    h, w = img.shape[:2]
    t = fresnel.tracer.Path(gpu_device, w=w, h=h)
    t._tracer.setLinearOutput(img)
    assert numpy.array_equal(t.linear_output[:], img, equal_nan=True)  # page-locked read-back
    counts, edges = t.histogram()
    assert counts.dtype == numpy.int64
    assert numpy.array_equal(edges, GOLDEN[name + "_edges"])
    _close(counts, GOLDEN[name + "_counts"])


def test_histogram_of_a_render_matches_restatement(gpu_device):
    scene = workloads.config1(gpu_device)
    scene.background_alpha = 0.0
    t = fresnel.tracer.Path(gpu_device, w=240, h=180)
    t.sample(scene, samples=8)
    lin = numpy.array(t.linear_output[:], copy=True)
    assert 0 < numpy.count_nonzero(lin[:, :, 3] > 0) < lin.shape[0] * lin.shape[1]
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        ref, ref_edges = output_path.histogram(lin)
    counts, edges = t.histogram()
    assert numpy.array_equal(edges, ref_edges)
    _close(counts, ref)
    # a second call gives the same counts (the buffer is cleared each time)
    assert numpy.array_equal(t.histogram()[0], counts)


def test_histogram_of_a_fresh_tracer_is_empty(gpu_device):
    t = fresnel.tracer.Preview(gpu_device, w=33, h=17)
    counts, _ = t.histogram()
    assert counts.sum() == 0


def test_histogram_at_full_hd(gpu_device):
    # every bin and the 8 KB read-back at the benchmark's image size
    rng = numpy.random.default_rng(9)
    img = rng.uniform(0.0, 1.1, (1080, 1920, 4)).astype(numpy.float32)
    img[..., 3] = rng.uniform(0, 1, (1080, 1920)) > 0.1
    t = fresnel.tracer.Path(gpu_device, w=1920, h=1080)
    t._tracer.setLinearOutput(img)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        ref, _ = output_path.histogram(img)
    _close(t.histogram()[0], ref)
