"""BVH refit (device option "refit"): after the primitives move, the refitted tree must find the
same closest hits as a tree built from scratch for the moved primitives.

Each case renders a scene once (building its trees), moves every primitive (positions jittered,
radii and orientations changed, counts kept), renders again with refit on, and compares the
Preview hit ids and the Path image with a fresh scene built from the moved arrays. The refit is
checked to have happened (tracer statistics) and the hit ids must be identical.
"""

import numpy
import pytest

import fresnel_b200 as fresnel
from fresnel_b200 import workloads
from parity import preview_hits

pytestmark = pytest.mark.gpu


@pytest.fixture
def refit_on(gpu_device):
    dd = gpu_device._device
    old = dd.getOption("refit")
    dd.setOption("refit", 1)
    yield
    dd.setOption("refit", old)


def _move(scene, rng):
    for g in scene.geometry:
        for name in ("position", "points"):
            if hasattr(g, name):
                a = getattr(g, name)
                arr = numpy.array(a[:], copy=True)
                arr += rng.uniform(-0.3, 0.3, arr.shape).astype(numpy.float32)
                a[:] = arr
        if hasattr(g, "radius") and not isinstance(g, fresnel.geometry.Cylinder):
            r = numpy.array(g.radius[:], copy=True)
            g.radius[:] = (r * rng.uniform(0.8, 1.2, r.shape)).astype(numpy.float32)
        if hasattr(g, "orientation"):
            q = rng.normal(size=g.orientation[:].shape)
            q /= numpy.linalg.norm(q, axis=1, keepdims=True)
            g.orientation[:] = q.astype(numpy.float32)


def _copy_arrays(src, dst):
    for gs, gd in zip(src.geometry, dst.geometry):
        for name in ("position", "points", "radius", "orientation", "color"):
            if hasattr(gs, name):
                getattr(gd, name)[:] = numpy.array(getattr(gs, name)[:], copy=True)


CASES = {
    "spheres": lambda d: workloads.random_spheres(d, 5000, 40.0, seed=31, colors=True),
    "mixed": lambda d: workloads.config3(d, scale=0.005),
}


@pytest.mark.parametrize("name", list(CASES))
def test_refit_matches_rebuild(name, gpu_device, refit_on):
    build = CASES[name]
    scene = build(gpu_device)
    w, h = 120, 90
    preview_hits(gpu_device, scene, w, h, 1)  # builds the trees
    _move(scene, numpy.random.default_rng(5))
    t = fresnel.tracer.Path(gpu_device, w=w, h=h)
    t.seed = 9
    t._tracer.resetStats()
    t.sample(scene, samples=3)
    st = t._tracer.getStats()
    # one tree per geometry, or one combined tree for a scene of several geometries
    assert st["bvh_builds"] >= 1 and st["bvh_refits"] == st["bvh_builds"]
    refit_path = numpy.array(t.linear_output[:], copy=True)
    refit_hits, refit_lin, _ = preview_hits(gpu_device, scene, w, h, 2)

    fresh = build(gpu_device)
    _copy_arrays(scene, fresh)
    fresh.camera = scene.camera
    dd = gpu_device._device
    dd.setOption("refit", 0)
    try:
        t2 = fresnel.tracer.Path(gpu_device, w=w, h=h)
        t2.seed = 9
        t2.sample(fresh, samples=3)
        fresh_hits, fresh_lin, _ = preview_hits(gpu_device, fresh, w, h, 2)
    finally:
        dd.setOption("refit", 1)
    assert numpy.count_nonzero(fresh_hits[..., 0]) > 0
    assert numpy.array_equal(refit_hits, fresh_hits)
    assert numpy.abs(refit_lin - fresh_lin).max() <= 1e-6
    close = numpy.all(numpy.abs(refit_path - numpy.array(t2.linear_output[:])) <= 1e-5, axis=-1)
    assert close.mean() >= 0.999
