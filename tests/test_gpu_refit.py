"""BVH refit (device option "refit"): after the primitives move, the refitted tree must find the
same closest hits as a tree built from scratch for the moved primitives, and the same ones as
the CPU oracle rendering the moved arrays.

Each case renders a scene once (building its trees), moves every primitive (positions jittered,
radii and orientations changed, counts kept), renders again with refit on, and compares the
Preview hit ids and the Path image with a fresh scene built from the moved arrays. The refit is
checked to have happened (tracer statistics) and the hit ids must be identical.
"""

import numpy
import pytest

import fresnel_b200 as fresnel
from fresnel_b200 import workloads
from grazing import check_hits
from parity import oracle_path_image, preview_hits, same_seed_fraction
from parity_record import record

pytestmark = pytest.mark.gpu


@pytest.fixture
def refit_on(gpu_device):
    """Refit on, and sphere scenes traced through their BVH (refit is a BVH operation; the
    automatic choice would give them a sphere grid, which is rebuilt instead)."""
    dd = gpu_device._device
    old = dd.getOption("refit"), dd.getOption("accel")
    dd.setOption("refit", 1)
    dd.setOption("accel", 0)
    yield
    dd.setOption("refit", old[0])
    dd.setOption("accel", old[1])


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


@pytest.mark.parametrize("name", list(CASES))
def test_refit_matches_oracle(name, gpu_device, oracle_device, refit_on):
    """The refitted scene against the oracle's own scene of the moved arrays (fresnel/util.py:
    54-62 and fresnel/gpu/Scene.h:64-83: an array write marks the geometry for update):
    Preview hit ids within the hit-id bar, same-seed Path on >= 99% of pixels within 1e-3."""
    build = CASES[name]
    scene = build(gpu_device)
    w, h = 120, 90
    preview_hits(gpu_device, scene, w, h, 1)  # builds the trees
    _move(scene, numpy.random.default_rng(6))
    t = fresnel.tracer.Path(gpu_device, w=w, h=h)
    t.seed = 4
    t._tracer.resetStats()
    t.sample(scene, samples=4)
    st = t._tracer.getStats()
    assert st["bvh_refits"] == st["bvh_builds"] >= 1
    gpath = numpy.array(t.linear_output[:], copy=True)
    gh, _, _ = preview_hits(gpu_device, scene, w, h, 2)

    oscene = build(oracle_device)
    _copy_arrays(scene, oscene)
    oscene.camera = scene.camera
    oh, _, _ = preview_hits(oracle_device, oscene, w, h, 2)
    check_hits("test_refit_matches_oracle", oracle_device, oscene, w, h, 2, gh, oh, scene=name)
    frac = same_seed_fraction(gpath, oracle_path_image(oracle_device, oscene, w, h, 5, 4))
    record("test_refit_matches_oracle", check="same_seed", scene=name, within_1e3=frac)
    assert frac >= 0.99
