"""The allocation-free path render (fr_tracer_render_path_static) against fr_tracer_render_path.

fr_tracer_render_path_static keeps its wavefront state in a fixed device array instead of
tracer-owned allocations. It traces fewer samples per wavefront (262144 slots / pixels), but every
path's arithmetic depends only on its (pixel, sample, light sample), and the running mean folds
samples in sample order. Its images must therefore equal the allocating entry point's. The test
compares them within 1e-6 after each of two calls in a row (the second call continues the first
one's running mean), on a sphere scene traced through its BVH, a dense sphere scene traced
through the sphere grid (also with the persistent and per-lane-refill kernel options), a scene
of every geometry type traced through one combined tree and a scene of spheres and bonds traced
through the grid over its parts. It also checks the size limit,
the built-scene rule, and that a static render leaves no stale primary hits behind.

The file name sorts last so that pytest collects it after every other test. It passes alone too.
"""

import numpy
import pytest

import fresnel_b200 as fresnel
from fresnel_b200 import workloads

pytestmark = pytest.mark.gpu

TOL = 1e-6


def _scene(device):
    return workloads.config1(device)


SCENES = {  # scene, device option "accel", grid kind (0 trees, 1 sphere grid, 2 parts grid)
    "spheres_bvh": (workloads.config1, 0, 0),
    "dense_grid": (lambda d: workloads.config2(d, n=20000, box=140.0 * 0.02**(1 / 3)), 2, 1),
    "mixed": (lambda d: workloads.config3(d, scale=0.002), 0, 0),
    "parts_grid": (lambda d: workloads.config3(d, scale=0.002), 2, 2),
    "parts_grid_no_mesh": (lambda d: workloads.serving_scene(d, 4000, 5), 2, 2),
}


def _pair(device, w, h, light_samples, build=_scene):
    scene = build(device)
    a = fresnel.tracer.Path(device, w=w, h=h)
    b = fresnel.tracer.Path(device, w=w, h=h)
    for t in (a, b):
        t.reset()
        t.seed = 7
        t._tracer.setLightSamples(light_samples)
    return scene, a, b


def _compare(scene, a, b, w, h, spp):
    for call in range(2):
        a._tracer.renderSamples(scene._scene, spp)
        b._tracer.renderSamplesStatic(scene._scene, spp)
        la = numpy.array(a.linear_output[:], copy=True)
        lb = numpy.array(b.linear_output[:], copy=True)
        assert la.shape == (h, w, 4)
        assert numpy.isfinite(la).all()
        diff = numpy.abs(la - lb).max()
        assert diff <= TOL, f"call {call}: max |linear difference| {diff}"
        sa = numpy.array(a.output[:], copy=True)
        sb = numpy.array(b.output[:], copy=True)
        assert (numpy.abs(sa.astype(int) - sb.astype(int)) <= 1).all()
    assert a._tracer.getNumSamples() == b._tracer.getNumSamples() == 2 * spp


@pytest.mark.parametrize("w,h,spp,ls", [(200, 150, 24, 1), (96, 64, 10, 3)])
def test_static_render_matches_allocating_render(gpu_device, w, h, spp, ls):
    scene, a, b = _pair(gpu_device, w, h, ls)
    scene._scene.build()
    _compare(scene, a, b, w, h, spp)


@pytest.mark.parametrize("name", list(SCENES))
def test_static_render_matches_on_each_structure(gpu_device, name):
    build, accel, grid = SCENES[name]
    dd = gpu_device._device
    old = dd.getOption("accel")
    try:
        dd.setOption("accel", accel)
        scene, a, b = _pair(gpu_device, 160, 96, 2, build)
        scene._scene.build()
        assert scene._scene.getAccel()[0] == grid
        _compare(scene, a, b, 160, 96, 6)
    finally:
        dd.setOption("accel", old)


@pytest.mark.parametrize("option", ["persistent", "refill"])
def test_static_render_matches_with_kernel_options(gpu_device, option):
    dd = gpu_device._device
    old = dd.getOption(option)
    try:
        dd.setOption(option, 1)
        build, _, _ = SCENES["dense_grid"]
        scene, a, b = _pair(gpu_device, 128, 80, 1, build)
        scene._scene.build()
        _compare(scene, a, b, 128, 80, 5)
    finally:
        dd.setOption(option, old)


def test_static_render_leaves_no_stale_primary_hits(gpu_device):
    scene = _scene(gpu_device)
    t = fresnel.tracer.Path(gpu_device, w=64, h=48)
    scene._scene.build()
    t._tracer.renderSamples(scene._scene, 2)
    assert t._tracer.primaryHits().shape[:2] == (48, 64)
    t._tracer.renderSamplesStatic(scene._scene, 2)
    with pytest.raises(RuntimeError, match="last path render was not this tracer's"):
        t._tracer.primaryHits()


def test_static_render_limits(gpu_device):
    scene = _scene(gpu_device)
    big = fresnel.tracer.Path(gpu_device, w=1024, h=512)
    scene._scene.build()
    with pytest.raises(RuntimeError, match="limit of 262144 pixels"):
        big._tracer.renderSamplesStatic(scene._scene, 1)

    small = fresnel.tracer.Path(gpu_device, w=64, h=64)
    scene.geometry[0].position[0] = (0.25, 0.5, 0.75)  # the BVH is now stale
    with pytest.raises(RuntimeError, match="needs a built scene"):
        small._tracer.renderSamplesStatic(scene._scene, 1)
    scene._scene.build()
    small._tracer.renderSamplesStatic(scene._scene, 2)
    assert numpy.isfinite(small.linear_output[:]).all()
