"""Edge cases of the GPU engine: geometries without primitives and a one-pixel image.

fresnel lets a geometry be created with N = 0 (fresnel/geometry.py: Sphere, Cylinder take N or the
length of their arrays). Such a geometry has no BVH; the per-geometry traversal skips it, and
the combined tree leaves it out. It must change no image, and a scene that holds only empty
geometries shows its background everywhere, as a scene with none does
(fresnel/common/TracerPathMethods.h:44-50 for the path tracer's primary misses).
"""

import numpy
import pytest

import fresnel_b200 as fresnel

pytestmark = pytest.mark.gpu


def _spheres(device, n=200, seed=0):
    scene = fresnel.Scene(device=device)
    pos = numpy.random.default_rng(seed).uniform(-5, 5, (n, 3)).astype(numpy.float32)
    fresnel.geometry.Sphere(scene, position=pos, radius=0.5)
    scene.camera = fresnel.camera.Orthographic.fit(scene)
    return scene


def _path(device, scene, w, h, spp, seed=3):
    t = fresnel.tracer.Path(device, w=w, h=h)
    t.seed = seed
    t.sample(scene, samples=spp, light_samples=1)
    return numpy.array(t.linear_output[:], copy=True)


def test_empty_geometries_change_no_image(gpu_device):
    scene = _spheres(gpu_device)
    prev_a = fresnel.preview(scene, w=64, h=48, anti_alias=False)[:]
    path_a = _path(gpu_device, scene, 64, 48, 4)
    assert prev_a[..., 3].max() == 255

    fresnel.geometry.Sphere(scene, N=0)
    fresnel.geometry.Cylinder(scene, N=0)
    assert len(scene.geometry) == 3
    prev_b = fresnel.preview(scene, w=64, h=48, anti_alias=False)[:]
    path_b = _path(gpu_device, scene, 64, 48, 4)
    numpy.testing.assert_array_equal(prev_a, prev_b)
    numpy.testing.assert_array_equal(path_a, path_b)


def test_scene_of_empty_geometries_shows_background(gpu_device):
    scene = fresnel.Scene(device=gpu_device)
    fresnel.geometry.Sphere(scene, N=0)
    bg = fresnel.color.linear((0.125, 0.75, 0.375))
    scene.background_color = bg
    scene.background_alpha = 0.5
    scene.camera = fresnel.camera.Orthographic(position=(0, 0, 10), look_at=(0, 0, 0),
                                               up=(0, 1, 0), height=7)
    lin = _path(gpu_device, scene, 40, 30, 3)
    assert lin.shape == (30, 40, 4)
    # every sample of every pixel is the background: the running mean stays exactly on it
    numpy.testing.assert_array_equal(lin[..., :3], numpy.broadcast_to(
        numpy.asarray(bg, numpy.float32), (30, 40, 3)))
    numpy.testing.assert_array_equal(lin[..., 3], numpy.full((30, 40), 0.5, numpy.float32))
    buf = fresnel.preview(scene, w=40, h=30, anti_alias=False)[:]
    numpy.testing.assert_array_equal(buf[:, :, 3], numpy.full((30, 40), 128, buf.dtype))


def test_one_pixel_image(gpu_device):
    scene = _spheres(gpu_device)
    lin = _path(gpu_device, scene, 1, 1, 8)
    assert lin.shape == (1, 1, 4) and numpy.isfinite(lin).all()
    out = fresnel.preview(scene, w=1, h=1, anti_alias=True)[:]
    assert out.shape == (1, 1, 4)
