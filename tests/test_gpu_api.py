"""Behaviour of the fresnel API on the GPU engine, following the reference's own tests
(fresnel/test/test_scene.py, test_tracer_direct.py, test_tracer_path.py, test_device.py,
test_geometry_*.py) where they check exact values, shapes, seeds and error handling."""

import math

import numpy
import pytest

import fresnel_b200 as fresnel
from fresnel_b200 import workloads

pytestmark = pytest.mark.gpu


def test_device_modes(gpu_device):
    assert 'gpu' in fresnel.Device.available_modes
    assert 'auto' in fresnel.Device.available_modes
    assert len(fresnel.Device.available_gpus) >= 1
    assert fresnel.Device(mode='gpu', n=1).mode == 'gpu'
    assert 'Enabled GPUs' in str(gpu_device)
    with pytest.raises(RuntimeError):
        fresnel.Device(mode='cpu')


def test_background_exact(gpu_device):
    # fresnel/test/test_scene.py:17-42: uniform background bytes
    scene = fresnel.Scene(device=gpu_device)
    scene.background_color = fresnel.color.linear((0.125, 0.75, 0.375))
    numpy.testing.assert_array_equal(scene.background_color,
                                     fresnel.color.linear((0.125, 0.75, 0.375)))
    scene.background_alpha = 0.5
    assert scene.background_alpha == 0.5
    scene.camera = fresnel.camera.Orthographic(position=(0, 0, 10), look_at=(0, 0, 0),
                                               up=(0, 1, 0), height=7)
    buf = fresnel.preview(scene, w=100, h=100, anti_alias=False)[:]
    numpy.testing.assert_array_equal(buf[:, :, 3], numpy.full((100, 100), 128, buf.dtype))
    numpy.testing.assert_array_equal(buf[:, :, 0:3],
                                     numpy.ones((100, 100, 3), buf.dtype) * (32, 191, 96))


def test_preview_resize(gpu_device):
    scene = workloads.hex_spheres(gpu_device)
    t = fresnel.tracer.Preview(device=gpu_device, w=100, h=100, anti_alias=False)
    assert t.output[:].shape == (100, 100, 4)
    t.resize(w=200, h=300)
    assert t.output[:].shape == (300, 200, 4)
    out = t.render(scene)[:]
    assert out.shape == (300, 200, 4) and out[..., 3].max() == 255
    with pytest.raises(RuntimeError):
        t.resize(0, 10)


def test_path_seed_schedule(gpu_device):
    scene = workloads.hex_spheres(gpu_device)
    t = fresnel.tracer.Path(device=gpu_device, w=32, h=32)
    assert t.seed == 1                       # constructor resets once
    t.sample(scene, samples=2)
    assert t.seed == 2 and t._tracer.getNumSamples() == 2
    t.sample(scene, samples=3, reset=False)
    assert t.seed == 2 and t._tracer.getNumSamples() == 5
    t.resize(16, 16)
    assert t.seed == 3 and t._tracer.getNumSamples() == 0
    t.seed = 11
    t.sample(scene, samples=1)
    assert t.seed == 12


def test_path_render_equals_sample(gpu_device):
    # sample(k) must equal k successive render() calls
    scene = workloads.hex_spheres(gpu_device)
    a = fresnel.tracer.Path(device=gpu_device, w=40, h=30)
    a.sample(scene, samples=5, light_samples=2)
    b = fresnel.tracer.Path(device=gpu_device, w=40, h=30)
    b.reset()
    b._tracer.setLightSamples(2)
    for _ in range(5):
        b.render(scene)
    numpy.testing.assert_array_equal(a.linear_output[:], b.linear_output[:])


def test_device_mismatch(gpu_device):
    other = fresnel.Device(mode='gpu')
    scene = workloads.hex_spheres(other)
    t = fresnel.tracer.Preview(device=gpu_device, w=10, h=10)
    with pytest.raises(RuntimeError, match="devices do not match"):
        t.render(scene)


def test_geometry_enable_disable_remove(gpu_device):
    scene = workloads.hex_spheres(gpu_device)
    g = scene.geometry[0]
    before = fresnel.preview(scene, w=50, h=50, anti_alias=False)[:]
    g.disable()
    empty = fresnel.preview(scene, w=50, h=50, anti_alias=False)[:]
    assert empty[..., 3].max() == 0
    g.enable()
    numpy.testing.assert_array_equal(fresnel.preview(scene, w=50, h=50, anti_alias=False)[:],
                                     before)
    g.remove()
    assert scene.geometry == []
    with pytest.raises(RuntimeError):
        g.enable()
    with pytest.raises(RuntimeError):
        g.disable()


def test_array_roundtrip_and_update(gpu_device):
    scene = fresnel.Scene(device=gpu_device)
    pos = numpy.random.default_rng(0).uniform(-5, 5, (50, 3)).astype(numpy.float32)
    g = fresnel.geometry.Sphere(scene, position=pos, radius=0.5)
    numpy.testing.assert_array_equal(g.position[:], pos)
    numpy.testing.assert_array_equal(g.radius[:], numpy.full(50, 0.5, numpy.float32))
    g.position[3] = (1, 2, 3)
    numpy.testing.assert_array_equal(g.position[3], (1, 2, 3))
    scene.camera = fresnel.camera.Orthographic.fit(scene)
    a = fresnel.preview(scene, w=64, h=64, anti_alias=False)[:]
    g.position[:] = pos + 100.0  # move everything out of view -> BVH rebuilt
    b = fresnel.preview(scene, w=64, h=64, anti_alias=False)[:]
    assert a[..., 3].max() == 255 and b[..., 3].max() == 0


def test_highlight_warning(gpu_device):
    scene = workloads.hex_spheres(gpu_device)
    scene.geometry[0].material = fresnel.material.Material(solid=1.0, color=(2.0, 2.0, 2.0))
    scene.geometry[0].outline_width = 0.0
    t = fresnel.tracer.Preview(device=gpu_device, w=50, h=50, anti_alias=False)
    t.enable_highlight_warning((0, 1, 0))
    out = t.render(scene)[:]
    fg = out[..., 3] == 255
    assert numpy.all(out[fg][:, :3] == (0, 255, 0))
    t.disable_highlight_warning()
    out = t.render(scene)[:]
    assert numpy.all(out[fg][:, :3] == (255, 255, 255))


def test_geometry_argument_errors(gpu_device):
    scene = fresnel.Scene(device=gpu_device)
    with pytest.raises(RuntimeError, match="multiple of three"):
        fresnel.geometry.Mesh(scene, numpy.zeros((4, 3), numpy.float32), N=1)
    with pytest.raises(RuntimeError):
        fresnel.geometry.ConvexPolyhedron(scene, {'face_origin': numpy.zeros((3, 3)),
                                                  'face_normal': numpy.zeros((2, 3)),
                                                  'face_color': numpy.zeros((3, 3)),
                                                  'radius': 1.0}, N=1)
    with pytest.raises(RuntimeError, match="Nvert by 2"):
        fresnel.geometry.Polygon(scene, vertices=[[0, 0, 0], [1, 0, 0], [0, 1, 0]],
                                 position=[[0, 0]])


def test_light_proxy_and_camera(gpu_device):
    scene = fresnel.Scene(device=gpu_device)
    lights = scene.lights
    assert len(lights) == 2
    scene.lights = [fresnel.light.Light(direction=(1, 2, 3))]
    assert len(lights) == 1 and lights[0].direction == (1, 2, 3)
    with pytest.raises(IndexError):
        scene.lights = [fresnel.light.Light(direction=(1, 0, 0))] * 5
    cam = fresnel.camera.Perspective(position=(0, 0, -10), look_at=(0, 0, 0), up=(0, 1, 0),
                                     focal_length=1.25, focus_distance=20, height=0.25,
                                     f_stop=1.5)
    scene.camera = cam
    assert scene.camera.focal_length == 1.25 and scene.camera.f_stop == 1.5
    scene.camera.height = 0.5
    assert scene.camera.height == 0.5
    assert math.isclose(cam.vertical_field_of_view, 2 * math.atan(0.25 / 2.5))


def test_stats_count_rays(gpu_device):
    scene = workloads.hex_spheres(gpu_device)
    t = fresnel.tracer.Path(device=gpu_device, w=20, h=10)
    t._tracer.resetStats()
    t.sample(scene, samples=3, light_samples=2)
    st = t._tracer.getStats()
    assert st["paths"] == 20 * 10 * 3 * 2
    assert st["rays"] >= 20 * 10 * 3


def test_reading_arrays_rebuilds_nothing(gpu_device):
    """Reading a geometry array (the whole array or a part) leaves its device copy and the
    acceleration structure as they are; a write rebuilds."""
    scene = workloads.hex_spheres(gpu_device)
    t = fresnel.tracer.Preview(device=gpu_device, w=48, h=48, anti_alias=False)
    first = t.render(scene)[:]
    st = t._tracer.getStats()
    built = st["bvh_builds"] + st["grid_builds"]
    g = scene.geometry[0]
    pos, rad, col = g.position[:], g.radius[:], g.color[:]
    assert g.position[2:4].shape == (2, 3)
    again = t.render(scene)[:]
    st = t._tracer.getStats()
    assert st["bvh_builds"] + st["grid_builds"] == built
    assert numpy.array_equal(first, again)
    g.position[:] = pos
    t.render(scene)
    st = t._tracer.getStats()
    assert st["bvh_builds"] + st["grid_builds"] == built + 1
    assert rad.shape == (pos.shape[0],) and col.shape == pos.shape


def test_output_reads_are_independent_copies(gpu_device):
    """A whole read of a tracer output (downloaded straight into the returned array) equals the
    mapped buffer's contents, and each read is a copy of its own that later renders leave as
    is."""
    scene = workloads.hex_spheres(gpu_device)
    t = fresnel.tracer.Path(device=gpu_device, w=40, h=30)
    t.sample(scene, samples=2)
    for arr in (t.output, t.linear_output):
        a = arr[:]
        arr.buf.map()
        mapped = numpy.array(arr.buf, copy=True)
        arr.buf.unmap()
        assert a.dtype == mapped.dtype and a.shape == mapped.shape
        assert numpy.array_equal(a, mapped, equal_nan=True)
        b = arr[...]
        assert not numpy.may_share_memory(a, b) and numpy.array_equal(a, b, equal_nan=True)
    kept = t.output[:]
    copy = kept.copy()
    del a, b
    scene.background_color = (0.9, 0.1, 0.1)
    scene.background_alpha = 1.0
    t.sample(scene, samples=1)
    later = t.output[:]
    assert numpy.array_equal(kept, copy) and not numpy.array_equal(later, kept)


def test_whole_and_partial_array_writes_render_alike(gpu_device):
    """Whole writes of large arrays (row blocks on the copy threads, streaming stores) give the
    renders that the same arrays written part by part give, also when an array is written twice
    before a render; a read between write and render sees the write."""
    n = 400_000  # positions and colours above the 4 MB of a threaded copy, radii below
    rng = numpy.random.default_rng(11)
    pos = [rng.uniform(-30, 30, (n, 3)).astype(numpy.float32) for _ in range(2)]
    col = rng.uniform(0, 1, (n, 3)).astype(numpy.float32)
    rad = rng.uniform(0.2, 0.6, n).astype(numpy.float32)

    def scene(parts):
        s = fresnel.Scene(device=gpu_device)
        g = fresnel.geometry.Sphere(s, N=n, material=fresnel.material.Material(
            primitive_color_mix=1.0, roughness=0.5))
        if parts == 1:
            g.position[:], g.color[:], g.radius[:] = pos[0], col, rad
        for k in range(0, n, n // parts) if parts > 1 else ():
            g.position[k:k + n // parts] = pos[0][k:k + n // parts]
            g.color[k:k + n // parts] = col[k:k + n // parts]
            g.radius[k:k + n // parts] = rad[k:k + n // parts]
        s.camera = fresnel.camera.Orthographic.fit(s)
        return s, g
    s_lazy, g_lazy = scene(4)  # partial writes
    s_q, g_q = scene(1)        # whole writes
    assert numpy.array_equal(g_q.position[:], pos[0])
    t = fresnel.tracer.Preview(device=gpu_device, w=96, h=96, anti_alias=False)
    a = t.render(s_lazy)[:]
    t_q = fresnel.tracer.Preview(device=gpu_device, w=96, h=96, anti_alias=False)
    b = t_q.render(s_q)[:]
    assert a[..., 3].max() == 255 and numpy.array_equal(a, b)
    g_q.position[:] = pos[1]
    g_q.position[:] = pos[0]  # written again before the render: the last write wins
    assert numpy.array_equal(g_q.position[:], pos[0])
    assert numpy.array_equal(t_q.render(s_q)[:], a)
    g_q.position[:] = pos[1]
    g_lazy.position[0:n] = pos[1]
    assert numpy.array_equal(t_q.render(s_q)[:], t.render(s_lazy)[:])
