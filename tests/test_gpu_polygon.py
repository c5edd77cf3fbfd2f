"""Polygon geometry on the GPU: the scenes of fresnel's own polygon tests
(fresnel/test/test_geometry_polygon.py) against the CPU oracle, which passes that file's
golden-image comparisons, and the Python API of geometry.Polygon (fresnel/geometry.py:391-501).
"""

import math

import numpy
import pytest

import fresnel_b200 as fresnel
from grazing import check_hits
from parity import preview_hits

pytestmark = pytest.mark.gpu

OUTLINE = [[-1, -1], [1, -1], [1, 1], [0, 0], [-1, 1]]


def _test_lights():
    # the lights of fresnel/test/conftest.py (two directional lights)
    return [fresnel.light.Light(direction=(math.sin(70 * math.pi / 180) * math.sin(45 * math.pi / 180),
                                           math.cos(70 * math.pi / 180),
                                           math.sin(70 * math.pi / 180) * math.cos(45 * math.pi / 180)),
                                color=(0.75, 0.75, 0.75), theta=math.pi / 8),
            fresnel.light.Light(direction=(math.sin(math.pi / 2) * math.sin(-math.pi / 4),
                                           math.cos(math.pi / 2),
                                           math.sin(math.pi / 2) * math.cos(-math.pi / 4)),
                                color=(0.1, 0.1, 0.1), theta=math.pi / 2)]


def reference_scene(device, rounding_radius, outline_width=0.0):
    """The two polygons of fresnel/test/test_geometry_polygon.py:18-75."""
    scene = fresnel.Scene(device, lights=_test_lights())
    mat = fresnel.material.Material(color=fresnel.color.linear([0.42, 0.267, 1]), solid=1)
    fresnel.geometry.Polygon(scene, N=2, rounding_radius=rounding_radius, vertices=OUTLINE,
                             position=[[-1.5, 0], [1.5, 0]], angle=[0.1, -0.2],
                             color=[[0, 0, 1], [0, 1, 0]], material=mat,
                             outline_width=outline_width)
    scene.camera = fresnel.camera.Orthographic(position=(0, 0, -2), look_at=(0, 0, 0),
                                               up=(0, 1, 0), height=5)
    return scene


@pytest.mark.parametrize("rounding_radius,outline", [(0.0, 0.0), (0.3, 0.1)],
                         ids=["sharp", "rounded_outline"])
@pytest.mark.parametrize("aa_n", [1, 3])
def test_reference_scenes_match_oracle(rounding_radius, outline, aa_n, gpu_device,
                                       oracle_device):
    w, h = 150, 100
    gh, gl, g8 = preview_hits(gpu_device, reference_scene(gpu_device, rounding_radius, outline),
                              w, h, aa_n)
    oscene = reference_scene(oracle_device, rounding_radius, outline)
    oh, ol, o8 = preview_hits(oracle_device, oscene, w, h, aa_n)
    assert numpy.count_nonzero(oh[..., 0]) > 0
    mism = check_hits("test_reference_scenes_match_oracle", oracle_device, oscene, w, h, aa_n,
                      gh, oh, scene=f"polygons r={rounding_radius} outline={outline}")
    agree = ~numpy.any(mism, axis=-1)
    assert numpy.abs(gl - ol)[agree].max() <= 1e-3
    assert numpy.all(g8 == o8, axis=-1)[agree].mean() >= 0.999


def test_polygon_attributes(gpu_device):
    # fresnel/test/test_geometry_polygon.py:84-130: arrays round trip, extents
    scene = reference_scene(gpu_device, 0.3)
    g = scene.geometry[0]
    a = numpy.array([-0.8, 0.5], dtype=numpy.float32)
    g.angle[:] = a
    numpy.testing.assert_array_equal(g.angle[:], a)
    p = numpy.array([[1.5, 2.5], [-3, 4]], dtype=numpy.float32)
    g.position[:] = p
    numpy.testing.assert_array_equal(g.position[:], p)
    c = numpy.array([[0.1, 0.2, 0.3], [0.4, 0.5, 0.6]], dtype=numpy.float32)
    g.color[:] = c
    numpy.testing.assert_array_equal(g.color[:], c)
    r = g._geometry.getRadius()
    assert r == pytest.approx(math.sqrt(2) + 0.3, rel=1e-6)
    ext = g.get_extents()
    numpy.testing.assert_allclose(ext, [[-3 - r, 2.5 - r, -1e-5], [1.5 + r, 4 + r, 1e-5]],
                                  rtol=1e-6)
    # the renderer sees the new angles and positions
    t = fresnel.tracer.Preview(gpu_device, w=64, h=48, anti_alias=False)
    t.render(scene)
    assert t.output[:].shape == (48, 64, 4)


def test_polygon_argument_errors(gpu_device):
    scene = fresnel.Scene(gpu_device)
    with pytest.raises(RuntimeError, match="2-dimensional"):
        fresnel.geometry.Polygon(scene, vertices=[1, 2, 3, 4], position=[[0, 0]])
    with pytest.raises(RuntimeError, match="Nvert by 2"):
        fresnel.geometry.Polygon(scene, vertices=[[0, 0, 0], [1, 0, 0], [0, 1, 0]],
                                 position=[[0, 0]])


def test_rotating_polygons_rebuilds_their_tree(gpu_device, oracle_device):
    # after the angles change, hits follow the new orientation (tree rebuilt or refitted)
    from fresnel_b200 import workloads
    scenes = [workloads.polygons(d, nx=6, ny=4, perspective=False) for d in
              (gpu_device, oracle_device)]
    preview_hits(gpu_device, scenes[0], 90, 60, 1)
    rng = numpy.random.default_rng(11)
    ang = rng.uniform(-3, 3, 24).astype(numpy.float32)
    for s in scenes:
        s.geometry[0].angle[:] = ang
    gh, gl, _ = preview_hits(gpu_device, scenes[0], 90, 60, 1)
    oh, ol, _ = preview_hits(oracle_device, scenes[1], 90, 60, 1)
    check_hits("test_rotating_polygons_rebuilds_their_tree", oracle_device, scenes[1], 90, 60,
               1, gh, oh, scene="polygons rotated")
