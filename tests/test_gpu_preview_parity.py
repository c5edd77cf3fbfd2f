"""Preview tracer on the GPU versus the CPU oracle: closest-hit ids and linear RGB.

Bars (from the reference CPU path as normative): hit ids bit-exact except at grazing samples --
every disagreement is classified with the oracle (tests/grazing.py: an exact or rounding-level
tie in t between the two primitives, or a ray within rounding of a silhouette) and none may be
non-grazing; all disagreements together stay at or below 1e-4 of the samples (each measured
rate is written through parity_record); linear RGB within 1e-3 wherever the hits agree; sRGB
bytes equal on at
least 99.9% of pixels (transcendental functions differ in the last place between CUDA and the
host libm).
"""

import numpy
import pytest

import fresnel_b200 as fresnel
from fresnel_b200 import workloads
from grazing import check_hits
from parity import odd_radii_scene, preview_hits

pytestmark = pytest.mark.gpu

RGB_TOL = 1e-3


def _dense(d):
    n = 20000
    return workloads.config2(d, n=n, box=140.0 * (n / 1e6)**(1 / 3))


SCENES = {
    "hex_spheres": (workloads.hex_spheres, 100, 100),
    "spheres_1k": (workloads.config1, 160, 160),
    "dense_spheres": (_dense, 192, 108),
    "mixed": (lambda d: workloads.config3(d, scale=0.002), 160, 90),
    "mixed_large": (lambda d: workloads.config3(d, scale=0.02), 128, 72),
    "odd_radii": (odd_radii_scene, 120, 120),
    "polygons": (workloads.polygons, 160, 120),
    "polygons_spheres": (lambda d: workloads.polygons(d, spheres=60), 160, 120),
    "polygons_ortho": (lambda d: workloads.polygons(d, perspective=False, rounding_radius=0.0),
                       150, 112),
}


@pytest.fixture(params=[0, 1], ids=["lbvh", "ploc"])
def builder(request, gpu_device):
    """Run with each BVH builder of the engine (the oracle keeps its own SAH tree)."""
    dd = gpu_device._device
    old = dd.getOption("builder")
    dd.setOption("builder", request.param)
    yield request.param
    dd.setOption("builder", old)


@pytest.mark.parametrize("aa_n", [1, 3])
@pytest.mark.parametrize("name", list(SCENES))
def test_preview_matches_oracle(name, aa_n, builder, gpu_device, oracle_device):
    build, w, h = SCENES[name]
    gh, gl, g8 = preview_hits(gpu_device, build(gpu_device), w, h, aa_n)
    oscene = build(oracle_device)
    oh, ol, o8 = preview_hits(oracle_device, oscene, w, h, aa_n)
    assert gh.shape == oh.shape
    assert numpy.count_nonzero(oh[..., 0]) > 0, "scene shows no geometry"
    mism = check_hits("test_preview_matches_oracle", oracle_device, oscene, w, h, aa_n, gh, oh,
                      scene=name, builder=("lbvh", "ploc")[builder])
    agree = ~numpy.any(mism, axis=-1)
    err = numpy.abs(gl - ol)[agree].max()
    assert err <= RGB_TOL, f"linear RGB differs by {err}"
    same = numpy.all(g8 == o8, axis=-1)[agree].mean()
    assert same >= 0.999, f"only {same:.4%} of sRGB pixels identical"


def test_coincident_primitives(builder, gpu_device, oracle_device):
    rng = numpy.random.default_rng(7)
    centres = rng.uniform(-6, 6, (40, 3)).astype(numpy.float32)
    pos = numpy.repeat(centres, 100, axis=0)
    w, h = 96, 96
    imgs = []
    for dev in (gpu_device, oracle_device):
        scene = fresnel.Scene(dev)
        fresnel.geometry.Sphere(scene, position=pos, radius=0.6, color=(0.2, 0.5, 0.8),
                                material=fresnel.material.Material(color=(0.9, 0.3, 0.1)))
        scene.camera = fresnel.camera.Orthographic.fit(scene)
        imgs.append(preview_hits(dev, scene, w, h, 1))
    (gh, gl, _), (oh, ol, _) = imgs
    # the same sphere copy need not win a tie, but every pixel sees the same surface
    assert numpy.array_equal(gh[..., 0] != 0, oh[..., 0] != 0)
    assert numpy.abs(gl - ol).max() <= RGB_TOL
