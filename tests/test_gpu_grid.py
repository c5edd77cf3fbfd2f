"""Sphere scenes traced through the uniform grid (device option "accel") against the CPU oracle
and against the BVH: the same closest hits (exact-t ties and rays grazing a silhouette aside,
classified by tests/grazing.py), the same path-traced images, and the automatic choice between
grid and BVH.
"""

import numpy
import pytest

import fresnel_b200 as fresnel
from fresnel_b200 import workloads
from grazing import check_hits
from parity import odd_radii_scene, path_render, preview_hits

pytestmark = pytest.mark.gpu


@pytest.fixture
def accel(gpu_device):
    dd = gpu_device._device
    old = dd.getOption("accel")

    def set_(v):
        dd.setOption("accel", v)
    yield set_
    dd.setOption("accel", old)


def _dense(d, n=20000):
    return workloads.config2(d, n=n, box=140.0 * (n / 1e6)**(1 / 3))


def _clustered(d):
    # most spheres in one small clump, a few spread over a large box
    rng = numpy.random.default_rng(4)
    pos = numpy.concatenate([rng.normal(0, 0.6, (9000, 3)), rng.uniform(-60, 60, (1000, 3))])
    scene = fresnel.Scene(d, lights=fresnel.light.lightbox())
    fresnel.geometry.Sphere(scene, position=pos.astype(numpy.float32), radius=0.3,
                            material=fresnel.material.Material(color=(0.8, 0.4, 0.2)))
    scene.camera = fresnel.camera.Orthographic.fit(scene)
    return scene


def _dense_with_clump(d):
    # an evenly filled box (the benchmark's density) plus a tight clump of 3000 spheres
    rng = numpy.random.default_rng(6)
    n = 20000
    box = 140.0 * (n / 1e6)**(1 / 3)
    pos = numpy.concatenate([rng.uniform(-box / 2, box / 2, (n, 3)),
                             rng.normal(0, 0.3, (3000, 3))])
    scene = fresnel.Scene(d, lights=fresnel.light.lightbox())
    fresnel.geometry.Sphere(scene, position=pos.astype(numpy.float32), radius=0.5)
    scene.camera = fresnel.camera.Orthographic.fit(scene)
    return scene


def _odd_radii(d):
    # the invalid-radius spheres alone (a grid needs a scene of one sphere geometry)
    scene = odd_radii_scene(d)
    scene.geometry[1].disable()
    return scene


def _inside(d):
    # perspective camera inside the cloud: primary rays start inside the grid
    scene = _dense(d)
    scene.camera = fresnel.camera.Perspective(position=(0.3, 0.2, 0.1), look_at=(5, 3, 2),
                                              up=(0, 0, 1), focal_length=0.5, height=0.6)
    return scene


SCENES = {
    "dense": (_dense, 160, 90),
    "hex": (workloads.hex_spheres, 100, 100),
    "spheres_1k": (workloads.config1, 128, 128),
    "clustered": (_clustered, 128, 128),
    "clump_in_box": (_dense_with_clump, 128, 128),
    "odd_radii": (_odd_radii, 120, 120),
    "inside": (_inside, 128, 96),
}


@pytest.mark.parametrize("aa_n", [1, 2])
@pytest.mark.parametrize("name", list(SCENES))
def test_forced_grid_matches_oracle(name, aa_n, accel, gpu_device, oracle_device):
    accel(1)
    build, w, h = SCENES[name]
    scene = build(gpu_device)
    gh, gl, g8 = preview_hits(gpu_device, scene, w, h, aa_n)
    assert scene._scene.getAccel()[0], scene._scene.getAccel()
    oscene = build(oracle_device)
    oh, ol, o8 = preview_hits(oracle_device, oscene, w, h, aa_n)
    assert numpy.count_nonzero(oh[..., 0]) > 0
    mism = check_hits("test_forced_grid_matches_oracle", oracle_device, oscene, w, h, aa_n, gh,
                      oh, scene=name, structure="sphere grid")
    agree = ~numpy.any(mism, axis=-1)
    assert numpy.abs(gl - ol)[agree].max() <= 1e-3


def test_grid_and_bvh_find_the_same_hits(accel, gpu_device):
    scene = _dense(gpu_device, 60000)
    out = []
    for mode in (0, 1):
        accel(mode)
        out.append(preview_hits(gpu_device, scene, 320, 180, 2))
        assert scene._scene.getAccel()[0] == (mode == 1)
    (ha, la, _), (hb, lb, _) = out
    same = numpy.all(ha == hb, axis=-1).mean()
    assert same >= 0.9999, f"{same:.5%} of hit ids agree"
    agree = numpy.all(numpy.all(ha == hb, axis=-1), axis=-1)
    assert numpy.abs(la - lb)[agree].max() <= 1e-6


def test_path_same_seed_with_grid(accel, gpu_device, oracle_device):
    accel(1)

    def build(d):
        return _dense(d, 20000)
    gl, g8, gt = path_render(gpu_device, build(gpu_device), 96, 54, 6, 1, seed=7)
    assert gt._tracer.getStats()["grid"] == 1
    ol, o8, _ = path_render(oracle_device, build(oracle_device), 96, 54, 6, 1, seed=7)
    close = numpy.all(numpy.abs(gl - ol) <= 1e-3, axis=-1).mean()
    assert close >= 0.99, f"only {close:.4%} of pixels within 1e-3"
    assert numpy.all(g8[..., 3] == o8[..., 3])


def test_automatic_choice(accel, gpu_device):
    accel(2)
    cases = {
        "dense": (_dense, True, ""),
        "spheres_1k": (workloads.config1, True, ""),
        "hex": (workloads.hex_spheres, True, ""),
        "sparse": (lambda d: workloads.random_spheres(d, 20000, 2000.0, 0.5, seed=3), True, ""),
        "clustered": (_dense_with_clump, False, "spheres too clustered"),
    }
    for name, (build, grid, reason) in cases.items():
        scene = build(gpu_device)
        preview_hits(gpu_device, scene, 32, 32, 1)
        got, why = scene._scene.getAccel()
        assert got == grid, (name, why)
        assert why == reason, (name, why)


def test_grid_follows_moving_spheres(accel, gpu_device, oracle_device):
    accel(1)
    scenes = [_dense(d, 12000) for d in (gpu_device, oracle_device)]
    preview_hits(gpu_device, scenes[0], 96, 64, 1)
    rng = numpy.random.default_rng(8)
    moved = (scenes[0].geometry[0].position[:] + rng.uniform(-3, 3, (12000, 3))).astype(
        numpy.float32)
    for s in scenes:
        s.geometry[0].position[:] = moved
    gh, _, _ = preview_hits(gpu_device, scenes[0], 96, 64, 1)
    oh, _, _ = preview_hits(oracle_device, scenes[1], 96, 64, 1)
    check_hits("test_grid_follows_moving_spheres", oracle_device, scenes[1], 96, 64, 1, gh, oh,
               scene="dense 12000 moved", structure="sphere grid")
    t = fresnel.tracer.Path(gpu_device, w=64, h=48)
    t.sample(scenes[0], samples=1)
    st = t._tracer.getStats()
    assert st["grid"] == 1 and st["grid_builds"] == 0  # built already by the preview render
