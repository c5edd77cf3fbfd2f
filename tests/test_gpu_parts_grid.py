"""Scenes of several geometries (or of one geometry that is not spheres) traced through the grid
over their parts (device option "accel": 1 forces it, 2 chooses it unless the primitives are
clustered or sparse; a mesh is referenced by instance)
against the CPU oracle: the same closest hits (exact-t ties and rays grazing a silhouette aside,
classified by tests/grazing.py), same-seed path images within the oracle's bar, the same images
as the trees give, and the automatic choice.
"""

import numpy
import pytest

from fresnel_b200 import workloads
from grazing import check_hits
from parity import odd_radii_scene, path_render, preview_hits

pytestmark = pytest.mark.gpu

PARTS_GRID = 2  # getAccel()[0] of a grid over parts (1: sphere grid, 0: trees)


@pytest.fixture
def accel(gpu_device):
    dd = gpu_device._device
    old = dd.getOption("accel")

    def set_(v):
        dd.setOption("accel", v)
    yield set_
    dd.setOption("accel", old)


def _spheres_bonds(d):
    # a serving-request scene: 80% spheres (r 0.3-0.7), 20% bonds between neighbours
    return workloads.serving_scene(d, 6000, 3)


def _mixed(d):
    # spheres, bonds, cubes and icosahedra (the mixed benchmark scene at 2% of its counts)
    return workloads.config3(d, scale=0.02)


def _polygons_and_spheres(d):
    return workloads.polygons(d, nx=12, ny=9, spheres=40)


def _icosahedra(d):
    # one mesh geometry alone (20 triangles per instance)
    s = workloads.config3(d, scale=0.05)
    for g in s.geometry:
        if type(g).__name__ != "Mesh":
            g.disable()
    return s


def _mixed_without_mesh(d):
    s = _mixed(d)
    for g in s.geometry:
        if type(g).__name__ == "Mesh":
            g.disable()
    return s


# name: (builder, width, height, accel mode that must give the parts grid)
SCENES = {
    "spheres_bonds": (_spheres_bonds, 160, 90, 2),
    "mixed": (_mixed, 160, 90, 2),
    "polygons_and_spheres": (_polygons_and_spheres, 128, 96, 2),
    "icosahedra": (_icosahedra, 128, 96, 2),
    "mixed_without_mesh": (_mixed_without_mesh, 160, 90, 2),
    "odd_radii": (odd_radii_scene, 120, 120, 2),
}


@pytest.mark.parametrize("aa_n", [1, 2])
@pytest.mark.parametrize("name", list(SCENES))
def test_parts_grid_matches_oracle(name, aa_n, accel, gpu_device, oracle_device):
    build, w, h, mode = SCENES[name]
    accel(mode)
    scene = build(gpu_device)
    gh, gl, g8 = preview_hits(gpu_device, scene, w, h, aa_n)
    assert scene._scene.getAccel()[0] == PARTS_GRID, scene._scene.getAccel()
    oscene = build(oracle_device)
    oh, ol, o8 = preview_hits(oracle_device, oscene, w, h, aa_n)
    assert numpy.count_nonzero(oh[..., 0]) > 0
    mism = check_hits("test_parts_grid_matches_oracle", oracle_device, oscene, w, h, aa_n, gh, oh,
                      scene=name, structure="parts grid")
    agree = ~numpy.any(mism, axis=-1)
    assert numpy.abs(gl - ol)[agree].max() <= 1e-3


@pytest.mark.parametrize("name", ["spheres_bonds", "mixed"])
def test_parts_grid_path_same_seed(name, accel, gpu_device, oracle_device):
    build, _, _, mode = SCENES[name]
    accel(mode)
    gl, g8, gt = path_render(gpu_device, build(gpu_device), 96, 54, 6, 1, seed=7)
    assert gt._tracer.getStats()["grid"] == PARTS_GRID
    ol, o8, _ = path_render(oracle_device, build(oracle_device), 96, 54, 6, 1, seed=7)
    close = numpy.all(numpy.abs(gl - ol) <= 1e-3, axis=-1).mean()
    assert close >= 0.99, f"only {close:.4%} of pixels within 1e-3"
    assert numpy.all(g8[..., 3] == o8[..., 3])


@pytest.mark.parametrize("name", ["spheres_bonds", "mixed"])
def test_parts_grid_and_trees_give_the_same_image(name, accel, gpu_device):
    build, _, _, mode = SCENES[name]
    scene = build(gpu_device)
    out = []
    for m in (0, mode):
        accel(m)
        lin, _, t = path_render(gpu_device, scene, 96, 64, 8, 1, seed=3)
        assert t._tracer.getStats()["grid"] == (PARTS_GRID if m else 0)
        out.append(lin)
    close = numpy.all(numpy.abs(out[0] - out[1]) <= 1e-6, axis=-1).mean()
    assert close >= 0.999, f"only {close:.4%} of pixels agree"


def test_automatic_choice_over_parts(accel, gpu_device):
    accel(2)
    cases = {
        "spheres_bonds": (_spheres_bonds, PARTS_GRID),
        "mixed": (_mixed, PARTS_GRID),
        "mixed_without_mesh": (_mixed_without_mesh, PARTS_GRID),
        "polygons_and_spheres": (_polygons_and_spheres, PARTS_GRID),
        "icosahedra": (_icosahedra, PARTS_GRID),
    }
    for name, (build, kind) in cases.items():
        scene = build(gpu_device)
        preview_hits(gpu_device, scene, 32, 32, 1)
        got, why = scene._scene.getAccel()
        assert got == kind, (name, why)


def test_parts_grid_follows_moving_primitives(accel, gpu_device, oracle_device):
    accel(2)
    scenes = [_spheres_bonds(d) for d in (gpu_device, oracle_device)]
    preview_hits(gpu_device, scenes[0], 96, 64, 1)
    rng = numpy.random.default_rng(9)
    sph = scenes[0].geometry[0].position[:]
    moved = (sph + rng.uniform(-1, 1, sph.shape)).astype(numpy.float32)
    pts = scenes[0].geometry[1].points[:]
    moved_pts = (pts + rng.uniform(-1, 1, (pts.shape[0], 1, 3))).astype(numpy.float32)
    for s in scenes:
        s.geometry[0].position[:] = moved
        s.geometry[1].points[:] = moved_pts
    gh, _, _ = preview_hits(gpu_device, scenes[0], 96, 64, 1)
    assert scenes[0]._scene.getAccel()[0] == PARTS_GRID
    oh, _, _ = preview_hits(oracle_device, scenes[1], 96, 64, 1)
    check_hits("test_parts_grid_follows_moving_primitives", oracle_device, scenes[1], 96, 64, 1,
               gh, oh, scene="spheres_bonds moved", structure="parts grid")


def test_parts_grid_follows_enabled_geometries(accel, gpu_device, oracle_device):
    """Disabling and enabling geometries changes the grid's parts: each render's hit ids match
    the oracle's on the same enabled set (the grid is rebuilt over the new parts each time)."""
    accel(2)
    scenes = [_mixed(d) for d in (gpu_device, oracle_device)]
    for step, off in enumerate([(), (3,), (0, 2), ()]):
        for s in scenes:
            for i, g in enumerate(s.geometry):
                if i in off:
                    g.disable()
                else:
                    g.enable()
        gh, _, _ = preview_hits(gpu_device, scenes[0], 96, 64, 1)
        assert scenes[0]._scene.getAccel()[0] == PARTS_GRID
        oh, _, _ = preview_hits(oracle_device, scenes[1], 96, 64, 1)
        check_hits("test_parts_grid_follows_enabled_geometries", oracle_device, scenes[1], 96,
                   64, 1, gh, oh, scene=f"mixed, disabled {off}", structure="parts grid")
