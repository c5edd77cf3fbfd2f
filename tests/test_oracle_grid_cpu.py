"""The oracle's restatements of the engine's uniform grids (oracle_core.cpp: build_sphere_grid,
walk_sphere_grid for the sphere grid; build_count_grid, walk_count_grid for the grid over a
scene's parts), used to freeze the grids' per-ray costs in bench.py's roofline.  The sphere
grid's walk must find the same closest sphere as the oracle's BVH on every logged ray; on a scene
of one sphere geometry the parts walk (which ends at the BVH's closest hit) must count exactly
the cells and spheres the sphere walk (which finds its own hits) does; and on the benchmark
frames the costs must reproduce the frozen values."""

import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from oracle import measure_ray_costs  # noqa: E402


def _small_sphere_costs():
    import bench
    from fresnel_b200 import workloads
    wl = bench.WORKLOADS["c2"]
    old = wl.scene
    bench.WORKLOADS["c2s"] = bench.Workload("c2s", "scaled", "config2", 320, 180)
    try:
        workloads.config2_small = lambda d: workloads.config2(d, n=20000,
                                                              box=140.0 * 0.02**(1 / 3))
        bench.WORKLOADS["c2s"].scene = "config2_small"
        res = measure_ray_costs.grid_costs("c2s", n_pixels=1024, spp=2)
        parts = measure_ray_costs.parts_grid_costs("c2s", n_pixels=1024, spp=2)
    finally:
        bench.WORKLOADS.pop("c2s", None)
        del workloads.config2_small
    assert wl.scene == old
    return res, parts


def test_grid_walk_finds_the_bvh_hits_small():
    res, parts = _small_sphere_costs()
    assert res["rays"] > 1000
    assert res["rays_hitting_differently"] == 0
    assert 1.0 < res["cells_per_ray"] < 10.0
    # one sphere geometry: the grid over parts is the sphere grid, walked to the same hits
    assert parts["rays"] == res["rays"]
    assert parts["cells"] == res["cells"] and parts["refs"] == res["refs"]
    assert parts["cells_per_ray"] == pytest.approx(res["cells_per_ray"], rel=1e-12)
    assert parts["refs_per_ray"] == pytest.approx(res["spheres_per_ray"], rel=1e-12)


def test_parts_grid_walk_small_mixed_scene():
    import bench
    bench.WORKLOADS["c3s"] = bench.Workload("c3s", "scaled", "config3", 320, 180)
    from fresnel_b200 import workloads
    try:
        workloads.config3_small = lambda d: workloads.config3(d, scale=0.02)
        bench.WORKLOADS["c3s"].scene = "config3_small"
        res = measure_ray_costs.parts_grid_costs("c3s", n_pixels=2048, spp=2)
    finally:
        bench.WORKLOADS.pop("c3s", None)
        del workloads.config3_small
    assert res["rays"] > 1000
    assert 1.0 < res["cells_per_ray"] < 20.0
    assert res["refs_per_ray"] > 0.5
    assert res["refs"] >= res["cells"] // 4


@pytest.mark.slow
def test_frozen_grid_costs_of_the_1m_sphere_frame():
    import bench
    wl = bench.WORKLOADS["c2"]
    res = measure_ray_costs.grid_costs("c2", n_pixels=4096, spp=4)
    assert res["rays_hitting_differently"] == 0
    # a smaller sample than the frozen one: within a few percent
    assert abs(res["cells_per_ray"] - wl.grid_cells) <= 0.05 * wl.grid_cells
    assert abs(res["spheres_per_ray"] - wl.grid_spheres) <= 0.05 * wl.grid_spheres


@pytest.mark.slow
def test_frozen_parts_grid_costs_of_the_mixed_scene():
    import bench
    wl = bench.WORKLOADS["c3"]
    res = measure_ray_costs.parts_grid_costs("c3", n_pixels=4096, spp=4)
    # a smaller sample than the frozen one: within a few percent
    assert abs(res["cells_per_ray"] - wl.grid_cells) <= 0.05 * wl.grid_cells
    assert abs(res["refs_per_ray"] - wl.grid_refs) <= 0.05 * wl.grid_refs
