"""The oracle's restatement of the engine's uniform sphere grid (oracle_core.cpp:
build_sphere_grid, walk_sphere_grid), used to freeze the grid's per-ray costs in bench.py's
roofline.  Its walk must find the same closest sphere as the oracle's BVH on every logged ray,
and on the 1M-sphere frame its cells and spheres per ray must reproduce the frozen values."""

import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from oracle import measure_ray_costs  # noqa: E402


def test_grid_walk_finds_the_bvh_hits_small():
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
    finally:
        bench.WORKLOADS.pop("c2s", None)
        del workloads.config2_small
    assert wl.scene == old
    assert res["rays"] > 1000
    assert res["rays_hitting_differently"] == 0
    assert 1.0 < res["cells_per_ray"] < 10.0


@pytest.mark.slow
def test_frozen_grid_costs_of_the_1m_sphere_frame():
    import bench
    wl = bench.WORKLOADS["c2"]
    res = measure_ray_costs.grid_costs("c2", n_pixels=4096, spp=4)
    assert res["rays_hitting_differently"] == 0
    # a smaller sample than the frozen one: within a few percent
    assert abs(res["cells_per_ray"] - wl.grid_cells) <= 0.05 * wl.grid_cells
    assert abs(res["spheres_per_ray"] - wl.grid_spheres) <= 0.05 * wl.grid_spheres
