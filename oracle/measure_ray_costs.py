"""Measure the per-ray traversal costs used by bench.py's roofline (TEST INFRASTRUCTURE).

Renders a seeded sample of a benchmark frame with the CPU oracle (binned-SAH BVH2, leaves of at
most 4 primitives) and reports, per closest-hit query, the mean number of AABB tests (A) and
primitive tests (P).  bench.py freezes these values per workload:
algorithmic bytes per ray = 24 + 16 + 32 A + prim_bytes P + 12.

Path workloads: n_pixels random pixels of the frame, spp samples each.  Preview: the frame at
1/8 of the resolution in each direction with the workload's AA level (same camera).

Sphere-grid costs (``--grid``): the same render with the oracle's ray log on, then every logged
ray walked through the oracle's restatement of the engine's uniform sphere grid (1.5 cells per
sphere, oracle_core.cpp: build_sphere_grid / walk_sphere_grid): cells visited (C) and spheres
tested (S) per ray, and the number of rays whose grid hit differs from the oracle's BVH hit.
bench.py freezes C and S for the sphere-grid roofline: bytes per ray = 52 + 8 C + 16 S.

Grid-over-parts costs (``--parts-grid``): the same, walked through the oracle's restatement of
the engine's grid over the scene's parts (every enabled geometry's primitives, a mesh by
instance; oracle_core.cpp: build_count_grid / walk_count_grid) up to the oracle's closest hit:
cells visited (C) and references listed in them (R) per ray.  bench.py freezes C and R for that
roofline: bytes per ray = 52 + 8 C + 36 R.

Run: python oracle/measure_ray_costs.py [workload] [n_pixels] [spp] [--grid | --parts-grid]
(workload: c1, c2, c3, c2-preview; default c2)
"""

import os
import sys
import time

import numpy

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)


def _ray_log(dev, scene, wl, n_pixels, spp, max_rays):
    """The rays an oracle render of n_pixels seeded pixels x spp samples traces: [n, 7] float32
    (origin, direction, tnear)."""
    from oracle import cpu_module
    lib = dev._device.lib
    log = numpy.zeros((max_rays, 7), numpy.float32)
    tr = dev.module.TracerPath(dev._device, wl.w, wl.h, wl.light_samples)
    tr.setSeed(2)
    rng = numpy.random.default_rng(0)
    pixels = numpy.sort(rng.choice(wl.w * wl.h, min(n_pixels, wl.w * wl.h),
                                   replace=False)).astype(numpy.uint32)
    lib.or_set_ray_log(cpu_module.ptr(log), max_rays)
    try:
        tr.render_pixels(scene._scene, pixels, 1, int(spp), want_m2=False)
    finally:
        n = int(lib.or_ray_log_count())
        lib.or_set_ray_log(None, 0)
    return numpy.ascontiguousarray(log[:min(n, max_rays)])


def grid_costs(key="c2", n_pixels=4096, spp=4, cells_per_sphere=1.5, max_rays=2_000_000):
    """Cells and spheres per ray of the sphere grid, on the rays of an oracle render."""
    import ctypes

    import bench
    from oracle import cpu_module
    wl = bench.WORKLOADS[key]
    dev = cpu_module.make_device("restated")
    scene = wl.build(dev)
    scene._scene.handle()
    g = scene.geometry[0]
    pos = numpy.ascontiguousarray(g.position[:], dtype=numpy.float32)
    rad = numpy.ascontiguousarray(g.radius[:], dtype=numpy.float32)
    lib = dev._device.lib
    log = _ray_log(dev, scene, wl, n_pixels, spp, max_rays)
    n = len(log)
    out = (ctypes.c_double * 6)()
    rc = lib.or_grid_walk_stats(scene._scene.handle(), 0, cpu_module.ptr(pos), cpu_module.ptr(rad),
                                len(rad), float(cells_per_sphere), cpu_module.ptr(log), n, 0, out)
    if rc != 0:
        raise RuntimeError("grid construction failed")
    res = {"rays": int(out[0]), "cells_per_ray": out[1], "spheres_per_ray": out[2],
           "rays_hitting_differently": int(out[3]), "cells": int(out[4]), "refs": int(out[5]),
           "bytes_per_ray": 52 + 8 * out[1] + 16 * out[2]}
    print(f"workload {key}: {n_pixels} pixels x {spp} spp, {res['rays']} rays through a grid of "
          f"{res['cells']} cells and {res['refs']} sphere references")
    print(f"C (cells per ray)   = {res['cells_per_ray']:.3f}")
    print(f"S (spheres per ray) = {res['spheres_per_ray']:.3f}")
    print(f"bytes per ray = 52 + 8 C + 16 S = {res['bytes_per_ray']:.1f}")
    print(f"rays whose grid hit differs from the BVH hit: {res['rays_hitting_differently']}")
    return res


def main(key="c2", n_pixels=20000, spp=2):
    import bench
    from oracle import cpu_module
    wl = bench.WORKLOADS[key]
    dev = cpu_module.make_device("restated")
    t0 = time.perf_counter()
    scene = wl.build(dev)
    nodes, prims = scene._scene.info()
    t1 = time.perf_counter()
    if wl.preview:
        tr = dev.module.TracerDirect(dev._device, max(1, wl.w // 8), max(1, wl.h // 8))
        tr.setAntialiasingN(wl.aa_n)
        tr.stats = cpu_module.OrStats()
        tr.render(scene._scene)
    else:
        tr = dev.module.TracerPath(dev._device, wl.w, wl.h, wl.light_samples)
        tr.setSeed(2)
        rng = numpy.random.default_rng(0)
        n = min(int(n_pixels), wl.w * wl.h)
        pixels = numpy.sort(rng.choice(wl.w * wl.h, n, replace=False)).astype(numpy.uint32)
        tr.stats = cpu_module.OrStats()
        tr.render_pixels(scene._scene, pixels, 1, int(spp), want_m2=False)
    t2 = time.perf_counter()
    s = tr.stats.as_dict()
    print(f"workload {key}: BVH {nodes} nodes over {prims} primitives, build {t1 - t0:.1f} s")
    print(f"{s['rays']} rays, {s['paths']} paths")
    print(f"A (box tests per ray)  = {s['box_tests'] / s['rays']:.2f}")
    print(f"P (prim tests per ray) = {s['prim_tests'] / s['rays']:.2f}")
    print(f"{s['rays'] / (t2 - t1) / 1e6:.2f} Mrays/s on {os.cpu_count()} threads")


def parts_grid_costs(key="c3", n_pixels=4096, spp=4, cells_per_prim=1.5, max_rays=2_000_000):
    """Cells and references per ray of the grid over the scene's parts, on the rays of an
    oracle render."""
    import ctypes

    import bench
    from oracle import cpu_module
    wl = bench.WORKLOADS[key]
    dev = cpu_module.make_device("restated")
    scene = wl.build(dev)
    scene._scene.handle()
    lib = dev._device.lib
    log = _ray_log(dev, scene, wl, n_pixels, spp, max_rays)
    out = (ctypes.c_double * 5)()
    rc = lib.or_parts_grid_walk_stats(scene._scene.handle(), float(cells_per_prim),
                                      cpu_module.ptr(log), len(log), 0, out)
    if rc != 0:
        raise RuntimeError("grid construction failed")
    res = {"rays": int(out[0]), "cells_per_ray": out[1], "refs_per_ray": out[2],
           "cells": int(out[3]), "refs": int(out[4]),
           "bytes_per_ray": 52 + 8 * out[1] + 36 * out[2]}
    print(f"workload {key}: {n_pixels} pixels x {spp} spp, {res['rays']} rays through a grid of "
          f"{res['cells']} cells and {res['refs']} references")
    print(f"C (cells per ray)      = {res['cells_per_ray']:.3f}")
    print(f"R (references per ray) = {res['refs_per_ray']:.3f}")
    print(f"bytes per ray = 52 + 8 C + 36 R = {res['bytes_per_ray']:.1f}")
    return res


if __name__ == "__main__":
    a = [x for x in sys.argv[1:] if not x.startswith("--")]
    if "--grid" in sys.argv:
        grid_costs(a[0] if a else "c2", *(int(x) for x in a[1:3]))
    elif "--parts-grid" in sys.argv:
        parts_grid_costs(a[0] if a else "c3", *(int(x) for x in a[1:3]))
    else:
        main(a[0] if a else "c2", *(int(x) for x in a[1:3]))
