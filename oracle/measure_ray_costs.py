"""Measure the per-ray traversal costs used by bench.py's roofline (TEST INFRASTRUCTURE).

Renders a seeded sample of a benchmark frame with the CPU oracle (binned-SAH BVH2, leaves of at
most 4 primitives) and reports, per closest-hit query, the mean number of AABB tests (A) and
primitive tests (P).  bench.py freezes these values per workload:
algorithmic bytes per ray = 24 + 16 + 32 A + prim_bytes P + 12.

Path workloads: n_pixels random pixels of the frame, spp samples each.  Preview: the frame at
1/8 of the resolution in each direction with the workload's AA level (same camera).

Run: python oracle/measure_ray_costs.py [workload] [n_pixels] [spp]   (workload: c1, c2, c3,
c2-preview; default c2)
"""

import os
import sys
import time

import numpy

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)


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


if __name__ == "__main__":
    a = sys.argv[1:]
    main(a[0] if a else "c2", *(int(x) for x in a[1:3]))
