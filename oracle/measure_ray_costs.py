"""Measure the per-ray traversal costs used by bench.py's roofline (TEST INFRASTRUCTURE).

Renders a seeded random subset of pixels of the 1M-sphere 1080p benchmark frame with the CPU
oracle (binned-SAH BVH2, leaves of at most 4 primitives) and reports, per closest-hit query,
the mean number of AABB tests (A) and primitive tests (P).  bench.py freezes these values:
algorithmic bytes per ray = 24 + 16 + 32 A + 16 P + 12.

Run: python oracle/measure_ray_costs.py [n_pixels] [spp]
"""

import os
import sys
import time

import numpy

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)


def main(n_pixels=20000, spp=2):
    from fresnel_b200 import workloads
    from oracle import cpu_module
    dev = cpu_module.make_device("restated")
    t0 = time.perf_counter()
    scene = workloads.config2(dev)
    nodes, prims = scene._scene.info()
    t1 = time.perf_counter()
    tr = dev.module.TracerPath(dev._device, 1920, 1080, 1)
    tr.setSeed(2)
    rng = numpy.random.default_rng(0)
    pixels = numpy.sort(rng.choice(1920 * 1080, n_pixels, replace=False)).astype(numpy.uint32)
    tr.stats = cpu_module.OrStats()
    tr.render_pixels(scene._scene, pixels, 1, spp, want_m2=False)
    t2 = time.perf_counter()
    s = tr.stats.as_dict()
    print(f"BVH: {nodes} nodes over {prims} primitives, build {t1 - t0:.1f} s")
    print(f"{s['rays']} rays, {s['paths']} paths, {s['rays'] / s['paths']:.3f} rays per path")
    print(f"A (box tests per ray)  = {s['box_tests'] / s['rays']:.2f}")
    print(f"P (prim tests per ray) = {s['prim_tests'] / s['rays']:.2f}")
    print(f"{s['rays'] / (t2 - t1) / 1e6:.2f} Mrays/s on {os.cpu_count()} threads")


if __name__ == "__main__":
    main(*(int(x) for x in sys.argv[1:3]))
