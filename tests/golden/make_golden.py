"""Regenerate the golden fixtures in this directory with the CPU oracle.

The oracle is pinned to the reference first (tests/test_oracle_pinning.py: bit-identical to the
reference's own fresnel/common math and passing the reference's golden-image suite); these
fixtures then freeze its outputs so that the GPU tests can check against them on a machine
without the reference tree.  Run ``python tests/golden/make_golden.py``.
"""

import os
import sys

import numpy

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.dirname(HERE))

from fresnel_b200 import workloads  # noqa: E402
from oracle import cpu_module  # noqa: E402
from parity import path_render, preview_hits  # noqa: E402

CASES = {
    # name: (scene builder, kind, w, h, options)
    "hex_preview": (workloads.hex_spheres, "preview", 100, 100, {"aa_n": 1}),
    "hex_preview_aa": (workloads.hex_spheres, "preview", 100, 100, {"aa_n": 3}),
    "mixed_preview": (lambda d: workloads.config3(d, scale=0.002), "preview", 96, 54,
                      {"aa_n": 1}),
    "spheres_1k_path": (workloads.config1, "path", 64, 64,
                        {"samples": 8, "light_samples": 2, "seed": 5}),
    "dense_path": (lambda d: workloads.config2(d, n=5000, box=140.0 * (0.005)**(1 / 3)), "path",
                   64, 36, {"samples": 8, "light_samples": 1, "seed": 1}),
    "polygons_preview": (lambda d: workloads.polygons(d, spheres=30), "preview", 96, 72,
                         {"aa_n": 2}),
    "polygons_path": (lambda d: workloads.polygons(d, nx=10, ny=8, spheres=20), "path", 64, 48,
                      {"samples": 6, "light_samples": 1, "seed": 3}),
}


def render(name, device):
    build, kind, w, h, opt = CASES[name]
    scene = build(device)
    if kind == "preview":
        hits, lin, srgb = preview_hits(device, scene, w, h, opt["aa_n"])
        return {"hits": hits, "linear": lin, "srgb": srgb}
    lin, srgb, _ = path_render(device, scene, w, h, opt["samples"], opt["light_samples"],
                               seed=opt["seed"])
    return {"linear": lin, "srgb": srgb}


def main():
    dev = cpu_module.make_device("restated")
    for name in CASES:
        out = render(name, dev)
        numpy.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
