"""Traversal variants against one ray per thread: warp-cooperative primary rays (device option
"packet") and extension rays with per-lane refill (device option "refill").

Each lane of a packet tests exactly the leaves its own ray reaches, so the primary hits must be
the same as with one ray per thread (only primitives at exactly equal distance could be ordered
differently): the primary hit ids of a render's last wavefront must agree on at least 99.99% of
pixels and the images within 1e-5 on at least 99.9%, on a dense sphere scene, a small one with
outlines and the mixed-geometry scene (combined tree).
"""

import numpy
import pytest

import fresnel_b200 as fresnel
from fresnel_b200 import workloads

pytestmark = pytest.mark.gpu

SCENES = {
    "dense": (lambda d: workloads.config2(d, n=30000, box=140.0 * 0.03 ** (1 / 3)), 160, 120),
    "spheres_1k": (workloads.config1, 100, 100),
    "mixed": (lambda d: workloads.config3(d, scale=0.005), 128, 72),
}


@pytest.mark.parametrize("option", ["packet", "refill"])
@pytest.mark.parametrize("name", list(SCENES))
def test_variant_matches_per_ray(name, option, gpu_device):
    build, w, h = SCENES[name]
    dd = gpu_device._device
    old = dd.getOption(option)
    out = []
    try:
        for value in (0, 1):
            dd.setOption(option, value)
            scene = build(gpu_device)
            t = fresnel.tracer.Path(gpu_device, w=w, h=h)
            t.seed = 17
            t.sample(scene, samples=8, reset=False)
            out.append((numpy.array(t.linear_output[:], copy=True), t._tracer.primaryHits()))
    finally:
        dd.setOption(option, old)
    (la, ha), (lb, hb) = out
    assert numpy.count_nonzero(ha[..., 0] != 0xFFFFFFFF) > 0
    same_hits = numpy.all(ha == hb, axis=-1).mean()
    assert same_hits >= 0.9999, f"{same_hits:.5%} of primary hits agree"
    close = numpy.all(numpy.abs(la - lb) <= 1e-5, axis=-1).mean()
    assert close >= 0.999, f"{close:.4%} of pixels agree"


def test_combined_tree_matches_per_geometry_trees(gpu_device):
    """A mixed scene traced through its combined tree finds the same closest hits as through
    one tree per geometry (Preview hit ids; exact-distance ties aside)."""
    from parity import preview_hits
    dd = gpu_device._device
    old = dd.getOption("combined")
    out = []
    try:
        for combined in (0, 1):
            dd.setOption("combined", combined)
            scene = workloads.config3(gpu_device, scale=0.01)
            out.append(preview_hits(gpu_device, scene, 160, 90, 2))
    finally:
        dd.setOption("combined", old)
    (ha, la, _), (hb, lb, _) = out
    assert numpy.count_nonzero(ha[..., 0]) > 0
    same = numpy.all(ha == hb, axis=-1).mean()
    assert same >= 0.9999, f"{same:.5%} of hit ids agree"
    agree = numpy.all(numpy.all(ha == hb, axis=-1), axis=-1)
    assert numpy.abs(la - lb)[agree].max() <= 1e-6
