"""Kernel options that change where the arithmetic runs, not what it is, give identical images:
shading fused into the tracing passes (device option "fuse_shade"; several light samples per
pixel sample, whose later light samples restart from the stored primary ray), per-lane refill,
the tail kernel, and Preview with one warp per pixel; on the sphere grid, the BVH of one
geometry and the combined BVH or grid over parts of a mixed scene."""

import numpy
import pytest

import fresnel_b200 as fresnel
from fresnel_b200 import workloads

pytestmark = pytest.mark.gpu

SCENES = {
    "spheres_1k_32ls": (workloads.config1, 96, 96, 3, 8),
    "dense_grid": (lambda d: workloads.config2(d, n=20000, box=140.0 * 0.02**(1 / 3)), 120, 68,
                   6, 1),
    "mixed": (lambda d: workloads.config3(d, scale=0.002), 96, 54, 4, 2),
}


@pytest.mark.parametrize("name", list(SCENES))
def test_fused_passes_give_identical_images(name, gpu_device):
    build, w, h, spp, ls = SCENES[name]
    dd = gpu_device._device
    old = dd.getOption("fuse_shade")
    out = []
    try:
        for fuse in (0, 1, 2):
            dd.setOption("fuse_shade", fuse)
            scene = build(gpu_device)
            t = fresnel.tracer.Path(gpu_device, w=w, h=h)
            t.seed = 3
            t.sample(scene, samples=spp, light_samples=ls)
            out.append((numpy.array(t.linear_output[:], copy=True),
                        t._tracer.getStats()["rays"]))
    finally:
        dd.setOption("fuse_shade", old)
    (a, ra), (b, rb), (c, rc) = out
    assert numpy.isfinite(a).all() and numpy.count_nonzero(a[..., 3]) > 0
    assert numpy.array_equal(a, b) and numpy.array_equal(a, c)
    assert ra == rb == rc


def test_grid_refill_extension_gives_identical_images(gpu_device):
    """Device option "refill" on a sphere-grid scene: extension rays walk the grid with per-lane
    refill and are shaded by the separate shade pass; the same arithmetic as the fused bounces."""
    dd = gpu_device._device
    old = dd.getOption("refill")
    out = []
    try:
        for refill in (0, 1):
            dd.setOption("refill", refill)
            scene = workloads.config2(gpu_device, n=20000, box=140.0 * 0.02**(1 / 3))
            t = fresnel.tracer.Path(gpu_device, w=120, h=68)
            t.seed = 5
            t.sample(scene, samples=6, light_samples=2)
            out.append((numpy.array(t.linear_output[:], copy=True),
                        t._tracer.getStats()["rays"]))
    finally:
        dd.setOption("refill", old)
    (a, ra), (b, rb) = out
    assert numpy.isfinite(a).all() and numpy.count_nonzero(a[..., 3]) > 0
    assert numpy.array_equal(a, b)
    assert ra == rb


def test_tail_kernel_gives_identical_images(gpu_device):
    """Device option "tail": the fused bounces of a sphere-grid scene run as that many bounce
    launches and then one persistent launch that follows every remaining path to its end (-1:
    bounce launches only).  Each path's arithmetic is the same, so the images and ray counts must
    be identical."""
    dd = gpu_device._device
    old = dd.getOption("tail")
    out = []
    try:
        for tail in (-1, 0, 1, 3):
            dd.setOption("tail", tail)
            scene = workloads.config2(gpu_device, n=20000, box=140.0 * 0.02**(1 / 3))
            t = fresnel.tracer.Path(gpu_device, w=120, h=68)
            t.seed = 6
            t.sample(scene, samples=7, light_samples=2)
            out.append((numpy.array(t.linear_output[:], copy=True),
                        t._tracer.getStats()["rays"]))
    finally:
        dd.setOption("tail", old)
    base, rays = out[0]
    assert numpy.isfinite(base).all() and numpy.count_nonzero(base[..., 3]) > 0
    for img, r in out[1:]:
        assert numpy.array_equal(base, img)
        assert r == rays


@pytest.mark.parametrize("name,accel", [("dense_grid", 2), ("dense_grid", 0), ("mixed", 2),
                                        ("mixed", 0), ("spheres_1k_32ls", 0)])
def test_preview_warp_per_pixel_gives_identical_output(name, accel, gpu_device):
    """Preview with a group of lanes per pixel (device option "preview_warp": 32 lanes at 8x8
    anti-aliasing, 16 at 4x4) sums each pixel's samples in the same order as one thread per
    pixel: identical hit ids, linear and sRGB outputs, through the sphere grid, the grid over
    parts and the trees; 2x2 and 3x3 anti-aliasing keep one thread per pixel."""
    from parity import preview_hits
    build, w, h, _, _ = SCENES[name]
    dd = gpu_device._device
    old = (dd.getOption("preview_warp"), dd.getOption("accel"))
    try:
        dd.setOption("accel", accel)
        scene = build(gpu_device)
        for aa in (8, 4, 2, 3):
            out = []
            for pw in (0, 1):
                dd.setOption("preview_warp", pw)
                out.append(preview_hits(gpu_device, scene, w, h, aa))
            for a, b in zip(out[0], out[1]):
                assert numpy.array_equal(a, b)
    finally:
        dd.setOption("preview_warp", old[0])
        dd.setOption("accel", old[1])
