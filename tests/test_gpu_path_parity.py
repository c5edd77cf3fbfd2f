"""Path tracer on the GPU versus the CPU oracle.

1. Same seed: the GPU follows the same random process (Philox keyed by pixel and seed,
   countered by sample, depth and light sample), so per-pixel means agree to float rounding
   except where a transcendental rounding difference flips a branch.  Bar: >= 99% of pixels
   within 1e-3 (linear RGB), the rest bounded by the Monte Carlo spread.
2. Monte Carlo error: a 256-spp GPU image against a 4096-spp oracle on a seeded sparse pixel
   set: z = (gpu - oracle) / sqrt(s2/256 + s2/4096) per pixel and channel, s2 the oracle's
   per-pixel sample variance.  Bar: mean z^2 <= 1.2 and at most 6% of |z| > 2 ("within 2x the
   Monte Carlo standard error").
"""

import numpy
import pytest

from fresnel_b200 import workloads
from parity import path_render
from parity_record import record

pytestmark = pytest.mark.gpu

SAME_SEED = {
    "hex_spheres": (workloads.hex_spheres, 64, 64, 8, 2),
    "spheres_1k": (workloads.config1, 96, 96, 4, 4),
    "dense_spheres": (lambda d: workloads.config2(d, n=20000,
                                                  box=140.0 * (0.02)**(1 / 3)), 96, 54, 6, 1),
    "mixed": (lambda d: workloads.config3(d, scale=0.002), 96, 54, 4, 1),
    "polygons_spheres": (lambda d: workloads.polygons(d, spheres=60), 96, 72, 6, 2),
}


@pytest.mark.parametrize("name", list(SAME_SEED))
def test_path_same_seed(name, gpu_device, oracle_device):
    build, w, h, spp, ls = SAME_SEED[name]
    gl, g8, gt = path_render(gpu_device, build(gpu_device), w, h, spp, ls, seed=7)
    ol, o8, ot = path_render(oracle_device, build(oracle_device), w, h, spp, ls, seed=7)
    assert gt.seed == ot.seed == 8
    assert gt._tracer.getNumSamples() == spp
    close = numpy.all(numpy.abs(gl - ol) <= 1e-3, axis=-1)
    frac = close.mean()
    record("test_path_same_seed", check="same_seed", scene=name, width=w, height=h, spp=spp,
           light_samples=ls, within_1e3=float(frac), max_abs=float(numpy.abs(gl - ol).max()))
    assert frac >= 0.99, f"only {frac:.4%} of pixels within 1e-3"
    assert numpy.all(g8[..., 3] == o8[..., 3])


def test_path_monte_carlo_error(gpu_device, oracle_device):
    w, h = 96, 96
    gpu_spp, ref_spp = 256, 4096
    gl, _, _ = path_render(gpu_device, workloads.config1(gpu_device), w, h, gpu_spp, 1, seed=3)
    scene = workloads.config1(oracle_device)
    rng = numpy.random.default_rng(1234)
    pixels = numpy.sort(rng.choice(w * h, size=512, replace=False)).astype(numpy.uint32)
    t = oracle_device.module.TracerPath(oracle_device._device, w, h, 1)
    t.setSeed(99)
    lin, _, m2 = t.render_pixels(scene._scene, pixels, 1, ref_spp)
    var = m2 / (ref_spp - 1)
    g = gl.reshape(-1, 4)[pixels, :3]
    se2 = var / gpu_spp + var / ref_spp
    mask = se2 > 1e-12
    z = (g - lin[:, :3])[mask] / numpy.sqrt(se2[mask])
    record("test_path_monte_carlo_error", check="monte_carlo", scene="spheres_1k", spp=gpu_spp,
           oracle_spp=ref_spp, values=int(z.size), mean_z2=float(numpy.mean(z**2)),
           frac_abs_z_gt_2=float(numpy.mean(numpy.abs(z) > 2)))
    assert z.size > 100
    assert numpy.mean(z**2) <= 1.2, f"mean z^2 = {numpy.mean(z**2):.3f}"
    assert numpy.mean(numpy.abs(z) > 2) <= 0.06
