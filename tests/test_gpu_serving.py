"""Continuous-batching server on the GPU: each request's image is the same alone and in the mix.

A trace of requests over three small serving scenes (spheres and bonds) with mixed resolutions
and sample counts is served by RenderServer with a small step size, so requests share batch
launches and are sliced over several steps, and then served again one at a time with plain
Path.sample calls. Every request's linear image must agree within 1e-6 and its sRGB image must
match exactly, and every request must get its ray count.
"""

import numpy
import pytest

from fresnel_b200 import serving, workloads
from parity import oracle_path_image, same_seed_fraction
from parity_record import record

pytestmark = pytest.mark.gpu


def test_served_equals_alone(gpu_device):
    sizes = {0: 1500, 1: 4000, 2: 800}
    scenes = {k: workloads.serving_scene(gpu_device, n, seed=50 + k) for k, n in sizes.items()}
    rng = numpy.random.default_rng(11)
    res = [(64, 48), (96, 64), (40, 40), (128, 72)]
    reqs = []
    for i in range(16):
        w, h = res[int(rng.integers(len(res)))]
        reqs.append(serving.Request(int(rng.integers(3)), w, h, int(rng.integers(1, 10)),
                                    seed=500 + i, arrival=0.0, tag=i))
    engine = serving.Engine(gpu_device)
    srv = serving.RenderServer(engine, lambda k: (scenes[k], workloads.serving_scene_bytes(sizes[k])),
                               step_paths=20000, max_active=6, keep_linear=True)
    serving.serve_trace(srv, reqs, realtime=False)
    assert srv.steps > 3
    served = {r.tag: (r.linear, r.image, r.rays) for r in reqs}

    alone = [serving.Request(r.scene_key, r.w, r.h, r.samples, seed=r.seed, tag=r.tag)
             for r in reqs]
    serving.plain_trace(engine, lambda k: scenes[k], alone, realtime=False, keep_linear=True)
    for r in alone:
        lin, img, rays = served[r.tag]
        assert numpy.isfinite(lin).all()
        diff = float(numpy.abs(lin - r.linear).max())
        assert diff <= 1e-6, f"request {r.tag}: max |linear difference| {diff}"
        assert numpy.array_equal(img, r.image)
        assert rays == r.rays > 0
    s = serving.latency_summary(reqs)
    assert s["requests"] == len(reqs)


def test_served_matches_oracle(gpu_device, oracle_device):
    """Requests served in a mix (sliced over several steps) against the CPU oracle rendering
    each request alone with the request's seed: >= 99% of pixels within 1e-3."""
    sizes = {0: 1200, 1: 3000}
    scenes = {k: workloads.serving_scene(gpu_device, n, seed=70 + k) for k, n in sizes.items()}
    oscenes = {k: workloads.serving_scene(oracle_device, n, seed=70 + k)
               for k, n in sizes.items()}
    reqs = [serving.Request(i % 2, w, h, spp, seed=900 + i, arrival=0.0, tag=i)
            for i, (w, h, spp) in enumerate([(64, 48, 5), (96, 64, 3), (40, 40, 8),
                                             (80, 60, 4), (72, 40, 6)])]
    engine = serving.Engine(gpu_device)
    srv = serving.RenderServer(engine, lambda k: (scenes[k], workloads.serving_scene_bytes(sizes[k])),
                               step_paths=8000, max_active=3, keep_linear=True)
    serving.serve_trace(srv, reqs, realtime=False)
    assert srv.steps >= 2
    for r in reqs:
        ora = oracle_path_image(oracle_device, oscenes[r.scene_key], r.w, r.h, r.seed, r.samples)
        frac = same_seed_fraction(r.linear, ora)
        record("test_served_matches_oracle", check="same_seed", request=r.tag,
               width=r.w, height=r.h, spp=r.samples, within_1e3=frac)
        assert frac >= 0.99, f"request {r.tag}: {frac:.4%} of pixels within 1e-3"
