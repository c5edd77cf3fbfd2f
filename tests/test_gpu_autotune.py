"""Autotuner on the GPU: it measures, picks and applies options, and the options it tunes do
not change the images beyond closest-hit ties (at least 99.9% of pixels equal within 1e-5)."""

import numpy
import pytest

import fresnel_b200 as fresnel
from fresnel_b200 import autotune, workloads

pytestmark = pytest.mark.gpu


def test_tuner_picks_and_applies(gpu_device):
    dd = gpu_device._device
    saved = {k: dd.getOption(k) for k in ("leaf_max", "tile", "path_slots")}
    try:
        jobs = [(workloads.random_spheres(gpu_device, 3000, 30.0, seed=21, colors=True), 96, 64, 1),
                (workloads.hex_spheres(gpu_device), 64, 64, 2)]
        space = (("leaf_max", (1, 4)), ("tile", (4, 16)), ("path_slots", (1 << 16, 1 << 20)))
        t = autotune.Tuner(gpu_device, space=space, probe_spp=1, repeats=1)
        ref = fresnel.tracer.Path(gpu_device, w=96, h=64)
        ref.seed = 3
        ref.sample(jobs[0][0], samples=4)
        before = numpy.array(ref.linear_output[:], copy=True)
        best, ms = t.tune(jobs)
        assert ms > 0 and len(t.log) >= 4
        assert {k: dd.getOption(k) for k in best} == {k: float(v) for k, v in best.items()}
        again = fresnel.tracer.Path(gpu_device, w=96, h=64)
        again.seed = 3
        again.sample(jobs[0][0], samples=4)
        after = numpy.array(again.linear_output[:], copy=True)
        close = numpy.all(numpy.abs(before - after) <= 1e-5, axis=-1).mean()
        assert close >= 0.999, f"{close:.4%} of pixels unchanged"
    finally:
        for k, v in saved.items():
            dd.setOption(k, v)
