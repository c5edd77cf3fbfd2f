"""Helpers that render the same scene with the engine and with the oracle (test infrastructure)."""

import numpy


def preview_hits(device, scene, w, h, aa_n):
    """(hit_ids[h, w, aa_n^2, 2], linear[h, w, 4], srgb[h, w, 4]) of a preview render."""
    t = device.module.TracerDirect(device._device, w, h)
    t.setAntialiasingN(aa_n)
    if hasattr(t, "renderHitIds"):  # engine
        hits = t.renderHitIds(scene._scene)
    else:  # oracle
        t.record_hits = True
        t.render(scene._scene)
        hits = t.last_hit_ids
    lin = t.getLinearOutputBuffer()
    srgb = t.getSRGBOutputBuffer()
    lin.map()
    srgb.map()
    out = hits, numpy.array(lin, copy=True), numpy.array(srgb, copy=True)
    lin.unmap()
    srgb.unmap()
    return out


def path_render(device, scene, w, h, samples, light_samples=1, seed=None):
    """Render with the Path tracer; returns (linear, srgb, tracer)."""
    from fresnel_b200 import tracer as tracer_mod
    t = tracer_mod.Path(device, w=w, h=h)
    if seed is not None:
        t.seed = seed
    t.sample(scene, samples=samples, light_samples=light_samples)
    return numpy.array(t.linear_output[:]), numpy.array(t.output[:]), t
