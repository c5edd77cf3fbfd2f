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


def odd_radii_scene(device, n=3000, seed=5):
    """Spheres among which some radii are negative, infinite, NaN or zero, and cylinders with
    some infinite or NaN radii: the reference's bounds of those are inverted or not finite, so
    they are never hit.  (A negative cylinder radius is left out: the reference's bounds of such
    a cylinder can be valid yet smaller than the capsule its intersector hits, so which rays
    reach it depends on each tree's boxes.)"""
    import fresnel_b200 as fresnel
    rng = numpy.random.default_rng(seed)
    pos = rng.uniform(-12, 12, (n, 3)).astype(numpy.float32)
    r = rng.uniform(0.2, 0.9, n).astype(numpy.float32)
    r[::97] = -0.5
    r[1::101] = numpy.inf
    r[2::103] = numpy.nan
    r[3::107] = 0.0
    scene = fresnel.Scene(device)
    fresnel.geometry.Sphere(scene, position=pos, radius=r,
                            material=fresnel.material.Material(color=(0.3, 0.6, 0.9)))
    m = 400
    a = rng.uniform(-12, 12, (m, 3)).astype(numpy.float32)
    pts = numpy.stack([a, a + rng.normal(0, 1.5, (m, 3)).astype(numpy.float32)], axis=1)
    rc = numpy.full(m, 0.15, numpy.float32)
    rc[::7] = numpy.inf
    rc[1::11] = numpy.nan
    fresnel.geometry.Cylinder(scene, points=pts, radius=rc,
                              material=fresnel.material.Material(color=(0.9, 0.5, 0.2)))
    scene.camera = fresnel.camera.Orthographic(position=(0, 0, 40), look_at=(0, 0, 0),
                                               up=(0, 1, 0), height=26)
    return scene


def oracle_path_image(oracle_device, scene, w, h, seed, samples, light_samples=1):
    """The oracle's Path image of ``samples`` samples (numbers 1..samples) rendered with
    exactly ``seed`` (the seed a GPU tracer renders with after its own reset/seed schedule)."""
    t = oracle_device.module.TracerPath(oracle_device._device, w, h, light_samples)
    t.setSeed(seed)
    t.renderSamples(scene._scene, samples)
    return numpy.array(t.getLinearOutputBuffer(), copy=True)


def same_seed_fraction(gpu_linear, oracle_linear, tol=1e-3):
    """Fraction of pixels whose linear RGBA agree within ``tol`` in every channel."""
    return float(numpy.all(numpy.abs(gpu_linear - oracle_linear) <= tol, axis=-1).mean())
