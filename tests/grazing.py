"""Classify closest-hit disagreements between the engine and the oracle (test infrastructure).

A disagreement is *grazing* when the two primitives are hit at nearly the same distance (an
exact tie or a difference within float rounding of t), or when the ray passes within float
rounding of a silhouette (outline distance |d| tiny relative to the scene scale).  Anything
else is a real disagreement.
"""

import numpy

from oracle import cpu_module


def classify(oracle_device, oracle_scene, tracer_w, tracer_h, aa_n, gpu_hits, ora_hits, seed=0,
             rel_tol=1e-5, kinds=None):
    """Returns (n_grazing, real) where real lists (pixel, sample, gpu_hit, oracle_hit, detail).
    ``kinds`` (a dict), when given, counts the grazing disagreements by kind: "exact_tie" (both
    primitives hit at the same t), "near_tie" (t within rel_tol), "silhouette" (a ray within
    rounding of an outline edge, hit on one side and missed on the other, or hitting two
    primitives at different t)."""
    lib = oracle_device._device.lib
    handle = oracle_scene._scene.handle()
    cam = cpu_module.camera_struct(oracle_scene._scene.getCamera())
    cam.f_stop = float("inf")
    bad = numpy.argwhere(numpy.any(gpu_hits != ora_hits, axis=-1))
    n_grazing = 0
    real = []
    f = cpu_module.ptr
    for j, i, smp in bad:
        o = numpy.zeros(3, numpy.float32)
        d = numpy.zeros(3, numpy.float32)
        lib.or_camera_ray(cam, tracer_w, tracer_h, seed, 1 if aa_n != 1 else 0, int(i), int(j),
                          int(smp), f(o), f(d))
        ts = {}
        for name, hit in (("gpu", gpu_hits[j, i, smp]), ("oracle", ora_hits[j, i, smp])):
            if hit[0] == 0:
                ts[name] = None
                continue
            out = numpy.zeros(3, numpy.float32)
            ok = lib.or_prim_hit(handle, int(hit[0]) - 1, int(hit[1]), f(o), f(d), 0.0, f(out))
            ts[name] = (float(out[0]), float(out[1])) if ok else "no-hit"
        g, r = ts["gpu"], ts["oracle"]
        scale = float(numpy.abs(o).max() + 1.0)
        grazing = False
        if isinstance(g, tuple) and isinstance(r, tuple):
            grazing = abs(g[0] - r[0]) <= rel_tol * max(abs(r[0]), 1e-6) or \
                min(abs(g[1]), abs(r[1])) <= 1e-5 * scale
        elif isinstance(r, tuple) and g is None:
            grazing = abs(r[1]) <= 1e-5 * scale
        elif isinstance(g, tuple) and r is None:
            grazing = abs(g[1]) <= 1e-5 * scale
        if grazing:
            n_grazing += 1
            if kinds is not None:
                if isinstance(g, tuple) and isinstance(r, tuple) and g[0] == r[0]:
                    kind = "exact_tie"
                elif isinstance(g, tuple) and isinstance(r, tuple) and \
                        abs(g[0] - r[0]) <= rel_tol * max(abs(r[0]), 1e-6):
                    kind = "near_tie"
                else:
                    kind = "silhouette"
                kinds[kind] = kinds.get(kind, 0) + 1
        else:
            real.append((int(j) * tracer_w + int(i), int(smp), tuple(gpu_hits[j, i, smp]),
                         tuple(ora_hits[j, i, smp]), (g, r)))
    return n_grazing, real


# Closest-hit id disagreements between the engine and the oracle, grazing ones included, per
# sample: the bar every hit-id parity test applies (non-grazing ones must be absent).
MISMATCH_MAX = 1e-4


def check_hits(test, oracle_device, oracle_scene, w, h, aa_n, gpu_hits, ora_hits, **extra):
    """Classify, record (parity_record) and check the hit-id disagreements of one render;
    returns the per-sample mismatch mask."""
    from parity_record import record
    mism = numpy.any(gpu_hits != ora_hits, axis=-1)
    kinds = {}
    n_grazing, real = classify(oracle_device, oracle_scene, w, h, aa_n, gpu_hits, ora_hits,
                               kinds=kinds)
    n = int(numpy.count_nonzero(mism))
    rate = n / mism.size
    record(test, check="preview_hits", width=w, height=h, aa=aa_n, samples=int(mism.size),
           mismatches=n, grazing=n_grazing, grazing_kinds=kinds, non_grazing=len(real),
           rate=rate, **extra)
    assert not real, f"non-grazing hit disagreements: {real[:5]}"
    assert rate <= MISMATCH_MAX, f"{n} of {mism.size} closest hits differ ({rate:.2e})"
    return mism
