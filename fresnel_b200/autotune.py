"""Autotuner for the engine's tuning options (no counterpart in fresnel, whose OptiX and Embree
backends tune themselves).

The knobs are the device options that change speed but not images:

* ``leaf_max``   largest BVH leaf (primitives) the surface-area collapse may form;
* ``tile``       block shape of the primary pass: square pixel tiles of 4, 8 or 16;
* ``path_slots`` queue depth: path slots traced together in one wavefront.

``Tuner.tune(jobs)`` times short probe renders of the caller's own scenes and image sizes (one
``PathBatch`` of every job at ``probe_spp`` samples) and does coordinate descent: knob by knob
in the order above, every value of the knob with the others held at the best so far, keeping
the fastest.  That costs the sum, not the product, of the knob sizes.  Results are cached per
workload signature (job count, pixel and primitive totals rounded to powers of two, geometry
types), so a server or a trajectory loop pays once per kind of workload.
"""

import math

DEFAULT_SPACE = (
    ("leaf_max", (1, 2, 4, 8)),
    ("tile", (4, 8, 16)),
    ("path_slots", (8 << 20, 16 << 20, 32 << 20, 64 << 20)),
)


def _bucket(x):
    return 0 if x <= 0 else int(round(math.log2(x)))


def signature(jobs):
    """Workload key of (scene, w, h, light_samples) jobs."""
    pixels = sum(w * h for _, w, h, _ in jobs)
    prims, kinds = 0, set()
    for scene, _, _, _ in jobs:
        for g in scene.geometry:
            kinds.add(type(g).__name__)
            try:
                prims += len(g.position[:]) if hasattr(g, "position") else len(g.points[:])
            except (AttributeError, RuntimeError):
                pass
    return (len(jobs), _bucket(pixels), _bucket(prims), tuple(sorted(kinds)))


class Tuner:
    """Coordinate-descent tuner over ``space`` for one device.

    Args:
        device: a ``fresnel_b200.Device``.
        space: sequence of (option name, candidate values), tuned in this order.
        probe_spp: samples per pixel of each probe render.
        repeats: timed probe renders per setting (the fastest counts).
        timer: ``(device, jobs, probe_spp) -> ms`` override (tests).
    """

    def __init__(self, device, space=DEFAULT_SPACE, probe_spp=2, repeats=2, timer=None):
        self.device = device
        self.space = tuple(space)
        self.probe_spp = int(probe_spp)
        self.repeats = int(repeats)
        self.cache = {}
        self.log = []
        self._timer = timer
        self._tracers = {}

    # ---- options -------------------------------------------------------------------------
    def options(self):
        dd = self.device._device
        return {name: dd.getOption(name) for name, _ in self.space}

    def apply(self, options):
        dd = self.device._device
        for name, value in options.items():
            if dd.getOption(name) != value:
                dd.setOption(name, value)

    # ---- one measurement -------------------------------------------------------------------
    def _time(self, jobs):
        if self._timer is not None:
            return self._timer(self.device, jobs, self.probe_spp)
        from . import tracer as tracer_mod
        dd = self.device._device
        for scene, _, _, _ in jobs:
            scene._scene.build()  # rebuild what the options made stale, outside the timing
        batch = tracer_mod.PathBatch(self.device)
        tracers = []
        for n, (scene, w, h, ls) in enumerate(jobs):
            key = (n, w, h)
            if key not in self._tracers:
                self._tracers[key] = tracer_mod.Path(self.device, w=w, h=h)
            tracers.append((self._tracers[key], scene, ls))

        def once():
            for t, scene, ls in tracers:
                batch.add(t, scene, samples=self.probe_spp, light_samples=ls)
            batch.render()

        once()  # warm: kernels, graph capture, buffers
        best = float("inf")
        for _ in range(self.repeats):
            dd.synchronize()
            dd.timerStart()
            once()
            best = min(best, dd.timerStop())
        return best

    def measure(self, jobs, options, seen=None):
        """Probe ms of `options` (reused from `seen`, a dict of settings already measured for
        these jobs)."""
        key = tuple(sorted((k, float(v)) for k, v in options.items()))
        if seen is not None and key in seen:
            return seen[key]
        self.apply(options)
        ms = self._time(jobs)
        self.log.append((dict(options), ms))
        if seen is not None:
            seen[key] = ms
        return ms

    # ---- search ----------------------------------------------------------------------------
    def tune(self, jobs, apply=True):
        """Best options for `jobs` (list of (scene, w, h, light_samples)); applied to the
        device unless ``apply`` is False.  Returns (options, probe ms)."""
        key = signature(jobs)
        if key in self.cache:
            best, ms = self.cache[key]
            if apply:
                self.apply(best)
            return dict(best), ms
        start = self.options()
        best = dict(start)
        seen = {}
        best_ms = self.measure(jobs, best, seen)
        for name, values in self.space:
            for v in values:
                trial = dict(best)
                trial[name] = v
                ms = self.measure(jobs, trial, seen)
                if ms < best_ms:
                    best, best_ms = trial, ms
        self.cache[key] = (dict(best), best_ms)
        self.apply(best if apply else start)
        return dict(best), best_ms
