"""Continuous-batching render server (no counterpart in fresnel, which renders one call at a time).

Requests (a scene, an image size, a sample count) arrive at any time.  The server keeps every
admitted request's accumulation buffer and its scene's BVH resident on the GPU and advances
them together in steps: each step queues slices of samples of the active requests (shortest
remaining work first, up to a path budget) into one ``tracer.PathBatch`` and traces it in one
CUDA graph launch.  Requests that arrive while a
step is on the GPU join at the next step boundary, as soon as the HBM budget has room for their
buffers (and their scene, if it is not resident yet); finished requests leave at the end of the
step that completes them, and their image is read back.  Samples of a request fold into its
image in sample order, so its image is the same whatever it was batched with and however its
samples were sliced into steps.

The scheduler is plain Python over the engine's batch API; ``engine`` objects are duck-typed so
the policy can be exercised without a GPU.
"""

import collections
import math
import time

import numpy


class Request:
    """One render request: ``samples`` samples of ``scene_key`` at ``w`` x ``h``.

    ``arrival`` is a time in seconds relative to the start of a trace (``serve_trace``);
    the server fills in ``t_arrive``, ``t_admit``, ``t_done`` (absolute clock values), ``image``
    (sRGB, h x w x 4 uint8) and ``rays``.
    """

    __slots__ = ("scene_key", "w", "h", "samples", "light_samples", "seed", "arrival", "t_arrive",
                 "t_admit", "t_done", "image", "linear", "done_samples", "tracer", "rays", "tag")

    def __init__(self, scene_key, w, h, samples, light_samples=1, seed=0, arrival=0.0, tag=None):
        self.scene_key = scene_key
        self.w, self.h = int(w), int(h)
        self.samples = int(samples)
        self.light_samples = int(light_samples)
        self.seed = int(seed)
        self.arrival = float(arrival)
        self.t_arrive = self.t_admit = self.t_done = None
        self.image = self.linear = None
        self.done_samples = 0
        self.tracer = None
        self.rays = 0
        self.tag = tag

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.t_arrive

    @property
    def output_bytes(self):
        return self.w * self.h * 20  # linear RGBA f32 + sRGB RGBA8


class Engine:
    """The GPU engine as the server sees it (tracers, batches, resident scenes)."""

    def __init__(self, device):
        from . import tracer as tracer_mod
        self.device = device
        self._tracer_mod = tracer_mod

    def new_tracer(self, w, h):
        return self._tracer_mod.Path(self.device, w=w, h=h)

    def new_batch(self):
        return self._tracer_mod.PathBatch(self.device)

    def reserve(self, batch, paths):
        """Size the batch's path state for a full step up front (at most the device's wavefront
        size), so that no step pays for growing it."""
        slots = int(self.device._device.getOption("path_slots"))
        batch.reserve(min(int(paths), slots))

    @staticmethod
    def start(tracer, seed):
        """Clear the tracer's image and set the seed of the request it now serves."""
        tracer.reset()
        tracer.seed = seed

    @staticmethod
    def rays(tracer):
        return int(tracer._tracer.getStats()["rays"])

    @staticmethod
    def read(tracer, keep_linear):
        img = numpy.array(tracer.output[:], copy=True)
        lin = numpy.array(tracer.linear_output[:], copy=True) if keep_linear else None
        return img, lin


class RenderServer:
    """Iteration-level scheduler over the batched path tracer.

    Args:
        engine: an ``Engine`` (or an object with the same methods).
        scene_factory: ``key -> (scene, nbytes)``; called once per key while it is resident.
        hbm_budget: bytes for resident scenes plus the accumulation buffers of active requests.
        step_paths: path budget (pixels x samples) of one step, filled shortest remaining
            work first (``plan_step``).  While all outstanding work fits in
            ``max_step_paths`` (8 x step_paths by default), a step takes all of it: at light
            load nothing is sliced, and a large request finishes in one launch.
        max_active: at most this many admitted requests (their buffers count against the
            budget; a request takes a tracer from the pool when it is first traced).
        keep_linear: also read back each finished request's linear (float) image.
        aging_s: waiting time that halves a request's scheduling key (0.25 s: against 1 s it
            took the serving trace's p99 at 250 requests/s from 577 to 404 ms and changed the
            other rates' p50 and p99 by at most their noise; 0.1 s was no better).
    """

    def __init__(self, engine, scene_factory, hbm_budget=120e9, step_paths=32 << 20,
                 max_active=256, keep_linear=False, clock=time.perf_counter, aging_s=0.25,
                 max_step_paths=None):
        self.engine = engine
        self.aging_s = float(aging_s)
        self.max_step_paths = int(8 * step_paths if max_step_paths is None else max_step_paths)
        self.scene_factory = scene_factory
        self.hbm_budget = float(hbm_budget)
        self.step_paths = int(step_paths)
        self.max_active = int(max_active)
        self.keep_linear = keep_linear
        self.clock = clock
        self.queue = collections.deque()
        self.active = []
        self.finished = []
        self.scenes = collections.OrderedDict()  # key -> [scene, nbytes, active users], LRU order
        self.pool = collections.defaultdict(list)  # (w, h) -> idle tracers
        self.bytes_in_use = 0.0
        self.steps = 0
        self.batch = engine.new_batch()
        reserve = getattr(engine, "reserve", None)
        if reserve is not None:
            reserve(self.batch, self.max_step_paths)
        # host seconds spent per phase of step() (admit, queue slices, trace, retire)
        self.phase_s = {"admit": 0.0, "queue": 0.0, "trace": 0.0, "retire": 0.0}

    # ---- admission -----------------------------------------------------------------------
    def submit(self, req, now=None):
        req.t_arrive = self.clock() if now is None else now
        self.queue.append(req)

    def _evict_for(self, need):
        """Drop idle resident scenes (least recently used first) until `need` bytes fit."""
        for key in list(self.scenes):
            if self.bytes_in_use + need <= self.hbm_budget:
                return True
            entry = self.scenes[key]
            if entry[2] == 0:
                self.bytes_in_use -= entry[1]
                del self.scenes[key]
        return self.bytes_in_use + need <= self.hbm_budget

    def _admit(self):
        while self.queue and len(self.active) < self.max_active:
            req = self.queue[0]
            resident = req.scene_key in self.scenes
            need = req.output_bytes
            if resident:
                if self.bytes_in_use + need > self.hbm_budget and not self._evict_for(need):
                    return
            else:
                # the factory's byte estimate is only known after building; build first, then
                # check (a scene larger than the whole budget is rejected)
                scene, nbytes = self.scene_factory(req.scene_key)
                if nbytes + need > self.hbm_budget:
                    self.queue.popleft()
                    raise RuntimeError(f"request for scene {req.scene_key!r} needs "
                                       f"{nbytes + need:.3g} bytes, more than the HBM budget")
                if not self._evict_for(nbytes + need):
                    return
                self.scenes[req.scene_key] = [scene, nbytes, 0]
                self.bytes_in_use += nbytes
            self.queue.popleft()
            entry = self.scenes[req.scene_key]
            self.scenes.move_to_end(req.scene_key)
            entry[2] += 1
            self.bytes_in_use += need
            req.t_admit = self.clock()
            self.active.append(req)

    def reserve_tracers(self, counts):
        """Create idle tracers ahead of time: ``counts`` maps (w, h) to how many."""
        for (w, h), n in counts.items():
            while len(self.pool[(w, h)]) < n:
                self.pool[(w, h)].append(self.engine.new_tracer(w, h))

    def _start(self, req):
        """Give a request its tracer (from the pool) when it is first traced."""
        idle = self.pool[(req.w, req.h)]
        req.tracer = idle.pop() if idle else self.engine.new_tracer(req.w, req.h)
        self.engine.start(req.tracer, req.seed)
        req.rays = -self.engine.rays(req.tracer)

    # ---- one step --------------------------------------------------------------------------
    def plan_step(self, now=None):
        """(request, samples) slices of the next step.

        Active requests are taken in order of remaining work (pixels x samples still to do),
        divided by 1 + waiting time / aging_s so that large requests keep moving; each takes
        what it still needs up to the step's path budget (at least one sample, and the first
        request always gets in).  Small requests therefore finish in the step after their
        arrival, and large ones fill the rest of every step.
        """
        now = self.clock() if now is None else now

        def key(r):
            rem = r.w * r.h * (r.samples - r.done_samples)
            return (rem / (1.0 + max(0.0, now - r.t_arrive) / self.aging_s), r.t_arrive)

        remaining = sum(r.w * r.h * (r.samples - r.done_samples) for r in self.active)
        budget = self.step_paths
        if remaining <= self.max_step_paths:
            budget = max(budget, remaining)
        plan = []
        for r in sorted(self.active, key=key):
            px = r.w * r.h
            if plan and px > budget:
                continue
            k = min(r.samples - r.done_samples, max(1, budget // px))
            plan.append((r, k))
            budget -= k * px
            if budget <= 0:
                break
        return plan

    def step(self):
        """Admit what fits, trace one step's slices, retire finished requests.
        Returns the requests finished in this step."""
        c = self.clock
        t0 = c()
        self._admit()
        t1 = c()
        self.phase_s["admit"] += t1 - t0
        if not self.active:
            return []
        plan = self.plan_step(t1)
        for r, k in plan:
            if r.tracer is None:
                self._start(r)
            self.batch.add(r.tracer, self.scenes[r.scene_key][0], samples=k, reset=False,
                           light_samples=r.light_samples)
        t2 = c()
        self.batch.render()
        t3 = c()
        self.phase_s["queue"] += t2 - t1
        self.phase_s["trace"] += t3 - t2
        self.steps += 1
        done = []
        for r, k in plan:
            r.done_samples += k
            if r.done_samples >= r.samples:
                done.append(r)
        finished = set(id(r) for r in done)
        self.active = [r for r in self.active if id(r) not in finished]
        for r in done:
            r.image, r.linear = self.engine.read(r.tracer, self.keep_linear)
            r.rays += self.engine.rays(r.tracer)
            r.t_done = self.clock()
            self.pool[(r.w, r.h)].append(r.tracer)
            r.tracer = None
            self.bytes_in_use -= r.output_bytes
            self.scenes[r.scene_key][2] -= 1
        self.finished.extend(done)
        self.phase_s["retire"] += c() - t3
        return done

    def idle(self):
        return not self.queue and not self.active

    def drain(self):
        while not self.idle():
            self.step()


def serve_trace(server, requests, realtime=True):
    """Feed `requests` (sorted by ``arrival``, seconds from now) to `server` and run it until
    all are finished.  With ``realtime`` the arrivals follow the wall clock (a request becomes
    visible once its arrival time has passed); otherwise all arrive at once."""
    clock = server.clock
    t0 = clock()
    pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
    while pending or not server.idle():
        now = clock() - t0
        while pending and (not realtime or pending[0].arrival <= now):
            r = pending.popleft()
            server.submit(r, now=t0 + r.arrival if realtime else t0)
        if server.idle():
            wait = pending[0].arrival - (clock() - t0)
            if wait > 0:
                time.sleep(min(wait, 0.005))
            continue
        server.step()
    return t0


def plain_trace(engine, scene_of, requests, realtime=True, clock=time.perf_counter,
                keep_linear=False, per_sample=False):
    """Baseline: the same requests served one at a time in arrival order, each by one plain
    ``Path.sample`` call on its own (pooled) tracer, image read back after the call.  With
    ``per_sample`` each request is rendered the way fresnel's own ``Path.sample`` does it
    (fresnel/tracer.py:250-260): one ``render`` call per sample, each returning the output."""
    t0 = clock()
    pool = collections.defaultdict(list)
    for r in sorted(requests, key=lambda q: q.arrival):
        r.t_arrive = t0 + r.arrival if realtime else t0
        while realtime:
            wait = r.t_arrive - clock()  # read the clock once: it may pass t_arrive meanwhile
            if wait <= 0.0:
                break
            time.sleep(min(wait, 0.005))
        idle = pool[(r.w, r.h)]
        t = idle.pop() if idle else engine.new_tracer(r.w, r.h)
        r.t_admit = clock()
        engine.start(t, r.seed)
        before = engine.rays(t)
        if per_sample:
            scene = scene_of(r.scene_key)
            t._tracer.setLightSamples(r.light_samples)
            for _ in range(r.samples):
                t.render(scene)
            t._tracer.setLightSamples(1)
        else:
            t.sample(scene_of(r.scene_key), samples=r.samples, reset=False,
                     light_samples=r.light_samples)
        r.image, r.linear = engine.read(t, keep_linear)
        r.rays = engine.rays(t) - before
        r.done_samples = r.samples
        r.t_done = clock()
        idle.append(t)
    return t0


def latency_summary(requests):
    """p50 / p99 / mean time-to-image (ms) and throughput of finished requests."""
    lat = numpy.array([r.latency for r in requests if r.latency is not None]) * 1e3
    if len(lat) == 0:
        return {"requests": 0}
    t_first = min(r.t_arrive for r in requests)
    t_last = max(r.t_done for r in requests)
    span = max(t_last - t_first, 1e-9)
    rays = sum(max(r.rays, 0) for r in requests)
    paths = sum(r.w * r.h * r.samples * r.light_samples for r in requests)
    return {"requests": int(len(lat)), "p50_ms": float(numpy.percentile(lat, 50)),
            "p99_ms": float(numpy.percentile(lat, 99)), "mean_ms": float(lat.mean()),
            "max_ms": float(lat.max()), "requests_per_s": len(lat) / span,
            "mrays_per_s": rays / span / 1e6, "mpaths_per_s": paths / span / 1e6,
            "span_s": span}


def poisson_arrivals(rate, n, rng):
    """n arrival times (seconds) of a Poisson process of the given rate."""
    gaps = rng.exponential(1.0 / rate, n)
    return numpy.cumsum(gaps) - gaps[0]


def log_uniform_int(rng, lo, hi):
    return int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
