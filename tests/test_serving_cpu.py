"""Scheduling policy of the continuous-batching server, against a fake engine (no GPU).

The fake engine records what the server queues into each batch, so the tests can check the
invariants the GPU results rely on: every request gets exactly its sample count, in consecutive
slices that start at sample 1 and never overlap, each slice in its own batch launch; requests
are admitted in arrival order within the active limit and the HBM budget; idle scenes are
evicted least-recently-used first when the budget needs room; a scene larger than the budget is
rejected; finished requests free their buffers.
"""

import collections

import numpy
import pytest

from fresnel_b200 import serving


class FakeTracer:
    def __init__(self, w, h):
        self.w, self.h = w, h
        self.seed = 0
        self.samples = []  # (first, count) slices since the last reset
        self.rays = 0

    def reset(self):
        self.samples = []
        self.seed += 1

    def image(self):
        n = sum(c for _, c in self.samples)
        return numpy.full((self.h, self.w, 4), (self.seed + n) % 256, numpy.uint8)

    def sample(self, scene, samples, reset=True, light_samples=1):
        first = 1 + sum(c for _, c in self.samples)
        self.samples.append((first, samples))
        self.rays += self.w * self.h * samples


class FakeBatch:
    def __init__(self, log):
        self.log = log
        self.items = []

    def add(self, tracer, scene, samples, reset=True, light_samples=1):
        assert not reset
        assert all(t is not tracer for t, _, _ in self.items), "one slice per tracer per batch"
        self.items.append((tracer, scene, samples))

    def render(self):
        self.log.append([(id(t), s, k) for t, s, k in self.items])
        for t, s, k in self.items:
            t.sample(s, k)
        self.items = []


class FakeEngine:
    def __init__(self):
        self.batches = []
        self.tracers = 0

    def new_tracer(self, w, h):
        self.tracers += 1
        return FakeTracer(w, h)

    def new_batch(self):
        return FakeBatch(self.batches)

    @staticmethod
    def start(tracer, seed):
        tracer.reset()
        tracer.seed = seed

    @staticmethod
    def rays(tracer):
        return tracer.rays

    @staticmethod
    def read(tracer, keep_linear):
        return tracer.image(), None


def factory(sizes, built=None):
    def make(key):
        if built is not None:
            built.append(key)
        return (f"scene{key}", sizes[key])
    return make


def requests(n, rng, keys=4):
    out = []
    for i in range(n):
        w, h = [(8, 8), (16, 8), (32, 16)][int(rng.integers(3))]
        out.append(serving.Request(int(rng.integers(keys)), w, h, int(rng.integers(1, 20)),
                                   seed=100 + i, arrival=0.001 * i, tag=i))
    return out


def test_every_request_gets_its_samples_in_order():
    rng = numpy.random.default_rng(0)
    eng = FakeEngine()
    srv = serving.RenderServer(eng, factory({k: 1000 for k in range(4)}), step_paths=600,
                               max_active=5)
    reqs = requests(30, rng)
    serving.serve_trace(srv, reqs, realtime=False)
    assert len(srv.finished) == 30
    for r in reqs:
        assert r.done_samples == r.samples
        assert r.t_done is not None and r.latency >= 0
        assert r.image is not None and r.image.shape == (r.h, r.w, 4)
    # every batch held at most max_active slices
    assert max(len(b) for b in eng.batches) <= 5
    assert len(eng.batches) == srv.steps
    # tracers are pooled by size: far fewer than requests
    assert eng.tracers <= 5 * 3


def test_slices_are_consecutive_and_complete():
    rng = numpy.random.default_rng(1)
    eng = FakeEngine()
    srv = serving.RenderServer(eng, factory({k: 10 for k in range(4)}), step_paths=300,
                               max_active=3)
    reqs = requests(12, rng)
    seen = {}
    start = eng.start

    def record(tracer, seed):
        start(tracer, seed)
        seen[seed] = tracer
    eng.start = record
    for r in reqs:
        srv.submit(r)
    while not srv.idle():
        done = srv.step()
        for r in done:
            t = seen[r.seed]
            firsts = [f for f, _ in t.samples]
            counts = [c for _, c in t.samples]
            assert firsts[0] == 1
            assert all(firsts[i + 1] == firsts[i] + counts[i] for i in range(len(firsts) - 1))
            assert sum(counts) == r.samples
            assert t.seed == r.seed


def test_admission_respects_the_budget_and_order():
    eng = FakeEngine()
    # each 16x16 request needs 16*16*20 = 5120 bytes of buffers, each scene 1000 bytes
    budget = 1000 + 2 * 5120
    srv = serving.RenderServer(eng, factory({0: 1000}), hbm_budget=budget, step_paths=10)
    reqs = [serving.Request(0, 16, 16, 5, seed=i, tag=i) for i in range(6)]
    for r in reqs:
        srv.submit(r)
    srv.step()
    assert [r.tag for r in srv.active] == [0, 1]  # only two fit
    assert srv.bytes_in_use <= budget
    srv.drain()
    admits = [r.t_admit for r in reqs]
    assert admits == sorted(admits)  # first come, first admitted
    assert srv.bytes_in_use == 1000  # only the resident scene remains


def test_idle_scenes_are_evicted_lru():
    eng = FakeEngine()
    built = []
    srv = serving.RenderServer(eng, factory({0: 4000, 1: 4000, 2: 4000}, built),
                               hbm_budget=9000, step_paths=1 << 20)
    for key in (0, 1, 0, 2, 1):
        srv.submit(serving.Request(key, 4, 4, 1))
        srv.drain()
    # 0 and 1 fit together; 2 evicts the least recently used idle scene (1, since 0 was used
    # after it), so the last request for 1 rebuilds it and evicts 0
    assert built == [0, 1, 2, 1]
    assert list(srv.scenes) == [2, 1]


def test_scene_larger_than_budget_is_rejected():
    srv = serving.RenderServer(FakeEngine(), factory({0: 10**6}), hbm_budget=1000)
    srv.submit(serving.Request(0, 4, 4, 1))
    with pytest.raises(RuntimeError, match="more than the HBM budget"):
        srv.step()


def test_latency_summary():
    rng = numpy.random.default_rng(3)
    srv = serving.RenderServer(FakeEngine(), factory({k: 10 for k in range(4)}), step_paths=500)
    reqs = requests(20, rng)
    serving.serve_trace(srv, reqs, realtime=False)
    s = serving.latency_summary(reqs)
    assert s["requests"] == 20
    assert s["p50_ms"] <= s["p99_ms"] <= s["max_ms"]
    assert s["requests_per_s"] > 0


def test_plain_trace_matches_request_counts():
    rng = numpy.random.default_rng(4)
    eng = FakeEngine()
    reqs = requests(10, rng)
    serving.plain_trace(eng, lambda k: f"scene{k}", reqs, realtime=False)
    for r in reqs:
        assert r.done_samples == r.samples and r.image is not None and r.rays > 0


def test_plain_trace_waits_with_a_clock_that_passes_the_arrival():
    """Real-time plain_trace reads the clock once per wait: a clock that crosses a request's
    arrival between two reads must end the wait, not ask for a negative sleep."""
    eng = FakeEngine()
    reqs = [serving.Request(0, 8, 8, 2, seed=1, arrival=0.01, tag=0)]
    ticks = iter([0.0, 0.0099, 0.02] + [0.02 + 1e-3 * i for i in range(100)])
    serving.plain_trace(eng, lambda k: "scene", reqs, realtime=True, clock=lambda: next(ticks))
    assert reqs[0].done_samples == 2 and reqs[0].t_admit >= reqs[0].t_arrive


def test_poisson_arrivals_rate():
    rng = numpy.random.default_rng(5)
    t = serving.poisson_arrivals(200.0, 4000, rng)
    assert t[0] == 0.0 and numpy.all(numpy.diff(t) >= 0)
    assert abs(len(t) / t[-1] - 200.0) < 20.0


def test_serving_trace_generator():
    from fresnel_b200 import workloads
    reqs, sizes = workloads.config5(50.0, 200)
    assert len(reqs) == 200 and len(sizes) == 32
    assert all(1000 <= v <= 2_000_000 for v in sizes.values())
    keys = collections.Counter(r.scene_key for r in reqs)
    assert set(keys) <= set(sizes)
    assert all((r.w, r.h) in workloads.SERVING_RESOLUTIONS for r in reqs)
    assert all(1 <= r.samples <= 64 for r in reqs)
    again, _ = workloads.config5(50.0, 200)
    assert [(r.scene_key, r.w, r.samples, r.arrival) for r in reqs] == \
        [(r.scene_key, r.w, r.samples, r.arrival) for r in again]


def test_plan_prefers_short_work_and_ages():
    t = [0.0]
    srv = serving.RenderServer(FakeEngine(), factory({0: 10}), step_paths=1000,
                               clock=lambda: t[0], aging_s=1.0, max_step_paths=1000)
    big = serving.Request(0, 10, 10, 50, tag="big")      # 5000 paths left
    small = serving.Request(0, 10, 10, 2, tag="small")   # 200 paths left
    srv.submit(big, now=0.0)
    srv.submit(small, now=0.0)
    srv._admit()
    plan = srv.plan_step(now=0.0)
    assert [r.tag for r, _ in plan] == ["small", "big"]
    assert dict((r.tag, k) for r, k in plan) == {"small": 2, "big": 8}
    # a later tiny request overtakes a big one that has waited briefly, but not one that has
    # waited long (aging)
    late = serving.Request(0, 10, 10, 40, tag="late")    # 4000 paths
    srv.submit(late, now=0.0)
    srv._admit()
    assert srv.plan_step(now=0.0)[0][0].tag == "small"
    late.t_arrive = 10.0
    assert [r.tag for r, _ in srv.plan_step(now=10.0)][:2] == ["small", "big"]


def test_light_load_runs_everything_in_one_step():
    srv = serving.RenderServer(FakeEngine(), factory({0: 10}), step_paths=1000)
    big = serving.Request(0, 40, 40, 3, tag="big")    # 4800 paths: above one step's budget,
    small = serving.Request(0, 10, 10, 2, tag="small")  # but all work fits 8 steps' worth
    srv.submit(big, now=0.0)
    srv.submit(small, now=0.0)
    srv._admit()
    plan = dict((r.tag, k) for r, k in srv.plan_step(now=0.0))
    assert plan == {"small": 2, "big": 3}
    srv.step()
    assert srv.idle() and srv.steps == 1
