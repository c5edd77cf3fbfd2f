"""Autotuner search logic against a fake device and a synthetic cost (no GPU)."""

from fresnel_b200 import autotune


class FakeDev:
    def __init__(self):
        self.opts = {"leaf_max": 2.0, "tile": 8.0, "path_slots": float(32 << 20)}
        self.sets = []

    def getOption(self, name):
        return self.opts[name]

    def setOption(self, name, value):
        self.sets.append((name, value))
        self.opts[name] = float(value)


class FakeDevice:
    def __init__(self):
        self._device = FakeDev()


class FakeScene:
    geometry = []


def cost(device, jobs, spp):
    o = device._device.opts
    # separable bowl with its minimum at leaf 4, tile 16, 16M slots
    return (1.0 + abs(o["leaf_max"] - 4) + 0.5 * abs(o["tile"] - 16) / 4
            + abs(o["path_slots"] - (16 << 20)) / (8 << 20))


def test_coordinate_descent_finds_the_separable_minimum():
    dev = FakeDevice()
    t = autotune.Tuner(dev, timer=cost)
    jobs = [(FakeScene(), 64, 64, 1)]
    best, ms = t.tune(jobs)
    assert best == {"leaf_max": 4, "tile": 16, "path_slots": 16 << 20}
    assert ms == 1.0
    # applied to the device
    assert dev._device.opts == {"leaf_max": 4.0, "tile": 16.0, "path_slots": float(16 << 20)}
    # cost: the start point plus every other value of every knob
    assert len(t.log) == 1 + 3 + 2 + 3


def test_cache_and_apply_false():
    dev = FakeDevice()
    t = autotune.Tuner(dev, timer=cost)
    jobs = [(FakeScene(), 64, 64, 1)]
    t.tune(jobs, apply=False)
    assert dev._device.opts["leaf_max"] == 2.0  # restored
    n = len(t.log)
    best, _ = t.tune(jobs)  # cached: no new measurements, but applied
    assert len(t.log) == n
    assert dev._device.opts["leaf_max"] == 4.0 and best["tile"] == 16


def test_signature_buckets():
    a = autotune.signature([(FakeScene(), 100, 100, 1)])
    b = autotune.signature([(FakeScene(), 110, 100, 1)])
    c = autotune.signature([(FakeScene(), 400, 400, 1)])
    assert a == b and a != c
