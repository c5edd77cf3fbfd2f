"""Batched path renders (tracer.PathBatch over fr_batch_*) against plain Path.sample calls.

A render gives the same image alone or in a batch: every path's arithmetic depends only on its
(pixel, sample, light sample), and each pixel folds its samples in sample order. The tests
compare every batched tracer with a twin tracer rendered by plain ``sample`` calls (same seed)
within 1e-6. They cover renders of different scenes, image sizes, sample counts and light
samples in one batch, renders split across several waves (a small path-state size forces this),
two renders of one tracer in one batch, mixed geometry, graph reuse, and the error paths.
"""

import numpy
import pytest

import fresnel_b200 as fresnel
from fresnel_b200 import workloads

pytestmark = pytest.mark.gpu

TOL = 1e-6


@pytest.fixture
def small_slots(gpu_device):
    """Shrink the wavefront so that batches need several waves; restore afterwards."""
    dd = gpu_device._device
    old = dd.getOption("path_slots")
    dd.setOption("path_slots", 30000)
    yield
    dd.setOption("path_slots", old)


def _twins(device, w, h, seed):
    a = fresnel.tracer.Path(device, w=w, h=h)
    b = fresnel.tracer.Path(device, w=w, h=h)
    a.seed = seed
    b.seed = seed
    return a, b


def _same(a, b):
    la = numpy.array(a.linear_output[:], copy=True)
    lb = numpy.array(b.linear_output[:], copy=True)
    assert numpy.isfinite(la).all()
    diff = float(numpy.abs(la - lb).max())
    assert diff <= TOL, f"max |linear difference| {diff}"
    sa = numpy.array(a.output[:], copy=True).astype(int)
    sb = numpy.array(b.output[:], copy=True).astype(int)
    assert (numpy.abs(sa - sb) <= 1).all()


def _scenes(device):
    s1 = workloads.random_spheres(device, 300, 12.0, seed=3, outline_width=0.05)
    s2 = workloads.random_spheres(device, 2000, 30.0, seed=4, colors=True,
                                  lights=fresnel.light.lightbox())
    s3 = workloads.hex_spheres(device)
    return [s1, s2, s3]


@pytest.mark.parametrize("waves", ["one", "many"])
def test_batch_matches_plain(gpu_device, request, waves):
    if waves == "many":
        request.getfixturevalue("small_slots")
    scenes = _scenes(gpu_device)
    cases = [(scenes[0], 64, 48, 6, 1), (scenes[1], 100, 80, 9, 1), (scenes[2], 33, 17, 4, 3),
             (scenes[1], 48, 64, 5, 2), (scenes[0], 20, 20, 12, 1)]
    batch = fresnel.tracer.PathBatch(gpu_device)
    pairs = []
    for n, (scene, w, h, spp, ls) in enumerate(cases):
        a, b = _twins(gpu_device, w, h, seed=11 + n)
        a.sample(scene, samples=spp, light_samples=ls)
        batch.add(b, scene, samples=spp, light_samples=ls)
        pairs.append((a, b))
    assert len(batch) == len(cases)
    batch.render()
    assert len(batch) == 0
    for a, b in pairs:
        _same(a, b)
        assert a._tracer.getNumSamples() == b._tracer.getNumSamples()
    st = batch.stats
    assert st["renders"] == len(cases)
    assert st["graph_launches"] == 1
    if waves == "many":
        assert st["waves"] > 1
    else:
        assert st["waves"] == 1


def test_batch_continues_a_tracer(gpu_device, small_slots):
    scene = _scenes(gpu_device)[1]
    a, b = _twins(gpu_device, 70, 50, seed=5)
    a.sample(scene, samples=3)
    a.sample(scene, samples=4, reset=False, light_samples=2)
    a.sample(scene, samples=2, reset=False)
    batch = fresnel.tracer.PathBatch(gpu_device)
    batch.add(b, scene, samples=3)
    batch.add(b, scene, samples=4, reset=False, light_samples=2)
    batch.render()
    batch.add(b, scene, samples=2, reset=False)
    batch.render()
    _same(a, b)
    assert b._tracer.getNumSamples() == 9
    st = batch.stats
    assert st["graph_launches"] == 2
    assert st["graph_captures"] == 1  # the second render reuses the captured graph


def test_batch_mixed_geometry(gpu_device):
    scene = workloads.config3(gpu_device, scale=0.01)
    other = _scenes(gpu_device)[0]
    a, b = _twins(gpu_device, 80, 60, seed=9)
    c, d = _twins(gpu_device, 40, 30, seed=10)
    a.sample(scene, samples=6)
    c.sample(other, samples=5)
    batch = fresnel.tracer.PathBatch(gpu_device)
    batch.add(b, scene, samples=6)
    batch.add(d, other, samples=5)
    batch.render()
    _same(a, b)
    _same(c, d)


def test_batch_errors(gpu_device):
    scene = _scenes(gpu_device)[2]
    t = fresnel.tracer.Path(gpu_device, w=16, h=16)
    batch = fresnel.tracer.PathBatch(gpu_device)
    batch.add(t, scene, samples=2)
    with pytest.raises(RuntimeError, match="already has queued renders"):
        batch.add(t, scene, samples=2)  # reset=True on a queued tracer
    batch.clear()
    assert len(batch) == 0
    batch.render()  # empty batch: nothing to do
    assert t._tracer.getNumSamples() == 0


def test_batch_matches_oracle(gpu_device, oracle_device, small_slots):
    """Renders batched together (several waves, mixed scenes, sizes, sample and light-sample
    counts, mixed geometry) against the CPU oracle rendering each alone with the seed the tracer
    renders with: >= 99% of pixels within 1e-3 (the same-seed bar of the plain Path tests)."""
    from parity import oracle_path_image, same_seed_fraction
    from parity_record import record

    def builds():
        return [lambda d: workloads.random_spheres(d, 300, 12.0, seed=3, outline_width=0.05),
                lambda d: workloads.random_spheres(d, 2000, 30.0, seed=4, colors=True,
                                                   lights=fresnel.light.lightbox()),
                lambda d: workloads.config3(d, scale=0.005)]
    gscenes = [b(gpu_device) for b in builds()]
    oscenes = [b(oracle_device) for b in builds()]
    cases = [(0, 64, 48, 6, 1), (1, 100, 80, 5, 1), (2, 72, 40, 4, 2), (1, 40, 56, 3, 3)]
    batch = fresnel.tracer.PathBatch(gpu_device)
    tracers = []
    for n, (k, w, h, spp, ls) in enumerate(cases):
        t = fresnel.tracer.Path(gpu_device, w=w, h=h)
        t.seed = 40 + n
        batch.add(t, gscenes[k], samples=spp, light_samples=ls)
        tracers.append(t)
    batch.render()
    assert batch.stats["waves"] > 1
    for n, ((k, w, h, spp, ls), t) in enumerate(zip(cases, tracers)):
        ora = oracle_path_image(oracle_device, oscenes[k], w, h, 41 + n, spp, ls)
        frac = same_seed_fraction(numpy.array(t.linear_output[:], copy=True), ora)
        record("test_batch_matches_oracle", check="same_seed", render=n, width=w, height=h,
               spp=spp, light_samples=ls, within_1e3=frac)
        assert frac >= 0.99, f"render {n}: {frac:.4%} of pixels within 1e-3"
