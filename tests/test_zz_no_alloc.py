"""The allocation-free path render (fr_tracer_render_path_static) against fr_tracer_render_path.

fr_tracer_render_path_static keeps its wavefront state in a fixed device array instead of
tracer-owned allocations. It traces fewer samples per wavefront (262144 slots / pixels), but every
path's arithmetic depends only on its (pixel, sample, light sample), and the running mean folds
samples in sample order. Its images must therefore equal the allocating entry point's. The test
compares them within 1e-6 after each of two calls in a row (the second call continues the first
one's running mean). It also checks the size limit and the built-scene rule.

The file name sorts last so that pytest collects it after every other test. It passes alone too.
"""

import numpy
import pytest

import fresnel_b200 as fresnel
from fresnel_b200 import workloads

pytestmark = pytest.mark.gpu

TOL = 1e-6


def _scene(device):
    return workloads.config1(device)


def _pair(device, w, h, light_samples):
    scene = _scene(device)
    a = fresnel.tracer.Path(device, w=w, h=h)
    b = fresnel.tracer.Path(device, w=w, h=h)
    for t in (a, b):
        t.reset()
        t.seed = 7
        t._tracer.setLightSamples(light_samples)
    return scene, a, b


@pytest.mark.parametrize("w,h,spp,ls", [(200, 150, 24, 1), (96, 64, 10, 3)])
def test_static_render_matches_allocating_render(gpu_device, w, h, spp, ls):
    scene, a, b = _pair(gpu_device, w, h, ls)
    scene._scene.build()
    for call in range(2):
        a._tracer.renderSamples(scene._scene, spp)
        b._tracer.renderSamplesStatic(scene._scene, spp)
        la = numpy.array(a.linear_output[:], copy=True)
        lb = numpy.array(b.linear_output[:], copy=True)
        assert la.shape == (h, w, 4)
        assert numpy.isfinite(la).all()
        diff = numpy.abs(la - lb).max()
        assert diff <= TOL, f"call {call}: max |linear difference| {diff}"
        sa = numpy.array(a.output[:], copy=True)
        sb = numpy.array(b.output[:], copy=True)
        assert (numpy.abs(sa.astype(int) - sb.astype(int)) <= 1).all()
    assert a._tracer.getNumSamples() == b._tracer.getNumSamples() == 2 * spp


def test_static_render_limits(gpu_device):
    scene = _scene(gpu_device)
    big = fresnel.tracer.Path(gpu_device, w=1024, h=512)
    scene._scene.build()
    with pytest.raises(RuntimeError, match="limit of 262144 pixels"):
        big._tracer.renderSamplesStatic(scene._scene, 1)

    small = fresnel.tracer.Path(gpu_device, w=64, h=64)
    scene.geometry[0].position[0] = (0.25, 0.5, 0.75)  # the BVH is now stale
    with pytest.raises(RuntimeError, match="needs a built scene"):
        small._tracer.renderSamplesStatic(scene._scene, 1)
    scene._scene.build()
    small._tracer.renderSamplesStatic(scene._scene, 2)
    assert numpy.isfinite(small.linear_output[:]).all()
