"""Pin the CPU oracle to the reference (CPU, no GPU needed).

1. The oracle core compiled against the reference's own fresnel/common/*.h headers
   (oracle/_ref) and against the restatement (oracle/_build) gives bit-identical images on
   every geometry type (polygons included), both tracers, orthographic and perspective (depth
   of field) cameras.
2. The reference's own pytest suite, run unmodified on the oracle, passes its golden-image
   comparisons (fresnel/test/reference/*.png).
3. The oracle reproduces the committed golden fixtures bit for bit.
Parts 1 and 2 need the reference tree and skip without it.
"""

import math
import os

import numpy
import pytest

import fresnel_b200 as fresnel
from fresnel_b200 import workloads
from oracle import cpu_module
from parity import path_render, preview_hits

import reference_overlay

HERE = os.path.dirname(os.path.abspath(__file__))
ref_lib = pytest.mark.skipif(not os.path.exists(cpu_module.LIB_PATHS["reference"]),
                             reason="oracle/_ref not built (reference tree absent)")


def _dof(d):
    s = workloads.hex_spheres(d)
    s.camera = fresnel.camera.Perspective(position=(0, -3, 12), look_at=(0, 0, 0), up=(0, 1, 0),
                                          focal_length=0.5, focus_distance=12, f_stop=2.0,
                                          height=0.24)
    return s


def _materials(d):
    s = workloads.hex_spheres(d)
    g = s.geometry[0]
    g.material = fresnel.material.Material(color=(0.8, 0.2, 0.2), roughness=0.2, metal=0.7,
                                           specular=0.9, spec_trans=0.3, primitive_color_mix=0.5)
    g.color[:] = numpy.linspace(0, 1, 18, dtype=numpy.float32).reshape(6, 3)
    return s


SCENES = {
    "hex": workloads.hex_spheres,
    "mixed": lambda d: workloads.config3(d, scale=0.002),
    "dof": _dof,
    "materials": _materials,
    "polygons": lambda d: workloads.polygons(d, nx=8, ny=6, spheres=10),
}


@ref_lib
@pytest.mark.parametrize("name", list(SCENES))
def test_restated_equals_reference_headers(name):
    res = cpu_module.make_device("restated")
    ref = cpu_module.make_device("reference")
    for aa in (1, 2):
        a = preview_hits(res, SCENES[name](res), 48, 40, aa)
        b = preview_hits(ref, SCENES[name](ref), 48, 40, aa)
        for x, y in zip(a, b):
            numpy.testing.assert_array_equal(x, y)
    a = path_render(res, SCENES[name](res), 40, 32, 3, 2, seed=4)
    b = path_render(ref, SCENES[name](ref), 40, 32, 3, 2, seed=4)
    numpy.testing.assert_array_equal(a[0], b[0])
    numpy.testing.assert_array_equal(a[1], b[1])


@ref_lib
def test_building_blocks_match_reference():
    res = cpu_module.load("restated")
    ref = cpu_module.load("reference")
    rng = numpy.random.default_rng(5)
    f = cpu_module.ptr
    for _ in range(200):
        m = cpu_module.FrMaterial()
        m.solid = 0.0
        m.color[:] = rng.uniform(0, 1, 3)
        m.primitive_color_mix, m.roughness, m.specular, m.metal, m.spec_trans = rng.uniform(0, 1, 5)
        n = rng.normal(size=3).astype(numpy.float32)
        n /= numpy.linalg.norm(n)
        v = rng.normal(size=3).astype(numpy.float32)
        v /= numpy.linalg.norm(v)
        key = rng.integers(0, 2**32, 2, dtype=numpy.uint64)
        o1 = numpy.zeros(5, numpy.float32)
        o2 = numpy.zeros(5, numpy.float32)
        args = (int(rng.integers(0, 5)), int(rng.integers(0, 10**6)), int(key[0]), int(key[1]))
        res.or_mis_sample(m, f(n), f(v), *args, f(o1))
        ref.or_mis_sample(m, f(n), f(v), *args, f(o2))
        numpy.testing.assert_array_equal(o1, o2)
        sc = rng.uniform(0, 1, 3).astype(numpy.float32)
        b1 = numpy.zeros(3, numpy.float32)
        b2 = numpy.zeros(3, numpy.float32)
        res.or_brdf(m, f(o1[:3].copy()), f(v), f(n), f(sc), f(b1))
        ref.or_brdf(m, f(o1[:3].copy()), f(v), f(n), f(sc), f(b2))
        numpy.testing.assert_array_equal(b1, b2)
        c = rng.uniform(-0.1, 1.5, 4).astype(numpy.float32)
        s1 = numpy.zeros(4, numpy.uint8)
        s2 = numpy.zeros(4, numpy.uint8)
        res.or_srgb(f(c), cpu_module.ptr(s1, cpu_module._bp))
        ref.or_srgb(f(c), cpu_module.ptr(s2, cpu_module._bp))
        if numpy.all(c[:3] >= 0):
            numpy.testing.assert_array_equal(s1, s2)


# The two failures expected from the reference suite come from its own camera.py:
# eval(repr(camera)) breaks because numpy >= 2 prints float32 scalars as np.float32(...).
EXPECTED_FAILURES = {"test_camera_orthographic.py::test_orthographic_attributes",
                     "test_camera_perspective.py::test_perspective_attributes"}


@pytest.mark.slow
@pytest.mark.skipif(not reference_overlay.available(), reason="reference tree absent")
def test_reference_suite_on_oracle():
    rc, out = reference_overlay.run("restated", ["-rf"])
    failed = {line.split(" ")[1].split("[")[0].replace("test/", "")
              for line in out.splitlines() if line.startswith("FAILED ")}
    assert failed <= EXPECTED_FAILURES, out[-3000:]
    passed = [line for line in out.splitlines() if " passed" in line]
    assert passed, out[-3000:]
    n_passed = int(passed[-1].split(" passed")[0].split()[-1])
    assert n_passed >= 100, out[-2000:]


@pytest.mark.parametrize("name", ["hex_preview", "hex_preview_aa", "mixed_preview",
                                  "spheres_1k_path", "dense_path", "polygons_preview",
                                  "polygons_path"])
def test_oracle_reproduces_golden_fixtures(name):
    import golden.make_golden as mg
    dev = cpu_module.make_device("restated")
    out = mg.render(name, dev)
    ref = numpy.load(os.path.join(HERE, "golden", name + ".npz"))
    for k, v in out.items():
        numpy.testing.assert_array_equal(v, ref[k], err_msg=f"{name}:{k}")
