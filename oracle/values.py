"""TEST INFRASTRUCTURE: fresnel's ``_common`` value types in plain Python, for the CPU oracle.

fresnel's Python package takes its value types from the compiled ``_common`` module
(fresnel/common/module-common.cc:37-115): RGBf, vec3f, Material, UserCamera, CameraModel,
CameraBasis, Lights, cpu_built() and gpu_built().  This module provides the same names with the
same fields, so that the reference's own Python package (or this repository's, or the oracle
alone) can drive the oracle with no compiled module of the product loaded.  Fields hold float32
values, as the C++ structs do: every assignment rounds to float32.

Defaults follow the reference's structs where it has them (fresnel/common/Camera.h:57-68 for
UserCamera); where the reference leaves a field uninitialised (Material, Lights) it starts at 0,
and fresnel's Python layer assigns every field before use.
"""

import enum

import numpy

_f32 = numpy.float32


def _f(v):
    return float(_f32(v))


class _Record:
    """A plain struct of float32 fields (``_FIELDS``), plus nested value fields."""

    _FIELDS = ()

    def __setattr__(self, name, value):
        if name in self._FIELDS:
            value = _f(value)
        object.__setattr__(self, name, value)


class RGBf(_Record):
    _FIELDS = ("r", "g", "b")

    def __init__(self, r=0.0, g=0.0, b=0.0):
        self.r, self.g, self.b = r, g, b

    def __repr__(self):
        return f"RGBf({self.r}, {self.g}, {self.b})"


class vec3f(_Record):  # noqa: N801 - fresnel's name
    _FIELDS = ("x", "y", "z")

    def __init__(self, x=0.0, y=0.0, z=0.0):
        self.x, self.y, self.z = x, y, z

    def __repr__(self):
        return f"vec3f({self.x}, {self.y}, {self.z})"


def _vec(v):
    return vec3f(v.x, v.y, v.z)


class Material(_Record):
    _FIELDS = ("solid", "primitive_color_mix", "roughness", "specular", "spec_trans", "metal")

    def __init__(self):
        self.solid = 0.0
        self.color = RGBf()
        self.primitive_color_mix = 0.0
        self.roughness = 0.0
        self.specular = 0.0
        self.spec_trans = 0.0
        self.metal = 0.0

    def __setattr__(self, name, value):
        if name == "color":
            value = RGBf(value.r, value.g, value.b)
        super().__setattr__(name, value)


class CameraModel(enum.IntEnum):
    """fresnel::CameraModel (fresnel/common/Camera.h): orthographic = 0, perspective = 1."""
    orthographic = 0
    perspective = 1


class UserCamera(_Record):
    _FIELDS = ("h", "f", "f_stop", "focus_distance")

    def __init__(self):
        self.position = vec3f(0, 0, 0)
        self.look_at = vec3f(0, 0, 1)
        self.up = vec3f(0, 1, 0)
        self.h = 1.0
        self.f = 1.0
        self.f_stop = 1.0
        self.focus_distance = 1.0
        self.model = CameraModel.orthographic

    def __setattr__(self, name, value):
        if name in ("position", "look_at", "up"):
            value = _vec(value)
        elif name == "model":
            value = CameraModel(int(value))
        super().__setattr__(name, value)


class CameraBasis:
    """Orthonormal camera basis (fresnel/common/Camera.h:89-113): u right, v up, w backward,
    evaluated in float32 in the reference's operation order."""

    def __init__(self, cam):
        def v3(a):
            return numpy.array([a.x, a.y, a.z], dtype=_f32)

        def dot(a, b):
            return _f32(_f32(a[0] * b[0]) + _f32(a[1] * b[1])) + _f32(a[2] * b[2])

        def cross(a, b):
            return numpy.array([_f32(a[1] * b[2]) - _f32(a[2] * b[1]),
                                _f32(a[2] * b[0]) - _f32(a[0] * b[2]),
                                _f32(a[0] * b[1]) - _f32(a[1] * b[0])], dtype=_f32)

        def unit(a):
            return a * (_f32(1.0) / numpy.sqrt(dot(a, a), dtype=_f32))

        d = unit(v3(cam.look_at) - v3(cam.position))
        v = unit(v3(cam.up))
        u = unit(cross(d, v))
        v = unit(cross(u, d))
        self.u = vec3f(*u)
        self.v = vec3f(*v)
        self.w = vec3f(*(-d))


class Lights:
    """Up to 4 lights (fresnel/common/Light.h:36-66)."""

    def __init__(self):
        self.N = 0
        self._direction = [vec3f() for _ in range(4)]
        self._color = [RGBf() for _ in range(4)]
        self._theta = [0.0] * 4

    @staticmethod
    def _slot(i):
        if not 0 <= int(i) < 4:
            raise IndexError("light index out of range (at most 4 lights)")
        return int(i)

    def getDirection(self, i):
        return _vec(self._direction[self._slot(i)])

    def setDirection(self, i, v):
        self._direction[self._slot(i)] = _vec(v)

    def getColor(self, i):
        c = self._color[self._slot(i)]
        return RGBf(c.r, c.g, c.b)

    def setColor(self, i, c):
        self._color[self._slot(i)] = RGBf(c.r, c.g, c.b)

    def getTheta(self, i):
        return self._theta[self._slot(i)]

    def setTheta(self, i, t):
        self._theta[self._slot(i)] = _f(t)


def cpu_built():
    return True


def gpu_built():
    return False


def find_polyhedron_faces(vertices):
    raise RuntimeError("find_polyhedron_faces is not provided by the oracle's value types")
