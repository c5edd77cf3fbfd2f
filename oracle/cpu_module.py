"""TEST INFRASTRUCTURE: the CPU oracle behind fresnel's backend-module interface.

This module exposes the class names of fresnel's ``_cpu`` pybind11 module
(fresnel/cpu/module-cpu.cc: Device, Scene, Geometry*, Tracer, TracerDirect, TracerPath) on top
of the oracle library (oracle/oracle_core.cpp) through ctypes, so that scenes built with the
fresnel Python API can be rendered by the oracle for comparison.  Only tests, the smoke check
and bench.py's CPU-baseline leg use it; the product never imports it.

``load(kind)`` selects the library: ``"restated"`` (oracle/_build/liboracle.so) or
``"reference"`` (oracle/_ref/libfresnel_ref.so, the reference's own math headers).
"""

import ctypes
import os

import numpy

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATHS = {
    "restated": os.path.join(HERE, "_build", "liboracle.so"),
    "reference": os.path.join(HERE, "_ref", "libfresnel_ref.so"),
}

FR_GEOM_SPHERE, FR_GEOM_CYLINDER, FR_GEOM_POLYHEDRON, FR_GEOM_MESH, FR_GEOM_POLYGON = 0, 1, 2, 3, 4

_fp = ctypes.POINTER(ctypes.c_float)
_up = ctypes.POINTER(ctypes.c_uint32)
_bp = ctypes.POINTER(ctypes.c_uint8)


class FrMaterial(ctypes.Structure):
    _fields_ = [("solid", ctypes.c_float), ("color", ctypes.c_float * 3),
                ("primitive_color_mix", ctypes.c_float), ("roughness", ctypes.c_float),
                ("specular", ctypes.c_float), ("metal", ctypes.c_float),
                ("spec_trans", ctypes.c_float)]


class FrUserCamera(ctypes.Structure):
    _fields_ = [("position", ctypes.c_float * 3), ("look_at", ctypes.c_float * 3),
                ("up", ctypes.c_float * 3), ("h", ctypes.c_float), ("f", ctypes.c_float),
                ("f_stop", ctypes.c_float), ("focus_distance", ctypes.c_float),
                ("model", ctypes.c_int32)]


class FrLights(ctypes.Structure):
    _fields_ = [("direction", (ctypes.c_float * 3) * 4), ("color", (ctypes.c_float * 3) * 4),
                ("theta", ctypes.c_float * 4), ("n", ctypes.c_uint32)]


class FrRenderParams(ctypes.Structure):
    _fields_ = [("camera", FrUserCamera), ("lights", FrLights),
                ("background_color", ctypes.c_float * 3), ("background_alpha", ctypes.c_float),
                ("seed", ctypes.c_uint32), ("highlight_warning", ctypes.c_int32),
                ("highlight_color", ctypes.c_float * 3)]


class OrGeometryDesc(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int32), ("enabled", ctypes.c_int32), ("n", ctypes.c_uint32),
                ("position", _fp), ("radius", _fp), ("color", _fp), ("points", _fp),
                ("orientation", _fp), ("vertices", _fp), ("n_vertices", ctypes.c_uint32),
                ("plane_origin", _fp), ("plane_normal", _fp), ("plane_color", _fp),
                ("n_planes", ctypes.c_uint32), ("poly_radius", ctypes.c_float),
                ("color_by_face", ctypes.c_float), ("material", FrMaterial),
                ("outline_material", FrMaterial), ("outline_width", ctypes.c_float),
                ("angle", _fp), ("rounding_radius", ctypes.c_float)]


class OrStats(ctypes.Structure):
    _fields_ = [("rays", ctypes.c_uint64), ("box_tests", ctypes.c_uint64),
                ("prim_tests", ctypes.c_uint64), ("paths", ctypes.c_uint64),
                ("nonfinite", ctypes.c_uint64)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


_LIBS = {}


def load(kind="restated"):
    """Load (once) and return the oracle library of the given kind."""
    if kind in _LIBS:
        return _LIBS[kind]
    path = LIB_PATHS[kind]
    if not os.path.exists(path):
        raise FileNotFoundError(f"oracle library {path} is not built (python oracle/build_oracle.py)")
    lib = ctypes.CDLL(path)
    lib.or_scene_create.restype = ctypes.c_void_p
    lib.or_scene_create.argtypes = [ctypes.POINTER(OrGeometryDesc), ctypes.c_uint32, ctypes.c_int]
    lib.or_scene_destroy.argtypes = [ctypes.c_void_p]
    lib.or_scene_info.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64),
                                  ctypes.POINTER(ctypes.c_uint64)]
    lib.or_render_path.argtypes = [ctypes.c_void_p, ctypes.POINTER(FrRenderParams), ctypes.c_uint32,
                                   ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                   ctypes.c_uint32, _fp, _bp, _fp, _up, ctypes.c_uint32,
                                   ctypes.c_int, ctypes.c_int, ctypes.POINTER(OrStats)]
    lib.or_render_preview.argtypes = [ctypes.c_void_p, ctypes.POINTER(FrRenderParams),
                                      ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _fp, _bp,
                                      _up, ctypes.c_int, ctypes.POINTER(OrStats)]
    lib.or_trace.argtypes = [ctypes.c_void_p, _fp, _fp, ctypes.c_float, _fp, _up, _up]
    lib.or_prim_hit.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, _fp, _fp,
                                ctypes.c_float, _fp]
    lib.or_philox4x32_10.argtypes = [_up, _up, _up]
    lib.or_u01.restype = ctypes.c_float
    lib.or_u01.argtypes = [ctypes.c_uint32]
    lib.or_srgb.argtypes = [_fp, _bp]
    lib.or_camera_ray.argtypes = [ctypes.POINTER(FrUserCamera), ctypes.c_uint32, ctypes.c_uint32,
                                  ctypes.c_uint32, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32,
                                  ctypes.c_uint32, _fp, _fp]
    lib.or_mis_sample.argtypes = [ctypes.POINTER(FrMaterial), _fp, _fp, ctypes.c_uint32,
                                  ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _fp]
    lib.or_brdf.argtypes = [ctypes.POINTER(FrMaterial), _fp, _fp, _fp, _fp, _fp]
    lib.or_math_kind.restype = ctypes.c_char_p
    lib.or_set_ray_log.argtypes = [_fp, ctypes.c_uint64]
    lib.or_ray_log_count.restype = ctypes.c_uint64
    lib.or_grid_walk_stats.argtypes = [ctypes.c_void_p, ctypes.c_uint32, _fp, _fp, ctypes.c_uint32,
                                       ctypes.c_float, _fp, ctypes.c_uint64, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_double)]
    lib.or_parts_grid_walk_stats.argtypes = [ctypes.c_void_p, ctypes.c_float, _fp, ctypes.c_uint64,
                                             ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    _LIBS[kind] = lib
    return lib


def ptr(a, typ=_fp):
    """ctypes pointer to a C-contiguous numpy array (None passes through)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(typ)


# ------------------------------------------------------------------------------------------
# conversions from the fresnel value types (_common.Material / UserCamera / Lights)
# ------------------------------------------------------------------------------------------
def material_struct(m):
    s = FrMaterial()
    s.solid = m.solid
    s.color[:] = (m.color.r, m.color.g, m.color.b)
    s.primitive_color_mix = m.primitive_color_mix
    s.roughness = m.roughness
    s.specular = m.specular
    s.metal = m.metal
    s.spec_trans = m.spec_trans
    return s


def camera_struct(c):
    s = FrUserCamera()
    s.position[:] = (c.position.x, c.position.y, c.position.z)
    s.look_at[:] = (c.look_at.x, c.look_at.y, c.look_at.z)
    s.up[:] = (c.up.x, c.up.y, c.up.z)
    s.h, s.f, s.f_stop, s.focus_distance = c.h, c.f, c.f_stop, c.focus_distance
    s.model = int(c.model)
    return s


def lights_struct(lights):
    s = FrLights()
    n = min(int(lights.N), 4)
    s.n = n
    for i in range(n):
        d = lights.getDirection(i)
        c = lights.getColor(i)
        s.direction[i][:] = (d.x, d.y, d.z)
        s.color[i][:] = (c.r, c.g, c.b)
        s.theta[i] = lights.getTheta(i)
    return s


def _common_module():
    """The value types handed back to the caller: those of fresnel_b200._common when the
    caller's package is already loaded (tests compare the two backends through one API),
    otherwise the oracle's own plain-Python ones (oracle/values.py), so that the oracle runs
    with no compiled module of the product loaded."""
    import sys
    if "fresnel_b200" in sys.modules:
        from fresnel_b200 import _common
        return _common
    from oracle import values
    return values


def _copy_material(m):
    _common = _common_module()
    r = _common.Material()
    for k in ("solid", "primitive_color_mix", "roughness", "specular", "spec_trans", "metal"):
        setattr(r, k, getattr(m, k))
    r.color = _common.RGBf(m.color.r, m.color.g, m.color.b)
    return r


def _default_material(color, solid=0.0):
    """fresnel::Material(color, solid) (fresnel/common/Material.h:59-64)."""
    _common = _common_module()
    m = _common.Material()
    m.solid = solid
    m.color = _common.RGBf(*color)
    m.primitive_color_mix = 0.0
    m.roughness = 0.1
    m.specular = 0.5
    m.metal = 0.0
    m.spec_trans = 0.0
    return m


class _Buffer(numpy.ndarray):
    """Host array with the backend Array map()/unmap() interface (no-ops on the CPU)."""

    def map(self):
        pass

    def unmap(self):
        pass


def _buffer(shape, dtype=numpy.float32):
    return numpy.zeros(shape, dtype=dtype).view(_Buffer)


# ------------------------------------------------------------------------------------------
# backend classes
# ------------------------------------------------------------------------------------------
class Device:
    """Oracle device (fresnel/cpu/Device.cc).  ``n`` is accepted; renders always use every
    hardware thread (results do not depend on the thread count)."""

    kind = "restated"

    def __init__(self, n=-1):
        self.lib = load(self.kind)
        self.threads = 0

    def describe(self):
        return f"CPU oracle ({self.lib.or_math_kind().decode()} math), {os.cpu_count()} threads"


class Scene:
    """fresnel/cpu/Scene.cc:15-28 defaults: black background, alpha 0, two lights."""

    def __init__(self, device):
        _common = _common_module()
        self._device = device
        self._camera = _common.UserCamera()
        self._bg = _common.RGBf(0, 0, 0)
        self._bg_alpha = 0.0
        self._lights = _common.Lights()
        self._lights.N = 2
        self._lights.setDirection(0, _common.vec3f(-1, 0.3, 1))
        self._lights.setColor(0, _common.RGBf(1, 1, 1))
        self._lights.setDirection(1, _common.vec3f(1, 0, 1))
        self._lights.setColor(1, _common.RGBf(0.1, 0.1, 0.1))
        self._geoms = []
        self._version = 0
        self._built = None  # (version, handle, keepalive)
        self.leaf_max = 4

    def getDevice(self):
        return self._device

    def setCamera(self, cam):
        # copy into the object getCamera() hands out (a reference, as in the reference module)
        for k in ("position", "look_at", "up", "h", "f", "f_stop", "focus_distance", "model"):
            setattr(self._camera, k, getattr(cam, k))

    def getCamera(self):
        return self._camera

    def getBackgroundColor(self):
        return self._bg

    def setBackgroundColor(self, c):
        self._bg = _common_module().RGBf(c.r, c.g, c.b)

    def getBackgroundAlpha(self):
        return self._bg_alpha

    def setBackgroundAlpha(self, a):
        self._bg_alpha = float(a)

    def getLights(self):
        return self._lights

    def setLights(self, lights):
        L = self._lights  # copy into the object getLights() hands out
        n = int(lights.N)
        for i in range(min(n, 4)):
            L.setDirection(i, lights.getDirection(i))
            L.setColor(i, lights.getColor(i))
            L.setTheta(i, lights.getTheta(i))
        L.N = n

    def _touch(self):
        self._version += 1

    def handle(self):
        """The oracle scene (built on first use after any change)."""
        if self._built is not None and self._built[0] == self._version:
            return self._built[1]
        if self._built is not None:
            self._device.lib.or_scene_destroy(self._built[1])
            self._built = None
        descs = (OrGeometryDesc * max(1, len(self._geoms)))()
        keep = []
        for i, g in enumerate(self._geoms):
            g._fill(descs[i], keep)
        h = self._device.lib.or_scene_create(descs, len(self._geoms), self.leaf_max)
        if not h:
            raise RuntimeError("oracle scene construction failed")
        self._built = (self._version, h, keep)
        return h

    def info(self):
        n = ctypes.c_uint64()
        p = ctypes.c_uint64()
        self._device.lib.or_scene_info(self.handle(), ctypes.byref(n), ctypes.byref(p))
        return int(n.value), int(p.value)

    def __del__(self):
        try:
            if self._built is not None:
                self._device.lib.or_scene_destroy(self._built[1])
        except Exception:
            pass


class Geometry:
    """fresnel/cpu/Geometry.cc; materials default to Material((1,0,1)) and a solid black
    outline (fresnel/cpu/GeometrySphere.cc:31-33)."""

    def __init__(self, scene):
        self._scene = scene
        self._valid = True
        self._enabled = True
        self._material = _default_material((1, 0, 1))
        self._outline = _default_material((0, 0, 0), 1.0)
        self._outline_width = 0.0
        scene._geoms.append(self)
        scene._touch()

    def getMaterial(self):
        return _copy_material(self._material)

    def setMaterial(self, m):
        self._material = _copy_material(m)
        self._scene._touch()

    def getOutlineMaterial(self):
        return _copy_material(self._outline)

    def setOutlineMaterial(self, m):
        self._outline = _copy_material(m)
        self._scene._touch()

    def getOutlineWidth(self):
        return self._outline_width

    def setOutlineWidth(self, w):
        self._outline_width = float(w)
        self._scene._touch()

    def enable(self):
        if not self._valid:
            raise RuntimeError("Cannot enable inactive Geometry")
        self._enabled = True
        self._scene._touch()

    def disable(self):
        if not self._valid:
            raise RuntimeError("Cannot disable inactive Geometry")
        self._enabled = False
        self._scene._touch()

    def remove(self):
        if self._valid:
            self._valid = False
            self._scene._touch()

    def update(self):
        self._scene._touch()

    def _fill_common(self, d, typ, n):
        d.type = typ
        d.enabled = 1 if (self._valid and self._enabled) else 0
        d.n = n
        d.material = material_struct(self._material)
        d.outline_material = material_struct(self._outline)
        d.outline_width = self._outline_width


def _c(a):
    return numpy.ascontiguousarray(a, dtype=numpy.float32)


class GeometrySphere(Geometry):
    def __init__(self, scene, N):
        super().__init__(scene)
        self._position = _buffer((N, 3))
        self._radius = _buffer((N,))
        self._color = _buffer((N, 3))

    def getPositionBuffer(self):
        return self._position

    def getRadiusBuffer(self):
        return self._radius

    def getColorBuffer(self):
        return self._color

    def _fill(self, d, keep):
        p, r, c = _c(self._position), _c(self._radius), _c(self._color)
        keep += [p, r, c]
        self._fill_common(d, FR_GEOM_SPHERE, len(r))
        d.position, d.radius, d.color = ptr(p), ptr(r), ptr(c)


class GeometryCylinder(Geometry):
    def __init__(self, scene, N):
        super().__init__(scene)
        self._points = _buffer((N, 2, 3))
        self._radius = _buffer((N,))
        self._color = _buffer((N, 2, 3))

    def getPointsBuffer(self):
        return self._points

    def getRadiusBuffer(self):
        return self._radius

    def getColorBuffer(self):
        return self._color

    def _fill(self, d, keep):
        p, r, c = _c(self._points), _c(self._radius), _c(self._color)
        keep += [p, r, c]
        self._fill_common(d, FR_GEOM_CYLINDER, len(r))
        d.points, d.radius, d.color = ptr(p), ptr(r), ptr(c)


class GeometryConvexPolyhedron(Geometry):
    """Plane normals are normalised on ingest as n * (1 / sqrt(n.n))
    (fresnel/cpu/GeometryConvexPolyhedron.cc:85-86)."""

    def __init__(self, scene, origins, normals, colors, N, r):
        o = numpy.ascontiguousarray(origins, dtype=numpy.float32)
        n = numpy.ascontiguousarray(normals, dtype=numpy.float32)
        c = numpy.ascontiguousarray(colors, dtype=numpy.float32)
        if o.ndim != 2:
            raise RuntimeError("plane_origins must be a 2-dimensional array")
        if o.shape[1] != 3:
            raise RuntimeError("plane_origins must be a Nvert by 3 array")
        if n.ndim != 2:
            raise RuntimeError("plane_normals must be a 2-dimensional array")
        if n.shape[1] != 3:
            raise RuntimeError("plane_normals must be a Nvert by 3 array")
        if n.shape[0] != o.shape[0]:
            raise RuntimeError("Number of vertices must match in origin and normal arrays")
        if c.ndim != 2:
            raise RuntimeError("plane_colors must be a 2-dimensional array")
        if c.shape[1] != 3:
            raise RuntimeError("plane_colors must be a Nvert by 3 array")
        if c.shape[0] != o.shape[0]:
            raise RuntimeError("Number of vertices must match in origin and color arrays")
        super().__init__(scene)
        nn = numpy.empty_like(n)
        for i in range(n.shape[0]):
            v = n[i]
            ln2 = numpy.float32(v[0] * v[0]) + numpy.float32(v[1] * v[1])
            ln2 = numpy.float32(ln2 + numpy.float32(v[2] * v[2]))
            q = numpy.float32(1.0) / numpy.sqrt(ln2, dtype=numpy.float32)
            nn[i] = v * q
        self._origins, self._normals, self._colors = o, nn, c
        self._poly_radius = float(r)
        self._color_by_face = 0.0
        self._position = _buffer((N, 3))
        self._orientation = _buffer((N, 4))
        self._color = _buffer((N, 3))

    def getPositionBuffer(self):
        return self._position

    def getOrientationBuffer(self):
        return self._orientation

    def getColorBuffer(self):
        return self._color

    def setColorByFace(self, f):
        self._color_by_face = float(f)
        self._scene._touch()

    def getColorByFace(self):
        return self._color_by_face

    def _fill(self, d, keep):
        p, q, c = _c(self._position), _c(self._orientation), _c(self._color)
        keep += [p, q, c]
        self._fill_common(d, FR_GEOM_POLYHEDRON, p.shape[0])
        d.position, d.orientation, d.color = ptr(p), ptr(q), ptr(c)
        d.plane_origin, d.plane_normal = ptr(self._origins), ptr(self._normals)
        d.plane_color = ptr(self._colors)
        d.n_planes = self._origins.shape[0]
        d.poly_radius = self._poly_radius
        d.color_by_face = self._color_by_face


class GeometryMesh(Geometry):
    def __init__(self, scene, vertices, N):
        v = numpy.ascontiguousarray(vertices, dtype=numpy.float32)
        if v.ndim != 2:
            raise RuntimeError("vertices must be a 2-dimensional array")
        if v.shape[1] != 3:
            raise RuntimeError("vertices must be a Nvert by 3 array")
        if v.shape[0] % 3 != 0:
            raise RuntimeError("the number of triangle vertices must be a multiple of three.")
        super().__init__(scene)
        self._vertices = v
        self._position = _buffer((N, 3))
        self._orientation = _buffer((N, 4))
        self._color = _buffer((v.shape[0], 3))

    def getPositionBuffer(self):
        return self._position

    def getOrientationBuffer(self):
        return self._orientation

    def getColorBuffer(self):
        return self._color

    def _fill(self, d, keep):
        p, q, c = _c(self._position), _c(self._orientation), _c(self._color)
        keep += [p, q, c]
        self._fill_common(d, FR_GEOM_MESH, p.shape[0])
        d.position, d.orientation, d.color = ptr(p), ptr(q), ptr(c)
        d.vertices, d.n_vertices = ptr(self._vertices), self._vertices.shape[0]


class GeometryPolygon(Geometry):
    """fresnel/cpu/GeometryPolygon.cc:20-82: vertices (N_vert, 2); position (N, 2), angle (N,),
    colour (N, 3) per polygon; the radius is the farthest vertex plus the rounding radius."""

    def __init__(self, scene, vertices, rounding_radius, N):
        v = numpy.ascontiguousarray(vertices, dtype=numpy.float32)
        if v.ndim != 2:
            raise RuntimeError("vertices must be a 2-dimensional array")
        if v.shape[1] != 2:
            raise RuntimeError("vertices must be a Nvert by 2 array")
        super().__init__(scene)
        self._vertices = v
        self._rounding_radius = float(numpy.float32(rounding_radius))
        r = numpy.float32(0)
        for x, y in v:
            r = max(r, numpy.sqrt(numpy.float32(x * x) + numpy.float32(y * y), dtype=numpy.float32))
        self._radius = float(numpy.float32(r + numpy.float32(self._rounding_radius)))
        self._position = _buffer((N, 2))
        self._angle = _buffer((N,))
        self._color = _buffer((N, 3))

    def getPositionBuffer(self):
        return self._position

    def getAngleBuffer(self):
        return self._angle

    def getColorBuffer(self):
        return self._color

    def getRadius(self):
        return self._radius

    def _fill(self, d, keep):
        p, a, c = _c(self._position), _c(self._angle), _c(self._color)
        keep += [p, a, c]
        self._fill_common(d, FR_GEOM_POLYGON, p.shape[0])
        d.position, d.angle, d.color = ptr(p), ptr(a), ptr(c)
        d.vertices, d.n_vertices = ptr(self._vertices), self._vertices.shape[0]
        d.rounding_radius = self._rounding_radius


class Tracer:
    """fresnel/cpu/Tracer.cc: output buffers, highlight warning, seed."""

    def __init__(self, device, w, h):
        self._device = device
        self._highlight = False
        self._highlight_color = (1.0, 0.0, 1.0)
        self._seed = 0
        self.stats = OrStats()
        self._alloc(w, h)

    def _alloc(self, w, h):
        if w == 0 or h == 0:
            raise RuntimeError("Invalid dimensions")
        self._w, self._h = int(w), int(h)
        self._linear = _buffer((h, w, 4))
        self._srgb = _buffer((h, w, 4), numpy.uint8)

    def resize(self, w, h):
        self._alloc(w, h)

    def _check(self, scene):
        if scene._device is not self._device:
            raise RuntimeError("Scene and Tracer devices do not match")

    def _params(self, scene):
        p = FrRenderParams()
        p.camera = camera_struct(scene._camera)
        p.lights = lights_struct(scene._lights)
        p.background_color[:] = (scene._bg.r, scene._bg.g, scene._bg.b)
        p.background_alpha = scene._bg_alpha
        p.seed = self._seed & 0xFFFFFFFF
        p.highlight_warning = 1 if self._highlight else 0
        p.highlight_color[:] = self._highlight_color
        return p

    def getSRGBOutputBuffer(self):
        return self._srgb

    def getLinearOutputBuffer(self):
        return self._linear

    def enableHighlightWarning(self, color):
        self._highlight = True
        self._highlight_color = (color.r, color.g, color.b)

    def disableHighlightWarning(self):
        self._highlight = False

    def getSeed(self):
        return self._seed

    def setSeed(self, seed):
        self._seed = int(seed) & 0xFFFFFFFF


class TracerDirect(Tracer):
    """fresnel/cpu/TracerDirect.cc; anti-aliasing n defaults to 8."""

    def __init__(self, device, w, h):
        super().__init__(device, w, h)
        self._aa_n = 8
        self.last_hit_ids = None
        self.record_hits = False

    def setAntialiasingN(self, n):
        self._aa_n = int(n)

    def getAntialiasingN(self):
        return self._aa_n

    def render(self, scene):
        self._check(scene)
        hits = None
        if self.record_hits:
            hits = numpy.zeros((self._h, self._w, self._aa_n * self._aa_n, 2), numpy.uint32)
        lin = numpy.ascontiguousarray(self._linear)
        srgb = numpy.ascontiguousarray(self._srgb)
        p = self._params(scene)
        rc = self._device.lib.or_render_preview(scene.handle(), ctypes.byref(p), self._w, self._h,
                                                self._aa_n, ptr(lin), ptr(srgb, _bp),
                                                ptr(hits, _up), self._device.threads,
                                                ctypes.byref(self.stats))
        if rc != 0:
            raise RuntimeError("oracle preview render failed")
        self.last_hit_ids = hits


class TracerPath(Tracer):
    """fresnel/cpu/TracerPath.cc: progressive sampling with Welford's running mean."""

    def __init__(self, device, w, h, light_samples):
        super().__init__(device, w, h)
        self._light_samples = int(light_samples)
        self._n_samples = 0
        self.nan_guard = False
        self.m2 = None  # optional Welford M2 buffer [h, w, 3]
        self.reset()

    def reset(self):
        self._n_samples = 0
        self._seed = (self._seed + 1) & 0xFFFFFFFF
        self._linear[...] = 0
        self._srgb[...] = 0
        if self.m2 is not None:
            self.m2[...] = 0

    def resize(self, w, h):
        self._alloc(w, h)
        self._n_samples = 0
        self._seed = (self._seed + 1) & 0xFFFFFFFF

    def getNumSamples(self):
        return self._n_samples

    def setLightSamples(self, n):
        self._light_samples = int(n)

    def render(self, scene):
        self.renderSamples(scene, 1)

    def renderSamples(self, scene, k):
        self._check(scene)
        first = self._n_samples + 1
        p = self._params(scene)
        rc = self._device.lib.or_render_path(
            scene.handle(), ctypes.byref(p), self._w, self._h, first, int(k),
            self._light_samples, ptr(self._linear), ptr(self._srgb, _bp), ptr(self.m2), None, 0,
            1 if self.nan_guard else 0, self._device.threads, ctypes.byref(self.stats))
        if rc != 0:
            raise RuntimeError("oracle path render failed")
        self._n_samples += int(k)

    def render_pixels(self, scene, pixels, first_sample, n_render, light_samples=None,
                      want_m2=True):
        """Render only ``pixels`` (flat indices j*w+i) for n_render samples starting at sample
        number ``first_sample``; returns (linear[n,4], srgb[n,4], m2[n,3])."""
        self._check(scene)
        pix = numpy.ascontiguousarray(pixels, dtype=numpy.uint32)
        n = pix.shape[0]
        lin = numpy.zeros((n, 4), numpy.float32)
        srgb = numpy.zeros((n, 4), numpy.uint8)
        m2 = numpy.zeros((n, 3), numpy.float32) if want_m2 else None
        p = self._params(scene)
        L = self._light_samples if light_samples is None else int(light_samples)
        rc = self._device.lib.or_render_path(
            scene.handle(), ctypes.byref(p), self._w, self._h, int(first_sample), int(n_render), L,
            ptr(lin), ptr(srgb, _bp), ptr(m2), ptr(pix, _up), n, 1 if self.nan_guard else 0,
            self._device.threads, ctypes.byref(self.stats))
        if rc != 0:
            raise RuntimeError("oracle path render failed")
        return lin, srgb, m2


def make_device(kind="restated"):
    """A fresnel-API Device object whose backend module is this oracle (for tests)."""
    import sys
    mod = sys.modules[__name__]

    class _Dev(Device):
        pass

    _Dev.kind = kind
    api_dev = object.__new__(_device_class())
    api_dev.module = _ModuleView(mod, _Dev)
    api_dev._device = _Dev()
    api_dev._mode = "cpu"
    return api_dev


def _device_class():
    import fresnel_b200
    return fresnel_b200.Device


class _ModuleView:
    """The module's classes, with Device replaced by a subclass bound to one library kind."""

    def __init__(self, mod, dev_cls):
        self._mod = mod
        self.Device = dev_cls

    def __getattr__(self, name):
        return getattr(self._mod, name)


__all__ = ["Device", "Scene", "Geometry", "GeometrySphere", "GeometryCylinder",
           "GeometryConvexPolyhedron", "GeometryMesh", "GeometryPolygon", "Tracer", "TracerDirect",
           "TracerPath", "load", "make_device"]
