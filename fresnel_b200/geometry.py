"""Geometric primitives (fresnel/geometry.py).

Each class owns a backend geometry object; its per-primitive arrays are exposed as
`util.Array` views, and writing to them marks the geometry's BVH stale.
"""

import numpy

from . import material as _material_mod
from . import util


def _default_outline():
    return _material_mod.Material(solid=1, color=(0, 0, 0))


class Geometry:
    """Common geometry operations (fresnel/geometry.py:21-96)."""

    def __init__(self):
        raise RuntimeError("Use a specific geometry class")

    def _setup(self, scene, material, outline_material, outline_width):
        self.material = _material_mod.Material() if material is None else material
        self.outline_material = (_default_outline()
                                 if outline_material is None else outline_material)
        self.outline_width = outline_width

    def _attach(self, scene):
        self.scene = scene
        scene.geometry.append(self)

    def enable(self):
        """Make the geometry visible."""
        self._geometry.enable()

    def disable(self):
        """Hide the geometry (reversible)."""
        self._geometry.disable()

    def remove(self):
        """Remove the geometry from its scene for good."""
        self._geometry.remove()
        self.scene.geometry.remove(self)

    @property
    def material(self):
        return _material_mod._MaterialProxy(self)

    @material.setter
    def material(self, mat):
        self._geometry.setMaterial(mat._get_cpp_material())

    @property
    def outline_material(self):
        return _material_mod._OutlineMaterialProxy(self)

    @outline_material.setter
    def outline_material(self, mat):
        self._geometry.setOutlineMaterial(mat._get_cpp_material())

    @property
    def outline_width(self):
        return self._geometry.getOutlineWidth()

    @outline_width.setter
    def outline_width(self, width):
        self._geometry.setOutlineWidth(width)

    def _array(self, buf):
        return util.Array(buf, geom=self)


class Cylinder(Geometry):
    """Spherocylinders between start and end points (fresnel/geometry.py:99-207).

    Args: scene, points (N, 2, 3), radius (N,), color (N, 2, 3), N, material,
    outline_material, outline_width.
    """

    def __init__(self, scene, points=((0, 0, 0), (0, 0, 0)), radius=0.5, color=(0, 0, 0), N=None,
                 material=None, outline_material=None, outline_width=0.0):
        if N is None:
            N = len(points)
        self._geometry = scene.device.module.GeometryCylinder(scene._scene, N)
        self._setup(scene, material, outline_material, outline_width)
        self.points[:] = points
        self.radius[:] = radius
        self.color[:] = color
        self._attach(scene)

    def get_extents(self):
        A = self.points[:, 0]
        B = self.points[:, 1]
        r = self.radius[:]
        r = r.reshape(len(r), 1)
        return numpy.array([
            numpy.min([numpy.min(A - r, axis=0), numpy.min(B - r, axis=0)], axis=0),
            numpy.max([numpy.max(A + r, axis=0), numpy.max(B + r, axis=0)], axis=0)])

    @property
    def points(self):
        return self._array(self._geometry.getPointsBuffer())

    @property
    def radius(self):
        return self._array(self._geometry.getRadiusBuffer())

    @property
    def color(self):
        return self._array(self._geometry.getColorBuffer())


class Box(Cylinder):
    """Outline of a (triclinic) box drawn with 12 spherocylinders (fresnel/geometry.py:210-388).

    ``box`` may be a number, a length 1/3/6 sequence ``[Lx, Ly, Lz, xy, xz, yz]``, a mapping
    with those keys, or an object with those attributes (HOOMD/GSD convention).
    """

    def __init__(self, scene, box, box_radius=0.5, box_color=(0, 0, 0)):
        super().__init__(scene=scene, N=12, material=_material_mod.Material(solid=1.0))
        self._box = self._from_box(box)
        self.points[:] = self._generate_points(self._box)
        self.box_radius = box_radius
        self.box_color = box_color

    @staticmethod
    def _from_box(box):
        try:
            Lx, Ly = box.Lx, box.Ly
            Lz = getattr(box, 'Lz', 0)
            xy, xz, yz = (getattr(box, k, 0) for k in ('xy', 'xz', 'yz'))
        except AttributeError:
            try:
                Lx, Ly = box['Lx'], box['Ly']
                Lz = box.get('Lz', 0)
                xy, xz, yz = (box.get(k, 0) for k in ('xy', 'xz', 'yz'))
            except (IndexError, KeyError, TypeError):
                try:
                    if len(box) not in (1, 3, 6):
                        raise ValueError("List-like objects must have length 1, 3, or 6 to be "
                                         "converted to a box.")
                    Lx = box[0]
                    Ly = box[0] if len(box) == 1 else box[1]
                    Lz = box[0] if len(box) == 1 else box[2]
                    xy, xz, yz = box[3:6] if len(box) == 6 else (0, 0, 0)
                except TypeError:
                    if isinstance(box, (int, float)):
                        Lx = Ly = Lz = box
                        xy = xz = yz = 0
                    else:
                        raise TypeError(f"unsupported box type {type(box)}")
        return (Lx, Ly, Lz, xy, xz, yz)

    @staticmethod
    def _generate_points(box):
        Lx, Ly, Lz, xy, xz, yz = box
        m = numpy.array([[Lx, xy * Ly, xz * Lz], [0, Ly, yz * Lz], [0, 0, Lz]])
        a1, a2, a3 = m.T
        A = -(a1 + a2 + a3) / 2
        B, C, D = A + a1, A + a2, A + a3
        E, F, G = A + a1 + a3, A + a2 + a3, A + a1 + a2
        H = A + a1 + a2 + a3
        return numpy.asarray([[A, B], [A, C], [A, D], [B, E], [B, G], [C, G], [C, F], [D, E],
                              [D, F], [E, H], [F, H], [G, H]])

    @property
    def box(self):
        return self._box

    @box.setter
    def box(self, box):
        self._box = self._from_box(box)
        self.points[:] = self._generate_points(self._box)

    @property
    def box_color(self):
        return self.material.color

    @box_color.setter
    def box_color(self, color):
        self.material.color = color

    @property
    def box_radius(self):
        return self.radius[:][0]

    @box_radius.setter
    def box_radius(self, radius):
        self.radius[:] = radius


class Polygon(Geometry):
    """Simple polygons in the xy plane with per-primitive 2-D position, rotation angle and
    colour, rounded by ``rounding_radius`` (fresnel/geometry.py:391-501).

    ``vertices`` (N_vert, 2) lists one polygon's outline counter-clockwise (concave shapes are
    allowed); every primitive is that polygon placed at its position and rotated about z by its
    angle.  Polygons are double sided.
    """

    def __init__(self, scene, vertices, position=(0, 0), angle=0, color=(0, 0, 0),
                 rounding_radius=0, N=None, material=None, outline_material=None,
                 outline_width=0.0):
        if N is None:
            N = len(position)
        self._geometry = scene.device.module.GeometryPolygon(scene._scene, vertices,
                                                             rounding_radius, N)
        self._setup(scene, material, outline_material, outline_width)
        self.position[:] = position
        self.angle[:] = angle
        self.color[:] = color
        self._attach(scene)

    @property
    def position(self):
        """(N, 2) `util.Array`: the position of each polygon."""
        return self._array(self._geometry.getPositionBuffer())

    @property
    def angle(self):
        """(N, ) `util.Array`: the rotation angle of each polygon (radians)."""
        return self._array(self._geometry.getAngleBuffer())

    @property
    def color(self):
        """(N, 3) `util.Array`: the colour of each polygon."""
        return self._array(self._geometry.getColorBuffer())

    def get_extents(self):
        """Lower and upper corners, shape (2, 3): the polygons' bounding squares, 1e-5 thick in z
        (fresnel/geometry.py:487-501)."""
        pos = self.position[:]
        r = self._geometry.getRadius()
        res2d = numpy.array([numpy.min(pos - r, axis=0), numpy.max(pos + r, axis=0)])
        return numpy.array([[res2d[0][0], res2d[0][1], -1e-5],
                            [res2d[1][0], res2d[1][1], 1e-5]])


class Sphere(Geometry):
    """Spheres with per-primitive position, radius and colour (fresnel/geometry.py:504-610)."""

    def __init__(self, scene, position=(0, 0, 0), radius=0.5, color=(0, 0, 0), N=None,
                 material=None, outline_material=None, outline_width=0.0):
        if N is None:
            N = len(position)
        self._geometry = scene.device.module.GeometrySphere(scene._scene, N)
        self._setup(scene, material, outline_material, outline_width)
        self.position[:] = position
        self.radius[:] = radius
        self.color[:] = color
        self._attach(scene)

    def get_extents(self):
        pos = self.position[:]
        r = self.radius[:]
        r = r.reshape(len(r), 1)
        return numpy.array([numpy.min(pos - r, axis=0), numpy.max(pos + r, axis=0)])

    @property
    def position(self):
        return self._array(self._geometry.getPositionBuffer())

    @property
    def radius(self):
        return self._array(self._geometry.getRadiusBuffer())

    @property
    def color(self):
        return self._array(self._geometry.getColorBuffer())


class Mesh(Geometry):
    """Instanced triangle meshes (fresnel/geometry.py:613-738).

    ``vertices`` (3T, 3) lists triangles contiguously (counter-clockwise seen from outside);
    ``color`` is per vertex of the shared prototype; position/orientation are per instance.
    """

    def __init__(self, scene, vertices, position=(0, 0, 0), orientation=(1, 0, 0, 0),
                 color=(0, 0, 0), N=None, material=None, outline_material=None,
                 outline_width=0.0):
        if N is None:
            N = len(position)
        self.vertices = numpy.asarray(vertices, dtype=numpy.float32)
        self._geometry = scene.device.module.GeometryMesh(scene._scene, self.vertices, N)
        self._setup(scene, material, outline_material, outline_width)
        self.position[:] = position
        self.orientation[:] = orientation
        self.color[:] = color
        self._attach(scene)

    @property
    def position(self):
        return self._array(self._geometry.getPositionBuffer())

    @property
    def orientation(self):
        return self._array(self._geometry.getOrientationBuffer())

    @property
    def color(self):
        return self._array(self._geometry.getColorBuffer())

    def get_extents(self):
        a = self.vertices[:, 0]
        b = self.vertices[:, 1]
        c = self.vertices[:, 2]
        r = numpy.array([
            numpy.min([numpy.min(a, axis=0), numpy.min(b, axis=0), numpy.min(c, axis=0)], axis=0),
            numpy.max([numpy.max(a, axis=0), numpy.max(b, axis=0), numpy.max(c, axis=0)], axis=0)])
        pos = self.position[:]
        return numpy.array([numpy.min(pos + r[0], axis=0), numpy.max(pos + r[1], axis=0)])


class ConvexPolyhedron(Geometry):
    """Convex polyhedra given by outward face planes (fresnel/geometry.py:741-873).

    ``polyhedron_info`` holds ``face_origin``, ``face_normal``, ``face_color`` and ``radius``
    (see `util.convex_polyhedron_from_vertices`).
    """

    def __init__(self, scene, polyhedron_info, position=(0, 0, 0), orientation=(1, 0, 0, 0),
                 color=(0, 0, 0), N=None, material=None, outline_material=None,
                 outline_width=0.0):
        if N is None:
            N = len(position)
        r = polyhedron_info['radius']
        self._geometry = scene.device.module.GeometryConvexPolyhedron(
            scene._scene, polyhedron_info['face_origin'], polyhedron_info['face_normal'],
            polyhedron_info['face_color'], N, r)
        self._setup(scene, material, outline_material, outline_width)
        self._radius = r
        self.position[:] = position
        self.orientation[:] = orientation
        self.color[:] = color
        self._attach(scene)

    def get_extents(self):
        pos = self.position[:]
        r = self._radius
        return numpy.array([numpy.min(pos - r, axis=0), numpy.max(pos + r, axis=0)])

    @property
    def position(self):
        return self._array(self._geometry.getPositionBuffer())

    @property
    def orientation(self):
        return self._array(self._geometry.getOrientationBuffer())

    @property
    def color(self):
        return self._array(self._geometry.getColorBuffer())

    @property
    def color_by_face(self):
        """float: 0 colours by the per-polyhedron colour, 1 by the per-face colour."""
        return self._geometry.getColorByFace()

    @color_by_face.setter
    def color_by_face(self, v):
        self._geometry.setColorByFace(v)
