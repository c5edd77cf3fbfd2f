"""Cameras (fresnel/camera.py).

A camera wraps a `_common.UserCamera`; scene space and camera space share units.  Camera space
has +x right, +y up and +z out of the screen.
"""

import math

import numpy

from . import _common


def _vec3(value, name):
    if len(value) != 3:
        raise ValueError(f"{name} must have length 3")
    return _common.vec3f(*value)


class Camera:
    """Camera base class (fresnel/camera.py:11-140)."""

    def __init__(self, _camera):
        self._camera = _camera

    def __copy__(self):
        src = self._camera
        cam = _common.UserCamera()
        for name in ("model", "position", "look_at", "up", "h", "f", "f_stop", "focus_distance"):
            setattr(cam, name, getattr(src, name))
        return _from_cpp(cam)

    @staticmethod
    def _as_array(v):
        return numpy.array([v.x, v.y, v.z], dtype=numpy.float32)

    @property
    def position(self):
        """(3,) float32: centre of projection."""
        return self._as_array(self._camera.position)

    @position.setter
    def position(self, value):
        self._camera.position = _vec3(value, "position")

    @property
    def look_at(self):
        """(3,) float32: point at the centre of the image."""
        return self._as_array(self._camera.look_at)

    @look_at.setter
    def look_at(self, value):
        self._camera.look_at = _vec3(value, "look_at")

    @property
    def up(self):
        """(3,) float32: vector toward +y in camera space."""
        return self._as_array(self._camera.up)

    @up.setter
    def up(self, value):
        self._camera.up = _vec3(value, "up")

    @property
    def height(self):
        """float: height of the image plane."""
        return self._camera.h

    @height.setter
    def height(self, value):
        self._camera.h = float(value)

    @property
    def basis(self):
        """(3, 3) float32: rows u, v, w of the orthonormal camera basis."""
        b = _common.CameraBasis(self._camera)
        return numpy.array([(b.u.x, b.u.y, b.u.z), (b.v.x, b.v.y, b.v.z), (b.w.x, b.w.y, b.w.z)],
                           dtype=numpy.float32)


_VIEWS = {
    'front': dict(v=numpy.array([0, 0, 1]), up=numpy.array([0, 1, 0]),
                  right=numpy.array([1, 0, 0])),
    'isometric': dict(v=numpy.array([1, 1, 1]) / math.sqrt(3),
                      up=numpy.array([-1, 2, -1]) / math.sqrt(6),
                      right=numpy.array([1, 0, -1]) / math.sqrt(2)),
}


class Orthographic(Camera):
    """Parallel-projection camera (fresnel/camera.py:143-279)."""

    def __init__(self, position, look_at, up, height):
        cam = _common.UserCamera()
        cam.model = _common.CameraModel.orthographic
        super().__init__(cam)
        self.position = position
        self.look_at = look_at
        self.up = up
        self.height = height

    def __repr__(self):
        return (f"fresnel.camera.Orthographic(position={tuple(self.position)}, "
                f"look_at={tuple(self.look_at)}, up={tuple(self.up)}, height={self.height})")

    @classmethod
    def fit(cls, scene, view='auto', margin=0.05):
        """Orthographic camera that frames the whole scene (fresnel/camera.py:196-279).

        ``view`` is 'auto', 'isometric' or 'front'; 'auto' picks 'front' when the scene is flat
        in z (z extent below 0.51 of the larger of the x and y extents).
        """
        if len(scene.geometry) == 0:
            raise ValueError('The camera cannot be fit because the scene has no geometries. '
                             'Add geometries to the scene before calling fit.')
        ext = scene.get_extents()
        if view == 'auto':
            xw = ext[1, 0] - ext[0, 0]
            yw = ext[1, 1] - ext[0, 1]
            zw = ext[1, 2] - ext[0, 2]
            view = 'front' if zw < 0.51 * max(xw, yw) else 'isometric'
        v = _VIEWS[view]['v']
        up = _VIEWS[view]['up']
        lo, hi = ext[0], ext[1]
        corners = numpy.array([[x, y, z] for x in (lo[0], hi[0]) for y in (lo[1], hi[1])
                               for z in (lo[2], hi[2])])
        center = (ext[0, :] + ext[1, :]) / 2
        corners = corners - center
        height = (1 + margin) * numpy.max(numpy.abs(numpy.dot(corners, up))) * 2
        distance = numpy.max(numpy.dot(corners, v)) * 1.10
        return cls(position=center + distance * v, look_at=center, up=up, height=height)


class Perspective(Camera):
    """Thin-lens perspective camera (fresnel/camera.py:282-560)."""

    def __init__(self, position, look_at, up, focal_length=.5, focus_distance=10, f_stop=math.inf,
                 height=0.24):
        cam = _common.UserCamera()
        cam.model = _common.CameraModel.perspective
        super().__init__(cam)
        self.position = position
        self.look_at = look_at
        self.up = up
        self.focus_distance = focus_distance
        self.focal_length = focal_length
        self.f_stop = f_stop
        self.height = height

    def __repr__(self):
        return (f"fresnel.camera.Perspective(position={tuple(self.position)}, "
                f"look_at={tuple(self.look_at)}, up={tuple(self.up)}, "
                f"focus_distance={self.focus_distance}, focal_length={self.focal_length}, "
                f"f_stop={self.f_stop}, height={self.height})")

    @property
    def focal_length(self):
        """float: focal length of the lens (sets the field of view with `height`)."""
        return self._camera.f

    @focal_length.setter
    def focal_length(self, value):
        self._camera.f = value

    @property
    def f_stop(self):
        """float: aperture in f-stops (``inf``: no depth of field)."""
        return self._camera.f_stop

    @f_stop.setter
    def f_stop(self, value):
        self._camera.f_stop = value

    @property
    def focus_distance(self):
        """float: distance from `position` to the focal plane."""
        return self._camera.focus_distance

    @focus_distance.setter
    def focus_distance(self, value):
        self._camera.focus_distance = value

    @property
    def depth_of_field(self):
        """float: extent of acceptably sharp focus around the focal plane.

        Circle of confusion c = height / 800 (0.03 mm on a 24 mm sensor); hyperfocal distance
        H = f^2 / (N c).  Setting it solves for `f_stop`.
        """
        f = self.focal_length
        N = self.f_stop
        s = self.focus_distance
        c = self.height / 800
        H = f**2 / (N * c)
        if H - (s - f) <= 0 or H + (s - f) <= 0:
            return math.inf
        return s * H * (1 / (H - (s - f)) - 1 / (H + (s - f)))

    @depth_of_field.setter
    def depth_of_field(self, value):
        f = self.focal_length
        d = value
        s = self.focus_distance
        c = self.height / 800
        a = math.sqrt(c**2 * f**4 * (d**2 + s**2) * (f - s)**2)
        b = c * f**2 * s * (f - s)
        self.f_stop = (a + b) / (c**2 * d * (f - s)**2)

    @property
    def focus_on(self):
        """(3,) point on the focal plane along the view direction; setting it moves the plane."""
        d = -self.basis[2, :]
        return self.position + d * self.focus_distance

    @focus_on.setter
    def focus_on(self, value):
        if len(value) != 3:
            raise ValueError("focus_on must have length 3")
        d = -self.basis[2, :]
        self.focus_distance = numpy.dot(d, value - self.position)

    @property
    def vertical_field_of_view(self):
        """float: vertical field of view in radians, 2 atan(height / (2 f))."""
        return 2 * math.atan(self.height / (2 * self.focal_length))

    @vertical_field_of_view.setter
    def vertical_field_of_view(self, value):
        self.focal_length = self.height / (2 * math.tan(value / 2))


def _from_cpp(cam):
    """Wrap a `_common.UserCamera` in the Python class matching its model."""
    if cam.model == _common.CameraModel.orthographic:
        result = Orthographic(position=(0, 0, 0), look_at=(0, 0, 1), up=(0, 1, 0), height=1)
    elif cam.model == _common.CameraModel.perspective:
        result = Perspective(position=(0, 0, 0), look_at=(0, 0, 1), up=(0, 1, 0),
                             focus_distance=1)
    else:
        raise RuntimeError("Invalid camera model")
    result._camera = cam
    return result
