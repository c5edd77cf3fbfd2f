"""Directional area lights and lighting presets (fresnel/light.py).

Lights point *toward* the light in camera space; at most 4 lights per scene.
"""

import math

from . import _common


class Light:
    """One area light at infinity (fresnel/light.py:14-49).

    Args:
        direction: vector toward the light, camera space.
        color: linear RGB intensity.
        theta (float): half angle of the light's cone, radians.
    """

    def __init__(self, direction, color=(1, 1, 1), theta=0.375):
        self.direction = tuple(direction)
        self.color = tuple(color)
        self.theta = float(theta)

    def __str__(self):
        return f"<Light object with direction {self.direction} and color {self.color}>"


class _LightProxy:
    """View of one entry of a scene's light list (fresnel/light.py:52-91)."""

    def __init__(self, light_list, idx):
        self._light_list = light_list
        self._idx = idx

    @property
    def direction(self):
        v = self._light_list._lights.getDirection(self._idx)
        return (v.x, v.y, v.z)

    @direction.setter
    def direction(self, v):
        self._light_list._lights.setDirection(self._idx, _common.vec3f(*v))

    @property
    def color(self):
        c = self._light_list._lights.getColor(self._idx)
        return (c.r, c.g, c.b)

    @color.setter
    def color(self, v):
        self._light_list._lights.setColor(self._idx, _common.RGBf(*v))

    @property
    def theta(self):
        return self._light_list._lights.getTheta(self._idx)

    @theta.setter
    def theta(self, v):
        self._light_list._lights.setTheta(self._idx, v)

    def __str__(self):
        return f"<Light proxy object with direction {self.direction} and color {self.color}>"


class _LightListProxy:
    """List-like access to a `_common.Lights` (fresnel/light.py:94-131)."""

    def __init__(self, _lights=None):
        if _lights is None:
            _lights = _common.Lights()
            _lights.N = 0
        self._lights = _lights

    def __len__(self):
        return self._lights.N

    def clear(self):
        self._lights.N = 0

    def append(self, light):
        if len(self) >= 4:
            raise IndexError("Cannot add more than 4 lights")
        i = self._lights.N
        self._lights.setDirection(i, _common.vec3f(*light.direction))
        self._lights.setColor(i, _common.RGBf(*light.color))
        self._lights.setTheta(i, light.theta)
        self._lights.N = i + 1

    def __getitem__(self, idx):
        if idx >= self._lights.N:
            raise IndexError("Indexing past the end of the list")
        return _LightProxy(self, idx)


def _spherical(theta_deg, phi_deg):
    """Unit vector with polar angle theta from +y and azimuth phi from +z toward +x."""
    th = theta_deg * math.pi / 180
    ph = phi_deg * math.pi / 180
    return (math.sin(th) * math.sin(ph), math.cos(th), math.sin(th) * math.cos(ph))


def butterfly():
    """Key light high above the camera, fill below (fresnel/light.py:134-159)."""
    t1 = 50 * math.pi / 180
    t2 = -30 * math.pi / 180
    return [Light(direction=(0, math.sin(t1), math.cos(t1)), color=(1.0, 1.0, 1.0),
                  theta=math.pi / 4),
            Light(direction=(0, math.sin(t2), math.cos(t2)), color=(0.1, 0.1, 0.1),
                  theta=math.pi / 2)]


def loop(side='right'):
    """Key light slightly to one side and up, fill level on the other (fresnel/light.py:162-196)."""
    sign = {'right': 1, 'left': -1}[side]
    return [Light(direction=_spherical(90 - 20, sign * 25), color=(1.0, 1.0, 1.0),
                  theta=math.pi / 4),
            Light(direction=_spherical(90, -sign * 40), color=(0.1, 0.1, 0.1),
                  theta=math.pi / 2)]


def rembrandt(side='right'):
    """Key light 45 degrees to one side and up, fill on the other (fresnel/light.py:199-233)."""
    sign = {'right': 1, 'left': -1}[side]
    return [Light(direction=_spherical(90 - 20, sign * 45), color=(1.0, 1.0, 1.0),
                  theta=math.pi / 4),
            Light(direction=_spherical(90, -sign * 45), color=(0.1, 0.1, 0.1),
                  theta=math.pi / 2)]


def lightbox():
    """One light covering the whole sphere of directions (fresnel/light.py:236-248)."""
    return [Light(direction=(0, 0, 1), color=(0.9, 0.9, 0.9), theta=math.pi)]


def cloudy():
    """Bright sky above, dim ground bounce below (fresnel/light.py:251-267)."""
    return [Light(direction=(0, 1, 0), color=(0.9, 0.9, 0.9), theta=math.pi / 2),
            Light(direction=(0, -1, 0), color=(0.1, 0.1, 0.1), theta=math.pi / 2)]


def ring():
    """Strong front light (fresnel/light.py)."""
    return [Light(direction=(0, 0, 1), color=(0.9, 0.9, 0.9), theta=math.pi / 4)]
