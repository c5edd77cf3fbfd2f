"""fresnel_b200: a B200 (sm_100a) ray tracing engine with fresnel's Python API.

``import fresnel_b200 as fresnel`` gives the classes and functions of the ``fresnel`` package
(``Device``, ``Scene``, ``preview``, ``pathtrace`` and the ``geometry``, ``tracer``, ``camera``,
``light``, ``material``, ``color`` and ``util`` modules) on top of native CUDA kernels.  The
only backend is the GPU one: there is no CPU fallback, and importing the package fails if the
compiled extension modules are missing.

Reference: fresnel/__init__.py (Device :23-127, Scene :149-281, preview :284-296,
pathtrace :299-315).
"""

import os

import numpy

from . import _common
from . import _gpu
from . import camera
from . import color  # noqa: F401
from . import geometry  # noqa: F401
from . import light
from . import material  # noqa: F401
from . import tracer
from . import util  # noqa: F401
from . import version  # noqa: F401

__all__ = ["Device", "Scene", "preview", "pathtrace", "camera", "color", "geometry", "light",
           "material", "tracer", "util", "version"]


class Device:
    """Hardware device used for ray tracing (fresnel/__init__.py:23-127).

    Args:
        mode (str): ``'auto'`` or ``'gpu'``.  ``'cpu'`` raises ``RuntimeError`` because this
            build has no CPU implementation.
        n (int): number of GPUs to use (``None``: all).  Rendering runs on the first one.
    """

    available_modes = []
    available_gpus = []

    def __init__(self, mode='auto', n=None):
        num_gpus = _gpu.get_num_available_devices()
        if mode == 'auto':
            if num_gpus == 0:
                raise RuntimeError("No GPUs available AND CPU implementation is not compiled")
            selected = 'gpu'
        elif mode == 'gpu':
            if num_gpus == 0:
                raise RuntimeError("No GPUs are available")
            selected = 'gpu'
        elif mode == 'cpu':
            raise RuntimeError("CPU implementation is not compiled")
        else:
            raise ValueError("Invalid mode")
        limit = -1 if n is None else int(n)
        self.module = _gpu
        self._device = _gpu.Device(os.path.dirname(os.path.realpath(__file__)), limit)
        self._mode = selected

    @property
    def mode(self):
        """str: the active mode."""
        return self._mode

    def __str__(self):
        return '<fresnel.Device: ' + self._device.describe() + '>'


def _probe_devices():
    if _gpu.get_num_available_devices() > 0:
        Device.available_modes.extend(['gpu', 'auto'])
    lines = _gpu.Device.getAllGPUs().split('\n')
    if len(lines) >= 2:
        Device.available_gpus = lines[:-1]


_probe_devices()


class Scene:
    """Geometry, camera, lights and background to ray trace (fresnel/__init__.py:149-281)."""

    def __init__(self, device=None, camera=None, lights=None):
        if device is None:
            device = Device()
        self._device = device
        self._scene = device.module.Scene(device._device)
        self.geometry = []
        if camera is None:
            camera = globals()['camera'].Orthographic(position=(0, 0, 100), look_at=(0, 0, 0),
                                                      up=(0, 1, 0), height=100)
        self.camera = camera
        self.lights = light.rembrandt() if lights is None else lights
        self._tracer = None

    def get_extents(self):
        """(2, 3) array: lower and upper corners of the union of the geometries' extents."""
        if not self.geometry:
            return numpy.array([[0, 0, 0], [0, 0, 0]], dtype=numpy.float32)
        ext = self.geometry[0].get_extents()
        for g in self.geometry[1:]:
            e = g.get_extents()
            ext[0, :] = numpy.min([ext[0, :], e[0, :]], axis=0)
            ext[1, :] = numpy.max([ext[1, :], e[1, :]], axis=0)
        return ext

    @property
    def device(self):
        return self._device

    @property
    def camera(self):
        return camera._from_cpp(self._scene.getCamera())

    @camera.setter
    def camera(self, value):
        if not isinstance(value, camera.Camera):
            raise TypeError(f"camera {value} is not a fresnel.camera.Camera")
        self._scene.setCamera(value._camera)

    @property
    def background_color(self):
        c = self._scene.getBackgroundColor()
        return numpy.array([c.r, c.g, c.b], dtype=numpy.float32)

    @background_color.setter
    def background_color(self, value):
        self._scene.setBackgroundColor(_common.RGBf(*value))

    @property
    def background_alpha(self):
        return self._scene.getBackgroundAlpha()

    @background_alpha.setter
    def background_alpha(self, value):
        self._scene.setBackgroundAlpha(value)

    @property
    def lights(self):
        return light._LightListProxy(self._scene.getLights())

    @lights.setter
    def lights(self, values):
        proxy = light._LightListProxy()
        for v in values:
            proxy.append(v)
        self._scene.setLights(proxy._lights)


def preview(scene, w=600, h=370, anti_alias=True):
    """Render with `tracer.Preview` (fresnel/__init__.py:284-296)."""
    return tracer.Preview(scene.device, w=w, h=h, anti_alias=anti_alias).render(scene)


def pathtrace(scene, w=600, h=370, samples=64, light_samples=1):
    """Render with `tracer.Path` (fresnel/__init__.py:299-315)."""
    t = tracer.Path(scene.device, w=w, h=h)
    t.sample(scene, samples=samples, light_samples=light_samples)
    return t.output
