"""Materials: how light interacts with a surface (fresnel/material.py)."""

from . import _common

_SCALARS = ("solid", "primitive_color_mix", "roughness", "specular", "spec_trans", "metal")


class Material:
    """Disney-style material parameters (fresnel/material.py:9-132).

    Args:
        solid (float): 1 to output a flat colour regardless of lighting.
        color: linear RGB base colour.
        primitive_color_mix (float): 0 uses `color`, 1 the geometry's per-primitive colour.
        roughness (float): nominally 0.1 to 1.
        specular (float): strength of specular highlights, 0 to 1.
        spec_trans (float): fraction of specular transmission, 0 to 1.
        metal (float): 0 dielectric, 1 metal.
    """

    def __init__(self, solid=0, color=(0.9, 0.9, 0.9), primitive_color_mix=0, roughness=0.3,
                 specular=0.5, spec_trans=0, metal=0):
        self._material = _common.Material()
        self.solid = solid
        self.color = color
        self.roughness = roughness
        self.specular = specular
        self.metal = metal
        self.spec_trans = spec_trans
        self.primitive_color_mix = primitive_color_mix

    def _get_cpp_material(self):
        return self._material


def _direct_scalar(name):
    def get(self):
        return getattr(self._material, name)

    def set(self, value):
        setattr(self._material, name, float(value))

    return property(get, set)


def _direct_color():
    def get(self):
        c = self._material.color
        return (c.r, c.g, c.b)

    def set(self, value):
        if len(value) != 3:
            raise ValueError("colors must have length 3")
        self._material.color = _common.RGBf(*value)

    return property(get, set)


for _name in _SCALARS:
    setattr(Material, _name, _direct_scalar(_name))
Material.color = _direct_color()


class _GeometryMaterialProxy:
    """Reads and writes a material held by a geometry; every write goes back to the backend
    (fresnel/material.py:135-332)."""

    _getter = "getMaterial"
    _setter = "setMaterial"

    def __init__(self, geometry):
        self._geometry = geometry._geometry

    def _get_cpp_material(self):
        return getattr(self._geometry, self._getter)()

    def _update(self, fn):
        m = getattr(self._geometry, self._getter)()
        fn(m)
        getattr(self._geometry, self._setter)(m)


def _proxy_scalar(name):
    def get(self):
        return getattr(self._get_cpp_material(), name)

    def set(self, value):
        self._update(lambda m: setattr(m, name, float(value)))

    return property(get, set)


def _proxy_color():
    def get(self):
        c = self._get_cpp_material().color
        return (c.r, c.g, c.b)

    def set(self, value):
        if len(value) != 3:
            raise ValueError("colors must have length 3")
        self._update(lambda m: setattr(m, "color", _common.RGBf(*value)))

    return property(get, set)


for _name in _SCALARS:
    setattr(_GeometryMaterialProxy, _name, _proxy_scalar(_name))
_GeometryMaterialProxy.color = _proxy_color()


class _MaterialProxy(_GeometryMaterialProxy):
    """Proxy for `Geometry.material`."""


class _OutlineMaterialProxy(_GeometryMaterialProxy):
    """Proxy for `Geometry.outline_material`."""

    _getter = "getOutlineMaterial"
    _setter = "setOutlineMaterial"
