// host_types.hpp -- value types shared by the `_common` and `_gpu` Python extension modules.
//
// They mirror the plain structs fresnel exposes through its `_common` module
// (fresnel/common/module-common.cc:37-115): RGBf, vec3f, Material, UserCamera, CameraModel,
// CameraBasis and Lights.  Both extension modules are built from the same definitions so that
// pybind11 sees one C++ type per Python class.  Conversions to the C-ABI structs are exact
// field copies.
#ifndef FR_HOST_TYPES_HPP
#define FR_HOST_TYPES_HPP

#include <cmath>
#include <cstdint>

#include "../../include/fresnel_b200.h"

namespace frh {

struct vec3f {
    float x = 0, y = 0, z = 0;
    vec3f() = default;
    vec3f(float a, float b, float c) : x(a), y(b), z(c) {}
};

struct RGBf {
    float r = 0, g = 0, b = 0;
    RGBf() = default;
    RGBf(float a, float b_, float c) : r(a), g(b_), b(c) {}
};

enum class CameraModel : int32_t { orthographic = FR_CAMERA_ORTHOGRAPHIC, perspective = FR_CAMERA_PERSPECTIVE };

// UserCamera defaults (fresnel/common/Camera.h:57-68).
struct UserCamera {
    vec3f position{0, 0, 0};
    vec3f look_at{0, 0, 1};
    vec3f up{0, 1, 0};
    float h = 1, f = 1, f_stop = 1, focus_distance = 1;
    CameraModel model = CameraModel::orthographic;
};

// Material: the reference's default constructor leaves fields uninitialised; the Python layer
// always assigns every field, so zero defaults are an equivalent, deterministic choice.
struct Material {
    float solid = 0;
    RGBf color{0, 0, 0};
    float primitive_color_mix = 0, roughness = 0, specular = 0, metal = 0, spec_trans = 0;
};

struct Lights {
    vec3f direction[4];
    RGBf color[4];
    float theta[4] = {0, 0, 0, 0};
    unsigned int N = 0;
};

inline fr_user_camera to_abi(const UserCamera& c)
{
    fr_user_camera o;
    o.position[0] = c.position.x;
    o.position[1] = c.position.y;
    o.position[2] = c.position.z;
    o.look_at[0] = c.look_at.x;
    o.look_at[1] = c.look_at.y;
    o.look_at[2] = c.look_at.z;
    o.up[0] = c.up.x;
    o.up[1] = c.up.y;
    o.up[2] = c.up.z;
    o.h = c.h;
    o.f = c.f;
    o.f_stop = c.f_stop;
    o.focus_distance = c.focus_distance;
    o.model = int32_t(c.model);
    return o;
}

inline fr_material to_abi(const Material& m)
{
    fr_material o;
    o.solid = m.solid;
    o.color[0] = m.color.r;
    o.color[1] = m.color.g;
    o.color[2] = m.color.b;
    o.primitive_color_mix = m.primitive_color_mix;
    o.roughness = m.roughness;
    o.specular = m.specular;
    o.metal = m.metal;
    o.spec_trans = m.spec_trans;
    return o;
}

inline fr_lights to_abi(const Lights& l)
{
    fr_lights o;
    for (int i = 0; i < 4; ++i) {
        o.direction[i][0] = l.direction[i].x;
        o.direction[i][1] = l.direction[i].y;
        o.direction[i][2] = l.direction[i].z;
        o.color[i][0] = l.color[i].r;
        o.color[i][1] = l.color[i].g;
        o.color[i][2] = l.color[i].b;
        o.theta[i] = l.theta[i];
    }
    o.n = l.N > 4 ? 4 : l.N;
    return o;
}

// CameraBasis (fresnel/common/Camera.h:89-113): orthonormal u (right), v (up), w (backward).
// Evaluated with the same operation order as the device code in frmath.cuh.
struct CameraBasis {
    vec3f u, v, w;
    CameraBasis() = default;
    explicit CameraBasis(const UserCamera& c)
    {
        auto dot = [](vec3f a, vec3f b) { return a.x * b.x + a.y * b.y + a.z * b.z; };
        auto cross = [](vec3f a, vec3f b) {
            return vec3f(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
        };
        auto scale = [](vec3f a, float s) { return vec3f(a.x * s, a.y * s, a.z * s); };
        vec3f d(c.look_at.x - c.position.x, c.look_at.y - c.position.y, c.look_at.z - c.position.z);
        d = scale(d, 1.0f / std::sqrt(dot(d, d)));
        vec3f vv = scale(c.up, 1.0f / std::sqrt(dot(c.up, c.up)));
        vec3f uu = cross(d, vv);
        uu = scale(uu, 1.0f / std::sqrt(dot(uu, uu)));
        vv = cross(uu, d);
        vv = scale(vv, 1.0f / std::sqrt(dot(vv, vv)));
        u = uu;
        v = vv;
        w = vec3f(-d.x, -d.y, -d.z);
    }
};

}  // namespace frh

#endif
