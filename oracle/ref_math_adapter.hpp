// ref_math_adapter.hpp -- TEST INFRASTRUCTURE (oracle/_ref build only).
//
// Routes the oracle core's math calls to the reference's own header-only code
// (fresnel/common/{Camera,RayGen,Material,Light,TracerPathMethods,Intersect*,ColorMath,
// VectorMath}.h), compiled unmodified from the reference tree.  Building the oracle core once
// with this adapter and once with restated_math.hpp, then comparing their outputs, pins the
// restatement to the reference arithmetic.  The adapter converts between the oracle's plain
// structs and the reference types field by field (exact copies of floats).
#ifndef FR_ORACLE_REF_MATH_ADAPTER_HPP
#define FR_ORACLE_REF_MATH_ADAPTER_HPP

#include "restated_math.hpp"

#include "common/Camera.h"
#include "common/ColorMath.h"
#include "common/GeometryMath.h"
#include "common/IntersectCylinder.h"
#include "common/IntersectSphere.h"
#include "common/IntersectTriangle.h"
#include "common/Light.h"
#include "common/Material.h"
#include "common/RayGen.h"
#include "common/TracerPathMethods.h"
#include "common/VectorMath.h"

namespace frref {

using frm::Basis;
using frm::CameraIn;
using frm::F3;
using frm::LightsW;
using frm::Mat;
using frm::PathState;
using frm::Quat;
using frm::RGB3;

inline fresnel::vec3<float> V(F3 a) { return fresnel::vec3<float>(a.x, a.y, a.z); }
inline F3 V(const fresnel::vec3<float>& a) { return F3{a.x, a.y, a.z}; }
inline fresnel::RGB<float> C(RGB3 a) { return fresnel::RGB<float>(a.r, a.g, a.b); }
inline RGB3 C(const fresnel::RGB<float>& a) { return RGB3{a.r, a.g, a.b}; }
inline fresnel::quat<float> Q(Quat q) { return fresnel::quat<float>(q.s, V(q.v)); }
inline Quat Q(const fresnel::quat<float>& q) { return Quat{q.s, V(q.v)}; }

inline fresnel::Material to_ref_mat(const Mat& m)
{
    fresnel::Material r;
    r.solid = m.solid;
    r.color = C(m.color);
    r.primitive_color_mix = m.primitive_color_mix;
    r.roughness = m.roughness;
    r.specular = m.specular;
    r.metal = m.metal;
    r.spec_trans = m.spec_trans;
    return r;
}

struct Cam {
    fresnel::Camera cam;
    Basis basis;
    unsigned width, height, seed;
};

inline fresnel::UserCamera user_camera(const CameraIn& c)
{
    fresnel::UserCamera u;
    u.position = V(c.position);
    u.look_at = V(c.look_at);
    u.up = V(c.up);
    u.h = c.h;
    u.f = c.f;
    u.f_stop = c.f_stop;
    u.focus_distance = c.focus_distance;
    u.model = (c.model == 0) ? fresnel::CameraModel::orthographic : fresnel::CameraModel::perspective;
    return u;
}

inline Basis make_basis(const CameraIn& c)
{
    fresnel::CameraBasis b(user_camera(c));
    return Basis{V(b.u), V(b.v), V(b.w)};
}

inline Cam make_camera(const CameraIn& c, unsigned width, unsigned height, unsigned seed,
                       bool sample_aa)
{
    Cam k;
    k.cam = fresnel::Camera(user_camera(c), width, height, seed, sample_aa);
    const fresnel::CameraBasis& b = k.cam.getBasis();
    k.basis = Basis{V(b.u), V(b.v), V(b.w)};
    k.width = width;
    k.height = height;
    k.seed = seed;
    return k;
}

inline void camera_ray(const Cam& k, unsigned i, unsigned j, unsigned sample, F3& o, F3& d)
{
    fresnel::vec3<float> org, dir;
    k.cam.generateRay(org, dir, i, j, sample);
    o = V(org);
    d = V(dir);
}

inline LightsW lights_to_world(const F3* dir_cam, const RGB3* color, const float* theta, unsigned n,
                               const Cam& k)
{
    fresnel::Lights in;
    in.N = n;
    for (unsigned i = 0; i < n; ++i) {
        in.direction[i] = V(dir_cam[i]);
        in.color[i] = C(color[i]);
        in.theta[i] = theta[i];
    }
    fresnel::Lights w(in, k.cam);
    LightsW out;
    out.n = w.N;
    for (unsigned i = 0; i < w.N; ++i) {
        out.dir[i] = V(w.direction[i]);
        out.color[i] = C(w.color[i]);
        out.theta[i] = w.theta[i];
    }
    return out;
}

inline fresnel::PRDpath to_prd(const PathState& s)
{
    fresnel::PRDpath p;
    p.result = C(s.result);
    p.a = s.a;
    p.attenuation = C(s.att);
    p.origin = V(s.origin);
    p.direction = V(s.dir);
    p.light_sample = s.light_sample;
    p.depth = s.depth;
    p.done = s.done;
    return p;
}
inline void from_prd(PathState& s, const fresnel::PRDpath& p)
{
    s.result = C(p.result);
    s.a = p.a;
    s.att = C(p.attenuation);
    s.origin = V(p.origin);
    s.dir = V(p.direction);
    s.light_sample = p.light_sample;
    s.depth = p.depth;
    s.done = p.done;
}

inline fresnel::Lights to_lights(const LightsW& L)
{
    fresnel::Lights r;
    r.N = L.n;
    for (unsigned i = 0; i < L.n; ++i) {
        r.direction[i] = V(L.dir[i]);
        r.color[i] = C(L.color[i]);
        r.theta[i] = L.theta[i];
    }
    return r;
}

inline void path_miss(PathState& s, RGB3 bg, float bg_alpha, unsigned light_samples,
                      const LightsW& L, F3 ray_dir)
{
    fresnel::PRDpath p = to_prd(s);
    fresnel::path_tracer_miss(p, C(bg), bg_alpha, light_samples, to_lights(L), V(ray_dir));
    from_prd(s, p);
}

// The reference's RayGen keys Philox with {j*width+i, seed}; (pixel, 0, width=1) gives the same key.
inline void path_hit(PathState& s, const Mat& material, const Mat& outline, float shading_distance,
                     float outline_width, RGB3 shading_color, F3 shading_normal, F3 ray_o,
                     F3 ray_d, float t_hit, unsigned key0, unsigned key1, unsigned n_samples,
                     unsigned light_samples)
{
    fresnel::PRDpath p = to_prd(s);
    fresnel::RayGen rg(key0, 0, 1, 1, key1);
    fresnel::path_tracer_hit(p, to_ref_mat(material), to_ref_mat(outline), shading_distance, outline_width,
                             C(shading_color), V(shading_normal), V(ray_o), V(ray_d), t_hit, rg,
                             n_samples, light_samples);
    from_prd(s, p);
}

inline bool is_solid(const Mat& m) { return to_ref_mat(m).isSolid(); }
inline RGB3 base_color(const Mat& m, RGB3 sc) { return C(to_ref_mat(m).getColor(C(sc))); }

inline RGB3 brdf_diffuse(const Mat& m, F3 l, F3 v, F3 n, RGB3 sc)
{
    return C(to_ref_mat(m).brdf_diffuse(V(l), V(v), V(n), C(sc)));
}
inline RGB3 brdf_specular(const Mat& m, F3 l, F3 v, F3 n, RGB3 sc, float half_angle)
{
    return C(to_ref_mat(m).brdf_specular(V(l), V(v), V(n), C(sc), half_angle));
}

inline RGB3 brdf(const Mat& m, F3 l, F3 v, F3 n, RGB3 sc)
{
    return C(to_ref_mat(m).brdf(V(l), V(v), V(n), C(sc)));
}

inline F3 mis_direction(float& factor, bool& transmit, F3 v, F3 n, unsigned depth, unsigned sample,
                        unsigned key0, unsigned key1, const Mat& m)
{
    fresnel::RayGen rg(key0, 0, 1, 1, key1);
    return V(rg.MISReflectionTransmission(factor, transmit, V(v), V(n), depth, sample,
                                          to_ref_mat(m)));
}

inline Quat conj(Quat q) { return Q(fresnel::conj(Q(q))); }
inline F3 rotate(Quat a, F3 b) { return V(fresnel::rotate(Q(a), V(b))); }
inline Quat from_axis_angle(F3 axis, float theta)
{
    return Q(fresnel::quat<float>::fromAxisAngle(V(axis), theta));
}

inline float point_segment_distance(float px, float py, float ax, float ay, float bx, float by)
{
    return fresnel::point_line_segment_distance(fresnel::vec2<float>(px, py),
                                                fresnel::vec2<float>(ax, ay),
                                                fresnel::vec2<float>(bx, by));
}

inline bool isect_sphere(float& t, float& d_edge, F3& N, F3 o, F3 d, F3 p, float r)
{
    fresnel::vec3<float> n;
    bool hit = fresnel::intersect_ray_sphere(t, d_edge, n, V(o), V(d), V(p), r);
    if (hit)
        N = V(n);
    return hit;
}

inline bool isect_spherocylinder(float& t, float& d_edge, F3& N, unsigned& color_index, F3 o, F3 d,
                                 F3 A, F3 B, float r)
{
    fresnel::vec3<float> n(0, 0, 0);
    bool hit = fresnel::intersect_ray_spherocylinder(t, d_edge, n, color_index, V(o), V(d), V(A),
                                                     V(B), r);
    N = V(n);
    return hit;
}

inline bool isect_triangle(float& u, float& v, float& w, float& t, float& d_edge, F3& n, F3 p, F3 q,
                           F3 a, F3 b, F3 c)
{
    fresnel::vec3<float> nn;
    bool hit = fresnel::intersect_ray_triangle(u, v, w, t, d_edge, nn, V(p), V(q), V(a), V(b), V(c));
    n = V(nn);
    return hit;
}

inline void srgb_encode(const float c[4], unsigned char out[4])
{
    fresnel::RGBA<unsigned char> r = fresnel::sRGB(fresnel::RGBA<float>(c[0], c[1], c[2], c[3]));
    out[0] = r.r;
    out[1] = r.g;
    out[2] = r.b;
    out[3] = r.a;
}

}  // namespace frref

#endif
