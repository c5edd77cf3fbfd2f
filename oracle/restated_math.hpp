// restated_math.hpp -- TEST INFRASTRUCTURE (oracle), not part of the product.
//
// A scalar CPU restatement of the shading, sampling and intersection arithmetic that fresnel
// keeps in its header-only "common" layer.  It follows the reference operation by operation
// (same association, same reciprocal-versus-true division, same float/double comparisons) so
// that, compiled with -ffp-contract=off, it reproduces the reference bit for bit.  That claim
// is checked by compiling the same oracle core a second time against the reference's own
// headers (see ref_math_adapter.hpp) and comparing outputs.
//
// Random numbers: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11) and the u01 float mapping of the Random123 library, which the reference
// includes from its (absent) extern/random123 submodule.
#ifndef FR_ORACLE_RESTATED_MATH_HPP
#define FR_ORACLE_RESTATED_MATH_HPP

#include <cfloat>
#include <cmath>
#include <cstdint>

namespace frm {

// ---------------------------------------------------------------------------------------------
// small vector / colour types (operators mirror fresnel/common/VectorMath.h:365-585 and
// fresnel/common/ColorMath.h:98-250: component-wise, left-to-right association)
// ---------------------------------------------------------------------------------------------
struct F3 {
    float x, y, z;
};
struct RGB3 {
    float r, g, b;
};
struct Quat {
    float s;
    F3 v;
};

inline F3 mk(float x, float y, float z) { return F3{x, y, z}; }
inline F3 operator+(F3 a, F3 b) { return F3{a.x + b.x, a.y + b.y, a.z + b.z}; }
inline F3 operator-(F3 a, F3 b) { return F3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline F3 operator-(F3 a) { return F3{-a.x, -a.y, -a.z}; }
inline F3 operator*(F3 a, float s) { return F3{a.x * s, a.y * s, a.z * s}; }
inline F3 operator*(float s, F3 a) { return F3{a.x * s, a.y * s, a.z * s}; }
inline float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline F3 cross(F3 a, F3 b)
{
    return F3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// "vec / scalar" in the reference multiplies by the reciprocal (VectorMath.h:506-510) ...
inline F3 div_recip(F3 a, float s)
{
    float q = 1.0f / s;
    return a * q;
}
// ... while "vec /= scalar" divides each component (VectorMath.h:533-539).
inline F3 div_each(F3 a, float s) { return F3{a.x / s, a.y / s, a.z / s}; }

inline RGB3 rgb(float r, float g, float b) { return RGB3{r, g, b}; }
inline RGB3 operator+(RGB3 a, RGB3 b) { return RGB3{a.r + b.r, a.g + b.g, a.b + b.b}; }
inline RGB3 operator-(RGB3 a, RGB3 b) { return RGB3{a.r - b.r, a.g - b.g, a.b - b.b}; }
inline RGB3 operator*(RGB3 a, RGB3 b) { return RGB3{a.r * b.r, a.g * b.g, a.b * b.b}; }
inline RGB3 operator*(RGB3 a, float s) { return RGB3{a.r * s, a.g * s, a.b * s}; }
inline RGB3 operator*(float s, RGB3 a) { return RGB3{a.r * s, a.g * s, a.b * s}; }
inline RGB3 rgb_div_recip(RGB3 a, float s)  // ColorMath.h:215-219
{
    float q = 1.0f / s;
    return a * q;
}
inline RGB3 rgb_div_each(RGB3 a, float s) { return RGB3{a.r / s, a.g / s, a.b / s}; }
// lerp(x, a, b) = (1-x)*a + x*b  (ColorMath.h:496-500)
inline RGB3 lerp(float x, RGB3 a, RGB3 b) { return (1.0f - x) * a + x * b; }

// Quaternion helpers (VectorMath.h:924-928, 1068-1092).  The reference's host build maps
// fast::cos/fast::sin to cosf/sinf.
inline Quat conj(Quat q) { return Quat{q.s, -q.v}; }
inline F3 rotate(Quat a, F3 b)
{
    return (a.s * a.s - dot(a.v, a.v)) * b + 2 * a.s * cross(a.v, b) + 2 * dot(a.v, b) * a.v;
}
inline Quat from_axis_angle(F3 axis, float theta)
{
    return Quat{cosf(theta / 2.0f), sinf(theta / 2.0f) * axis};
}

// Distance from p to the segment ab in 2-D (fresnel/common/GeometryMath.h:28-39): clamp the
// projection parameter with std::min/std::max semantics, then the length of p - projection.
inline float point_segment_distance(float px, float py, float ax, float ay, float bx, float by)
{
    const float abx = bx - ax, aby = by - ay;
    const float L = abx * abx + aby * aby;
    const float q = ((px - ax) * abx + (py - ay) * aby) / L;
    const float lo = (q < 1.0f) ? q : 1.0f;  // std::min(1.0f, q)
    const float t = (0.0f < lo) ? lo : 0.0f;  // std::max(0.0f, lo)
    const float vx = px - (ax + t * abx), vy = py - (ay + t * aby);
    return sqrtf(vx * vx + vy * vy);
}

// ---------------------------------------------------------------------------------------------
// Philox4x32-10 and u01 (Random123 semantics used at fresnel/common/RayGen.h:49-61,
// fresnel/common/Camera.h:190-201,230-242)
// ---------------------------------------------------------------------------------------------
struct Ctr4 {
    uint32_t v[4];
};

inline void mul_hi_lo(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo)
{
    uint64_t p = uint64_t(a) * uint64_t(b);
    hi = uint32_t(p >> 32);
    lo = uint32_t(p);
}

// 10 rounds; the key is bumped by the Weyl constants between rounds.
inline Ctr4 philox4x32_10(Ctr4 c, uint32_t k0, uint32_t k1)
{
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int round = 0; round < 10; ++round) {
        if (round > 0) {
            k0 += W0;
            k1 += W1;
        }
        uint32_t hi0, lo0, hi1, lo1;
        mul_hi_lo(M0, c.v[0], hi0, lo0);
        mul_hi_lo(M1, c.v[2], hi1, lo1);
        Ctr4 n;
        n.v[0] = hi1 ^ c.v[1] ^ k0;
        n.v[1] = lo1;
        n.v[2] = hi0 ^ c.v[3] ^ k1;
        n.v[3] = lo0;
        c = n;
    }
    return c;
}

// Random123 u01<float>: a 32-bit word to (0,1] as x * 2^-32 + 2^-33, in float arithmetic.
inline float u01(uint32_t x)
{
    const float factor = 1.0f / 4294967296.0f;
    const float half_factor = 0.5f * factor;
    return float(x) * factor + half_factor;
}

// Counter tags (fresnel/common/Camera.h:302-305, fresnel/common/RayGen.h:31-37).
const uint32_t TAG_APERTURE = 0x983abc12u;
const uint32_t TAG_AA = 0x22ab5871u;
const uint32_t TAG_MIS = 0x8754abcdu;
const uint32_t TAG_RR = 0x54abf853u;

// ---------------------------------------------------------------------------------------------
// Camera (fresnel/common/Camera.h:55-309)
// ---------------------------------------------------------------------------------------------
struct CameraIn {
    F3 position, look_at, up;
    float h, f, f_stop, focus_distance;
    int model;  // 0 orthographic, 1 perspective
};

struct Basis {
    F3 u, v, w;
};

// CameraBasis(const UserCamera&) (Camera.h:89-113)
inline Basis make_basis(const CameraIn& c)
{
    Basis b;
    F3 d = c.look_at - c.position;
    F3 v = c.up;
    float sd = 1.0f / sqrtf(dot(d, d));
    d = d * sd;
    float sv = 1.0f / sqrtf(dot(v, v));
    v = v * sv;
    F3 u = cross(d, v);
    float su = 1.0f / sqrtf(dot(u, u));
    u = u * su;
    v = cross(u, d);
    sv = 1.0f / sqrtf(dot(v, v));
    v = v * sv;
    b.u = u;
    b.v = v;
    b.w = -d;
    return b;
}

struct Cam {
    F3 p;
    Basis basis;
    float focal_h, focal_d, aperture;
    int model;
    unsigned width, height, seed;
    bool sample_aa;
};

inline Cam make_camera(const CameraIn& c, unsigned width, unsigned height, unsigned seed,
                       bool sample_aa)
{
    Cam k;
    k.p = c.position;
    k.basis = make_basis(c);
    k.focal_d = c.focus_distance;
    k.aperture = c.f / c.f_stop;
    k.model = c.model;
    k.width = width;
    k.height = height;
    k.seed = seed;
    k.sample_aa = sample_aa;
    k.focal_h = (c.model == 0) ? c.h : c.h / c.f * k.focal_d;
    return k;
}

// importanceSampleAA (Camera.h:226-269): tent filter of half-width 1/sqrt(2) px.
inline void image_plane_sample(const Cam& k, unsigned i, unsigned j, unsigned sample, float& xs,
                               float& ys)
{
    float i_f, j_f;
    if (k.sample_aa) {
        unsigned pixel = j * k.width + i;
        Ctr4 c{{0u, 0u, sample, TAG_AA}};
        Ctr4 r = philox4x32_10(c, pixel, k.seed);
        float r1 = u01(r.v[0]) * 2.0f;
        float r2 = u01(r.v[1]) * 2.0f;
        float dx = (r1 < 1.0f) ? sqrtf(r1) - 1.0f : 1.0f - sqrtf(2.0f - r1);
        float dy = (r2 < 1.0f) ? sqrtf(r2) - 1.0f : 1.0f - sqrtf(2.0f - r2);
        const float aa_w = 0.707106781f;
        i_f = float(i) + 0.5f + dx * aa_w;
        j_f = float(j) + 0.5f + dy * aa_w;
    } else {
        i_f = float(i) + 0.5f;
        j_f = float(j) + 0.5f;
    }
    ys = -1.0f * (j_f / float(k.height) - 0.5f);
    xs = i_f / float(k.height) - 0.5f * float(k.width) / float(k.height);
}

// generateRay (Camera.h:169-209)
inline void camera_ray(const Cam& k, unsigned i, unsigned j, unsigned sample, F3& origin,
                       F3& direction)
{
    float xs, ys;
    image_plane_sample(k, i, j, sample, xs, ys);
    F3 plane = ys * k.basis.v + xs * k.basis.u;
    if (k.model == 0) {
        origin = k.p + plane * k.focal_h;
        direction = -k.basis.w;
        return;
    }
    F3 F = k.p - k.basis.w * k.focal_d;
    F3 C = F + plane * k.focal_h;
    {
        unsigned pixel = j * k.width + i;
        Ctr4 c{{0u, 0u, sample, TAG_APERTURE}};
        Ctr4 r = philox4x32_10(c, pixel, k.seed);
        float theta = u01(r.v[0]) * 2.0f * float(M_PI);
        float rad = u01(r.v[1]) * k.aperture * 0.5f;
        F3 offset = rad * cosf(theta) * k.basis.u + rad * sinf(theta) * k.basis.v;
        origin = k.p + offset;
    }
    direction = C - origin;
    float s = 1.0f / sqrtf(dot(direction, direction));
    direction = direction * s;
}

// ---------------------------------------------------------------------------------------------
// Lights in scene space (fresnel/common/Light.h:47-66)
// ---------------------------------------------------------------------------------------------
struct LightsW {
    F3 dir[4];
    RGB3 color[4];
    float theta[4];
    unsigned n;
};

inline LightsW lights_to_world(const F3* dir_cam, const RGB3* color, const float* theta,
                               unsigned n, const Cam& k)
{
    LightsW L;
    L.n = n;
    for (unsigned i = 0; i < n; ++i) {
        L.color[i] = color[i];
        F3 v = dir_cam[i];
        float s = 1.0f / sqrtf(dot(v, v));
        v = v * s;
        L.dir[i] = v.x * k.basis.u + v.y * k.basis.v + v.z * k.basis.w;
        L.theta[i] = theta[i];
    }
    return L;
}

// ---------------------------------------------------------------------------------------------
// Material: Disney principled BRDF (fresnel/common/Material.h:24-313)
// ---------------------------------------------------------------------------------------------
struct Mat {
    float solid;
    RGB3 color;
    float primitive_color_mix, roughness, specular, metal, spec_trans;
};

inline float schlick5(float x)  // Material.h:27-34
{
    float v = 1.0f - x;
    float v2 = v * v;
    return v2 * v2 * v;
}

inline bool is_solid(const Mat& m) { return m.solid > 0.5f; }
inline RGB3 base_color(const Mat& m, RGB3 shading) { return lerp(m.primitive_color_mix, m.color, shading); }

// The D (GTR2), F (Schlick) and V (Smith-like) terms shared by brdf and brdf_specular.
inline float ggx_d(float alpha_sq, float ndoth)
{
    float denom_rt = (1.0f + (alpha_sq - 1.0f) * ndoth * ndoth);
    return alpha_sq / (float(M_PI) * denom_rt * denom_rt);
}
inline RGB3 fresnel_f(const Mat& m, RGB3 base, float ldoth)
{
    RGB3 f0d = rgb(0.08f * m.specular, 0.08f * m.specular, 0.08f * m.specular);
    RGB3 f0 = lerp(m.metal, f0d, base);
    return f0 + (rgb(1.0f, 1.0f, 1.0f) - f0) * schlick5(ldoth);
}
inline float smith_v(float alpha_sq, float ndotv, float ndotl)
{
    float ndotv_sq = ndotv * ndotv;
    float ndotl_sq = ndotl * ndotl;
    float v1 = 1.0f / (ndotv + sqrtf(alpha_sq + ndotv_sq - alpha_sq * ndotv_sq));
    float v2 = 1.0f / (ndotl + sqrtf(alpha_sq + ndotl_sq - alpha_sq * ndotl_sq));
    return v1 * v2;
}
inline RGB3 diffuse_term(const Mat& m, RGB3 base, float ndotl, float ndotv, float ldoth)
{
    float FL = schlick5(ndotl);
    float FV = schlick5(ndotv);
    float RR = 2 * m.roughness * ldoth * ldoth;
    float s = (1.0f - 0.5f * FL) * (1.0f - 0.5f * FV) + RR * (FL + FV + FL * FV * (RR - 1.0f));
    return rgb_div_recip(base, float(M_PI)) * s;
}

// Material::brdf (Material.h:67-122)
inline RGB3 brdf(const Mat& m, F3 l, F3 v, F3 n, RGB3 shading)
{
    float ndotv = dot(n, v);
    if (ndotv <= 0)
        return rgb(0, 0, 0);
    F3 h = div_each(l + v, sqrtf(dot(l + v, l + v)));
    float ndotl = dot(n, l);
    float ldoth = dot(l, h);
    float ndoth = dot(n, h);
    RGB3 base = base_color(m, shading);
    RGB3 f_d = diffuse_term(m, base, ndotl, ndotv, ldoth);
    float alpha = m.roughness * m.roughness;
    float alpha_sq = alpha * alpha;
    float D = ggx_d(alpha_sq, ndoth);
    RGB3 F = fresnel_f(m, base, ldoth);
    float V = smith_v(alpha_sq, ndotv, ndotl);
    RGB3 f_s = D * F * V;
    return f_d * (1.0f - m.metal) + f_s;
}

// Material::brdf_diffuse (Material.h:124-151)
inline RGB3 brdf_diffuse(const Mat& m, F3 l, F3 v, F3 n, RGB3 shading)
{
    float ndotv = dot(n, v);
    if (ndotv <= 0 || m.metal == 1.0f)
        return rgb(0, 0, 0);
    F3 h = div_each(l + v, sqrtf(dot(l + v, l + v)));
    float ndotl = dot(n, l);
    float ldoth = dot(l, h);
    RGB3 base = base_color(m, shading);
    return diffuse_term(m, base, ndotl, ndotv, ldoth) * (1.0f - m.metal);
}

// Material::brdf_specular (Material.h:153-218), with the representative-point normalisation.
inline RGB3 brdf_specular(const Mat& m, F3 l, F3 v, F3 n, RGB3 shading, float light_half_angle)
{
    float ndotv = dot(n, v);
    if (ndotv <= 0)
        return rgb(0, 0, 0);
    F3 h = div_each(l + v, sqrtf(dot(l + v, l + v)));
    float ndotl = dot(n, l);
    float ldoth = dot(l, h);
    float ndoth = dot(n, h);
    RGB3 base = base_color(m, shading);
    float alpha = m.roughness * m.roughness;
    float alpha_sq = alpha * alpha;
    float D = ggx_d(alpha_sq, ndoth);
    if (light_half_angle > 0.99f * float(M_PI) / 2.0f)
        light_half_angle = 0.99f * float(M_PI) / 2.0f;
    if (light_half_angle > 0.0f) {
        float alpha_prime = alpha + 0.5f * tanf(light_half_angle);
        if (alpha_prime > 1.0f)
            alpha_prime = 1.0f;
        D = D * alpha_sq / (alpha_prime * alpha_prime);
    }
    RGB3 F = fresnel_f(m, base, ldoth);
    float V = smith_v(alpha_sq, ndotv, ndotl);
    return D * F * V;
}

// Tangent frame used by both importance samplers (Material.h:241-250, 294-301).  The pole test
// compares in double, as `fabs(float) > 0.999` does in the reference.
inline void tangent_frame(F3 n, F3& t_x, F3& t_y)
{
    F3 up = mk(0, 0, 1.0f);
    if (double(fabsf(n.z)) > 0.999)
        up = mk(1.0f, 0, 0);
    t_x = cross(up, n);
    t_x = div_recip(t_x, sqrtf(dot(t_x, t_x)));
    t_y = cross(n, t_x);
}

// importanceSampleGGX (Material.h:230-256)
inline F3 sample_ggx(const Mat& m, float xi0, float xi1, F3 v, F3 n)
{
    float alpha = m.roughness * m.roughness;
    float phi = 2.0f * float(M_PI) * xi0;
    float cos_t = sqrtf((1.0f - xi1) / (1.0f + (alpha * alpha - 1.0f) * xi1));
    float sin_t = sqrtf(1.0f - cos_t * cos_t);
    F3 ht = mk(sin_t * cosf(phi), sin_t * sinf(phi), cos_t);
    F3 t_x, t_y;
    tangent_frame(n, t_x, t_y);
    F3 h = t_x * ht.x + t_y * ht.y + n * ht.z;
    return 2.0f * dot(v, h) * h - v;
}

// pdfGGX (Material.h:258-280)
inline float pdf_ggx(const Mat& m, F3 l, F3 v, F3 n)
{
    F3 h = div_each(l + v, sqrtf(dot(l + v, l + v)));
    float ldoth = dot(l, h);
    float ndoth = dot(n, h);
    float alpha = m.roughness * m.roughness;
    float alpha_sq = alpha * alpha;
    float D = ggx_d(alpha_sq, ndoth);
    float pdf = D * ndoth / (4.0f * ldoth);
    return (pdf > 0.0f) ? pdf : 0.0f;
}

// importanceSampleDiffuse (Material.h:282-304): cosine-weighted hemisphere.
inline F3 sample_diffuse(float xi0, float xi1, F3 v, F3 n)
{
    (void)v;
    const float r = sqrtf(xi0);
    const float theta = 2 * float(M_PI) * xi1;
    F3 vt = mk(r * cosf(theta), r * sinf(theta), sqrtf(1.0f - xi0));
    F3 t_x, t_y;
    tangent_frame(n, t_x, t_y);
    return t_x * vt.x + t_y * vt.y + n * vt.z;
}

// pdfDiffuse (Material.h:306-313)
inline float pdf_diffuse(F3 l, F3 n)
{
    float ndotl = dot(n, l);
    return (ndotl > 0.0f) ? ndotl / float(M_PI) : 0.0f;
}

// ---------------------------------------------------------------------------------------------
// Path tracing kernels (fresnel/common/RayGen.h:110-186, fresnel/common/TracerPathMethods.h)
// ---------------------------------------------------------------------------------------------
struct PathState {  // PRDpath (TracerPathMethods.h:24-34)
    RGB3 result;
    float a;
    RGB3 att;
    F3 origin, dir;
    unsigned light_sample, depth;
    bool done;
};

// MISReflectionTransmission (RayGen.h:110-157)
inline F3 mis_direction(float& factor, bool& transmit, F3 v, F3 n, unsigned depth, unsigned sample,
                        unsigned key0, unsigned key1, const Mat& m)
{
    Ctr4 c{{0u, depth, sample, TAG_MIS}};
    Ctr4 r = philox4x32_10(c, key0, key1);
    float xi0 = u01(r.v[0]);
    float xi1 = u01(r.v[1]);
    float choice_mis = u01(r.v[2]);
    float choice_trans = u01(r.v[3]);
    F3 l;
    transmit = (choice_trans <= m.spec_trans);
    if (transmit) {
        l = -v;
    } else if (choice_mis <= 0.5f) {
        l = sample_diffuse(xi0, xi1, v, n);
        float pd = pdf_diffuse(l, n);
        float pg = pdf_ggx(m, l, v, n);
        float w = pd / (pd + pg);
        factor = w / (0.5f * pd);
    } else {
        l = sample_ggx(m, xi0, xi1, v, n);
        float pd = pdf_diffuse(l, n);
        float pg = pdf_ggx(m, l, v, n);
        float w = pg / (pd + pg);
        factor = w / (0.5f * pg);
    }
    return l;
}

// shouldTerminatePath (RayGen.h:168-186)
inline bool russian_roulette(RGB3& att, unsigned depth, unsigned sample, unsigned key0,
                             unsigned key1)
{
    Ctr4 c{{0u, depth, sample, TAG_RR}};
    Ctr4 r = philox4x32_10(c, key0, key1);
    float p = fmaxf(att.r, fmaxf(att.g, att.b));
    p = fminf(p, 1.0f);
    if (u01(r.v[0]) > p)
        return true;
    att = rgb_div_each(att, p);
    return false;
}

// path_tracer_miss (TracerPathMethods.h:36-77)
inline void path_miss(PathState& s, RGB3 bg, float bg_alpha, unsigned light_samples,
                      const LightsW& L, F3 ray_dir)
{
    if (s.depth == 0) {
        s.result = bg * float(light_samples);
        s.a = bg_alpha;
    } else {
        for (unsigned i = 0; i < L.n; ++i) {
            F3 l = L.dir[i];
            float half = L.theta[i];
            float cos_half = cosf(half);
            if (half > float(M_PI) / 2.0f)
                half = float(M_PI) / 2.0f;
            float ldotd = dot(l, ray_dir);
            if (ldotd >= cos_half)
                s.result = s.result + rgb_div_recip(s.att * L.color[i], sinf(half));
        }
    }
    s.done = true;
}

// path_tracer_hit (TracerPathMethods.h:79-168)
inline void path_hit(PathState& s, const Mat& material, const Mat& outline, float shading_distance,
                     float outline_width, RGB3 shading_color, F3 shading_normal, F3 ray_o,
                     F3 ray_d, float t_hit, unsigned key0, unsigned key1, unsigned n_samples,
                     unsigned light_samples)
{
    const Mat& m = (shading_distance >= outline_width) ? material : outline;
    F3 n = shading_normal * (1.0f / sqrtf(dot(shading_normal, shading_normal)));
    F3 v = -ray_d;
    if (is_solid(m)) {
        s.result = s.result + s.att * base_color(m, shading_color);
        s.done = true;
        return;
    }
    float factor = 1.0f;
    bool transmit = false;
    unsigned sample = (n_samples - 1) * light_samples + s.light_sample;
    F3 l = mis_direction(factor, transmit, v, n, s.depth, sample, key0, key1, m);
    if (transmit) {
        RGB3 tc = base_color(m, shading_color);
        tc.r = sqrtf(tc.r);
        tc.g = sqrtf(tc.g);
        tc.b = sqrtf(tc.b);
        s.att = s.att * tc;
    } else {
        float ndotl = dot(n, l);
        if (dot(n, v) > 0.0f && ndotl > 0.0f) {
            s.att = s.att * (brdf(m, l, v, n, shading_color) * ndotl * factor);
        } else {
            s.att = rgb(0, 0, 0);
            s.done = true;
        }
    }
    s.origin = ray_o + ray_d * t_hit;
    s.dir = l;
    if (russian_roulette(s.att, s.depth, sample, key0, key1))
        s.done = true;
}

// ---------------------------------------------------------------------------------------------
// Intersectors (fresnel/common/IntersectSphere.h, IntersectCylinder.h, IntersectTriangle.h)
// ---------------------------------------------------------------------------------------------

// intersect_ray_sphere (IntersectSphere.h:36-85)
inline bool isect_sphere(float& t, float& d_edge, F3& N, F3 o, F3 d, F3 p, float r)
{
    const float eps = 1e-4f;
    F3 v = p - o;
    float b = dot(v, d);
    float det = b * b - dot(v, v) + r * r;
    if (det < 0)
        return false;
    F3 w = cross(v, d);
    float Dsq = dot(w, w);
    d_edge = r - sqrtf(Dsq);
    det = sqrtf(det);
    t = b - det;
    if (t > eps) {
        N = o + t * d - p;
        return true;
    }
    t = b + det;
    if (t > eps) {
        N = -(o + t * d - p);
        return true;
    }
    return false;
}

// intersect_ray_cylinder (IntersectCylinder.h:35-113)
inline bool isect_cylinder(float& t, F3& N, F3 o, F3 d, F3 A, F3 B, float r)
{
    const float eps = 1e-4f;
    const F3 Oa = o - A;
    const F3 C = B - A;
    float cc_inv = 1.0f / dot(C, C);
    float cd = dot(C, d);
    float co = dot(C, Oa);
    float a = (1.0f - cd * cd * cc_inv);
    float mb = -2.0f * (dot(Oa, d) - co * cd * cc_inv);
    float c = dot(Oa, Oa) - co * co * cc_inv - r * r;
    float det = mb * mb - 4 * a * c;
    if (det < 0)
        return false;
    det = sqrtf(det);
    bool hit = false;
    F3 P = mk(0, 0, 0);
    float pc = 0;
    t = (mb - det) / (2.0f * a);
    if (t > eps) {
        P = Oa + t * d;
        pc = dot(P, C);
        if (pc >= 0 && pc <= dot(C, C))
            hit = true;
    }
    if (!hit) {
        t = (mb + det) / (2.0f * a);
        if (t > eps) {
            P = Oa + t * d;
            pc = dot(P, C);
            if (pc >= 0 && pc <= dot(C, C))
                hit = true;
        }
    }
    if (hit) {
        N = (P - pc * cc_inv * C);
        if (dot(N, d) > 0)
            N = -N;
    }
    return hit;
}

// intersect_ray_spherocylinder (IntersectCylinder.h:131-227)
inline bool isect_spherocylinder(float& t, float& d_edge, F3& N, unsigned& color_index, F3 o, F3 d,
                                 F3 A, F3 B, float r)
{
    t = HUGE_VALF;
    float t_sc = 0;
    float de_sc = HUGE_VALF;
    F3 N_sc = mk(0, 0, 0);
    const F3 Oa = o - A;
    const F3 C = B - A;
    const float cdotc = dot(C, C);
    bool hit_cyl = isect_cylinder(t_sc, N_sc, o, d, A, B, r);
    if (hit_cyl && t_sc < t) {
        t = t_sc;
        N = N_sc;
    }
    bool hit_A = isect_sphere(t_sc, de_sc, N_sc, o, d, A, r);
    if (hit_A && (t_sc < t)) {
        const F3 PA = Oa + t_sc * d;
        if (dot(PA, C) <= 0) {
            t = t_sc;
            N = N_sc;
        } else {
            hit_A = false;
        }
    }
    bool hit_B = isect_sphere(t_sc, de_sc, N_sc, o, d, B, r);
    if (hit_B && (t_sc < t)) {
        const F3 PA = Oa + t_sc * d;
        if (dot(PA, C) >= cdotc) {
            t = t_sc;
            N = N_sc;
        } else {
            hit_B = false;
        }
    }
    const F3 P = Oa + t * d;
    const float pdotc = dot(P, C);
    color_index = (pdotc < cdotc / 2.0f) ? 0u : 1u;
    const F3 C_vp = C - dot(C, d) * d;
    const F3 Oa_vp = Oa - dot(Oa, d) * d;
    const float oc = dot(Oa_vp, C_vp);
    const float cc = dot(C_vp, C_vp);
    if (oc < 0) {
        d_edge = r - sqrtf(dot(Oa_vp, Oa_vp));
    } else if (oc > cc) {
        d_edge = r - sqrtf(dot(Oa_vp - C_vp, Oa_vp - C_vp));
    } else {
        const F3 n_vp = Oa_vp - oc / cc * C_vp;
        d_edge = r - sqrtf(dot(n_vp, n_vp));
    }
    return hit_A || hit_B || hit_cyl;
}

// intersect_ray_triangle (IntersectTriangle.h:43-132): Ericson's segment/triangle test against
// the counter-clockwise face, barycentrics and the distance to the nearest edge.
inline bool isect_triangle(float& u, float& v, float& w, float& t, float& d_edge, F3& n, F3 p, F3 q,
                           F3 a, F3 b, F3 c)
{
    F3 ab = b - a;
    F3 ac = c - a;
    F3 qp = p - q;
    n = cross(ab, ac);
    float d = dot(qp, n);
    if (d <= 0.0f)
        return false;
    F3 ap = p - a;
    t = dot(ap, n);
    if (t < 0.0f)
        return false;
    F3 e = cross(qp, ap);
    v = dot(ac, e);
    if (v < 0.0f || v > d)
        return false;
    w = -dot(ab, e);
    if (w < 0.0f || v + w > d)
        return false;
    float ood = 1.0f / d;
    t *= ood;
    v *= ood;
    w *= ood;
    u = 1.0f - v - w;
    F3 edge, pt;
    if (u < v) {
        if (u < w) {
            edge = c - b;
            pt = b;
        } else {
            edge = b - a;
            pt = a;
        }
    } else {
        if (v < w) {
            edge = a - c;
            pt = c;
        } else {
            edge = b - a;
            pt = a;
        }
    }
    F3 r_hit = p + t * (q - p);
    F3 vec = cross(edge, r_hit - pt);
    float dsq = dot(vec, vec) / dot(edge, edge);
    d_edge = sqrtf(dsq);
    return true;
}

// ---------------------------------------------------------------------------------------------
// sRGB encoding (fresnel/common/ColorMath.h:506-546)
// ---------------------------------------------------------------------------------------------
inline unsigned char to_byte(float x) { return (unsigned char)(x * 255.0f + 0.5f); }

inline void srgb_encode(const float c[4], unsigned char out[4])
{
    float t[3];
    for (int k = 0; k < 3; ++k) {
        float x = c[k];
        float y = (x < 0.0031308f) ? 12.92f * x : (1.0f + 0.055f) * powf(x, 1.0f / 2.4f) - 0.055f;
        if (y > 1.0f)
            y = 1.0f;
        t[k] = y;
    }
    out[0] = to_byte(t[0]);
    out[1] = to_byte(t[1]);
    out[2] = to_byte(t[2]);
    out[3] = to_byte(c[3]);
}

}  // namespace frm

#endif
