// frmath.cuh -- shading, sampling and intersection arithmetic of the path-tracing hot path.
//
// Host+device inline functions restating fresnel's header-only "common" layer
// (fresnel/common/{Camera,RayGen,Material,Light,TracerPathMethods,IntersectSphere,
// IntersectCylinder,IntersectTriangle,ColorMath,VectorMath}.h) for sm_100a.  Every expression
// keeps the reference's association order, its reciprocal-versus-true divisions and its
// float/double comparisons; the library is compiled with -fmad=false, so additions and
// multiplications round exactly as the reference's host build does and the closest-hit t of
// every intersector is bit-identical.  Transcendentals go through hsin/hcos/htan/hacos/hpow
// below: on the host they are the C library's float functions, as in the reference; on the
// device they are the double-precision functions rounded once to float.
#ifndef FR_FRMATH_CUH
#define FR_FRMATH_CUH

#include <cstdint>
#include <math_constants.h>

#ifndef FR_HD
#define FR_HD __host__ __device__ __forceinline__
#endif

namespace fr {

// --------------------------------------------------------------------------------------------
// transcendentals
//
// The reference's CPU path calls the host C library's sinf, cosf, tanf, acosf and powf.  A
// float function with at most about half an ulp of error returns the correctly rounded result
// almost everywhere; on the device the double-precision function rounded once to float gives
// exactly that (but for arguments whose exact value lies within a double's rounding of the
// midpoint between two floats).  The two agree bit for bit on all but about 0.1% of the
// arguments of sin and cos over [0, 2 pi] with glibc 2.39 (every float argument checked),
// where CUDA's single-precision functions (a few ulp of error) differ far more often.  Bit
// agreement matters because a last-place difference in a sampled direction is amplified bounce
// after bounce in dense scenes until the paths take different branches.
// --------------------------------------------------------------------------------------------
FR_HD float hsin(float x)
{
#ifdef __CUDA_ARCH__
    return float(sin(double(x)));
#else
    return sinf(x);
#endif
}
FR_HD float hcos(float x)
{
#ifdef __CUDA_ARCH__
    return float(cos(double(x)));
#else
    return cosf(x);
#endif
}
// sin and cos of one argument (the direction samplers)
FR_HD void hsincos(float x, float& s, float& c)
{
#ifdef __CUDA_ARCH__
    double sd, cd;
    sincos(double(x), &sd, &cd);
    s = float(sd);
    c = float(cd);
#else
    s = sinf(x);
    c = cosf(x);
#endif
}
FR_HD float htan(float x)
{
#ifdef __CUDA_ARCH__
    return float(tan(double(x)));
#else
    return tanf(x);
#endif
}
FR_HD float hacos(float x)
{
#ifdef __CUDA_ARCH__
    return float(acos(double(x)));
#else
    return acosf(x);
#endif
}
FR_HD float hpow(float x, float y)
{
#ifdef __CUDA_ARCH__
    return float(pow(double(x), double(y)));
#else
    return powf(x, y);
#endif
}

// --------------------------------------------------------------------------------------------
// vectors and colours (fresnel/common/VectorMath.h:365-585, ColorMath.h:98-250)
// --------------------------------------------------------------------------------------------
struct V3 {
    float x, y, z;
};
struct C3 {
    float r, g, b;
};
struct Qt {
    float s;
    V3 v;
};

FR_HD V3 v3(float x, float y, float z) { return V3{x, y, z}; }
FR_HD V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
FR_HD V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
FR_HD V3 operator-(V3 a) { return V3{-a.x, -a.y, -a.z}; }
FR_HD V3 operator*(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
FR_HD V3 operator*(float s, V3 a) { return V3{a.x * s, a.y * s, a.z * s}; }
FR_HD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
FR_HD V3 cross(V3 a, V3 b)
{
    return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// vec / scalar multiplies by the reciprocal (VectorMath.h:506-510) ...
FR_HD V3 div_recip(V3 a, float s)
{
    float q = 1.0f / s;
    return a * q;
}
// ... and vec /= scalar divides component-wise (VectorMath.h:533-539).
FR_HD V3 div_each(V3 a, float s) { return V3{a.x / s, a.y / s, a.z / s}; }

FR_HD C3 c3(float r, float g, float b) { return C3{r, g, b}; }
FR_HD C3 operator+(C3 a, C3 b) { return C3{a.r + b.r, a.g + b.g, a.b + b.b}; }
FR_HD C3 operator-(C3 a, C3 b) { return C3{a.r - b.r, a.g - b.g, a.b - b.b}; }
FR_HD C3 operator*(C3 a, C3 b) { return C3{a.r * b.r, a.g * b.g, a.b * b.b}; }
FR_HD C3 operator*(C3 a, float s) { return C3{a.r * s, a.g * s, a.b * s}; }
FR_HD C3 operator*(float s, C3 a) { return C3{a.r * s, a.g * s, a.b * s}; }
FR_HD C3 c_div_recip(C3 a, float s)
{
    float q = 1.0f / s;
    return a * q;
}
FR_HD C3 c_div_each(C3 a, float s) { return C3{a.r / s, a.g / s, a.b / s}; }
FR_HD C3 lerp(float x, C3 a, C3 b) { return (1.0f - x) * a + x * b; }

// quaternions (s, x, y, z) (VectorMath.h:924-928, 1068-1092)
FR_HD Qt conj(Qt q) { return Qt{q.s, -q.v}; }
FR_HD V3 rotate(Qt a, V3 b)
{
    return (a.s * a.s - dot(a.v, a.v)) * b + 2 * a.s * cross(a.v, b) + 2 * dot(a.v, b) * a.v;
}
FR_HD Qt from_axis_angle(V3 axis, float theta)
{
    return Qt{hcos(theta / 2.0f), hsin(theta / 2.0f) * axis};
}

// --------------------------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC'11) and Random123's u01<float>, keyed and countered as in
// fresnel/common/RayGen.h:49-61 and Camera.h:190-201,230-242.
// --------------------------------------------------------------------------------------------
struct U4 {
    uint32_t x, y, z, w;
};

FR_HD U4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1)
{
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int round = 0; round < 10; ++round) {
        // one 32x32 -> 64-bit product per multiplier gives both halves
        const uint64_t p0 = uint64_t(M0) * c0, p1 = uint64_t(M1) * c2;
        uint32_t n0 = uint32_t(p1 >> 32) ^ c1 ^ k0, n2 = uint32_t(p0 >> 32) ^ c3 ^ k1;
        c0 = n0;
        c1 = uint32_t(p1);
        c2 = n2;
        c3 = uint32_t(p0);
        k0 += W0;
        k1 += W1;
    }
    return U4{c0, c1, c2, c3};
}

// x * 2^-32 + 2^-33 in float: the product is exact, so fused or not the result is the same.
FR_HD float u01(uint32_t x) { return float(x) * 2.3283064365386963e-10f + 1.1641532182693481e-10f; }

constexpr uint32_t TAG_APERTURE = 0x983abc12u;
constexpr uint32_t TAG_AA = 0x22ab5871u;
constexpr uint32_t TAG_MIS = 0x8754abcdu;
constexpr uint32_t TAG_RR = 0x54abf853u;

constexpr float PI_F = 3.14159265358979323846f;

// --------------------------------------------------------------------------------------------
// camera (fresnel/common/Camera.h:89-309); the per-render constants are prepared on the host.
// --------------------------------------------------------------------------------------------
struct CamK {
    V3 p, u, v, w;
    float focal_h, focal_d, aperture;
    int model;      // 0 orthographic, 1 perspective
    int sample_aa;  // tent-filter jitter on/off
    uint32_t width, height, seed;
};

// CameraBasis (Camera.h:89-113)
FR_HD void camera_basis(V3 position, V3 look_at, V3 up, V3& u, V3& v, V3& w)
{
    V3 d = look_at - position;
    d = d * (1.0f / sqrtf(dot(d, d)));
    V3 vv = up * (1.0f / sqrtf(dot(up, up)));
    V3 uu = cross(d, vv);
    uu = uu * (1.0f / sqrtf(dot(uu, uu)));
    vv = cross(uu, d);
    vv = vv * (1.0f / sqrtf(dot(vv, vv)));
    u = uu;
    v = vv;
    w = -d;
}

// importanceSampleAA + generateRay (Camera.h:169-269)
FR_HD void camera_ray(const CamK& k, uint32_t i, uint32_t j, uint32_t sample, V3& origin, V3& dir)
{
    float i_f, j_f;
    const uint32_t pixel = j * k.width + i;
    if (k.sample_aa) {
        U4 r = philox(0u, 0u, sample, TAG_AA, pixel, k.seed);
        float r1 = u01(r.x) * 2.0f;
        float r2 = u01(r.y) * 2.0f;
        float dx = (r1 < 1.0f) ? sqrtf(r1) - 1.0f : 1.0f - sqrtf(2.0f - r1);
        float dy = (r2 < 1.0f) ? sqrtf(r2) - 1.0f : 1.0f - sqrtf(2.0f - r2);
        const float aa_w = 0.707106781f;
        i_f = float(i) + 0.5f + dx * aa_w;
        j_f = float(j) + 0.5f + dy * aa_w;
    } else {
        i_f = float(i) + 0.5f;
        j_f = float(j) + 0.5f;
    }
    float ys = -1.0f * (j_f / float(k.height) - 0.5f);
    float xs = i_f / float(k.height) - 0.5f * float(k.width) / float(k.height);
    V3 plane = ys * k.v + xs * k.u;
    if (k.model == 0) {
        origin = k.p + plane * k.focal_h;
        dir = -k.w;
        return;
    }
    V3 F = k.p - k.w * k.focal_d;
    V3 C = F + plane * k.focal_h;
    if (k.aperture == 0.0f && k.p.x != 0.0f && k.p.y != 0.0f && k.p.z != 0.0f) {
        // pinhole (f_stop infinite): the lens sample is scaled by a zero aperture, so the offset
        // is a signed zero in each component and p + offset is exactly p (no component of p is
        // zero); the lens sample need not be drawn
        origin = k.p;
    } else {
        U4 r = philox(0u, 0u, sample, TAG_APERTURE, pixel, k.seed);
        float theta = u01(r.x) * 2.0f * PI_F;
        float rad = u01(r.y) * k.aperture * 0.5f;
        float st, ct;
        hsincos(theta, st, ct);
        V3 offset = rad * ct * k.u + rad * st * k.v;
        origin = k.p + offset;
    }
    dir = C - origin;
    dir = dir * (1.0f / sqrtf(dot(dir, dir)));
}

// --------------------------------------------------------------------------------------------
// materials: Disney principled BRDF (fresnel/common/Material.h:24-313)
// --------------------------------------------------------------------------------------------
struct Mat {
    float solid;
    C3 color;
    float primitive_color_mix, roughness, specular, metal, spec_trans;
};

FR_HD float schlick5(float x)
{
    float v = 1.0f - x;
    float v2 = v * v;
    return v2 * v2 * v;
}
FR_HD bool is_solid(const Mat& m) { return m.solid > 0.5f; }
FR_HD C3 base_color(const Mat& m, C3 sc) { return lerp(m.primitive_color_mix, m.color, sc); }
FR_HD float ggx_d(float alpha_sq, float ndoth)
{
    float denom_rt = (1.0f + (alpha_sq - 1.0f) * ndoth * ndoth);
    return alpha_sq / (PI_F * denom_rt * denom_rt);
}
FR_HD C3 fresnel_term(const Mat& m, C3 base, float ldoth)
{
    C3 f0d = c3(0.08f * m.specular, 0.08f * m.specular, 0.08f * m.specular);
    C3 f0 = lerp(m.metal, f0d, base);
    return f0 + (c3(1.0f, 1.0f, 1.0f) - f0) * schlick5(ldoth);
}
FR_HD float smith_v(float alpha_sq, float ndotv, float ndotl)
{
    float a = ndotv * ndotv;
    float b = ndotl * ndotl;
    float v1 = 1.0f / (ndotv + sqrtf(alpha_sq + a - alpha_sq * a));
    float v2 = 1.0f / (ndotl + sqrtf(alpha_sq + b - alpha_sq * b));
    return v1 * v2;
}
FR_HD C3 diffuse_term(const Mat& m, C3 base, float ndotl, float ndotv, float ldoth)
{
    float FL = schlick5(ndotl);
    float FV = schlick5(ndotv);
    float RR = 2 * m.roughness * ldoth * ldoth;
    float s = (1.0f - 0.5f * FL) * (1.0f - 0.5f * FV) + RR * (FL + FV + FL * FV * (RR - 1.0f));
    return c_div_recip(base, PI_F) * s;
}

// Material::brdf (Material.h:67-122)
FR_HD C3 brdf(const Mat& m, V3 l, V3 v, V3 n, C3 sc)
{
    float ndotv = dot(n, v);
    if (ndotv <= 0)
        return c3(0, 0, 0);
    V3 hh = l + v;
    V3 h = div_each(hh, sqrtf(dot(hh, hh)));
    float ndotl = dot(n, l);
    float ldoth = dot(l, h);
    float ndoth = dot(n, h);
    C3 base = base_color(m, sc);
    C3 f_d = diffuse_term(m, base, ndotl, ndotv, ldoth);
    float alpha = m.roughness * m.roughness;
    float alpha_sq = alpha * alpha;
    float D = ggx_d(alpha_sq, ndoth);
    C3 F = fresnel_term(m, base, ldoth);
    float V = smith_v(alpha_sq, ndotv, ndotl);
    C3 f_s = D * F * V;
    return f_d * (1.0f - m.metal) + f_s;
}

// Material::brdf_diffuse (Material.h:124-151)
FR_HD C3 brdf_diffuse(const Mat& m, V3 l, V3 v, V3 n, C3 sc)
{
    float ndotv = dot(n, v);
    if (ndotv <= 0 || m.metal == 1.0f)
        return c3(0, 0, 0);
    V3 hh = l + v;
    V3 h = div_each(hh, sqrtf(dot(hh, hh)));
    float ndotl = dot(n, l);
    float ldoth = dot(l, h);
    return diffuse_term(m, base_color(m, sc), ndotl, ndotv, ldoth) * (1.0f - m.metal);
}

// Material::brdf_specular (Material.h:153-218)
FR_HD C3 brdf_specular(const Mat& m, V3 l, V3 v, V3 n, C3 sc, float half_angle)
{
    float ndotv = dot(n, v);
    if (ndotv <= 0)
        return c3(0, 0, 0);
    V3 hh = l + v;
    V3 h = div_each(hh, sqrtf(dot(hh, hh)));
    float ndotl = dot(n, l);
    float ldoth = dot(l, h);
    float ndoth = dot(n, h);
    C3 base = base_color(m, sc);
    float alpha = m.roughness * m.roughness;
    float alpha_sq = alpha * alpha;
    float D = ggx_d(alpha_sq, ndoth);
    if (half_angle > 0.99f * PI_F / 2.0f)
        half_angle = 0.99f * PI_F / 2.0f;
    if (half_angle > 0.0f) {
        float ap = alpha + 0.5f * htan(half_angle);
        if (ap > 1.0f)
            ap = 1.0f;
        D = D * alpha_sq / (ap * ap);
    }
    C3 F = fresnel_term(m, base, ldoth);
    float V = smith_v(alpha_sq, ndotv, ndotl);
    return D * F * V;
}

// tangent frame of the importance samplers; `fabs(float) > 0.999` compares in double
FR_HD void tangent_frame(V3 n, V3& tx, V3& ty)
{
    V3 up = v3(0, 0, 1.0f);
    if (double(fabsf(n.z)) > 0.999)
        up = v3(1.0f, 0, 0);
    tx = cross(up, n);
    tx = div_recip(tx, sqrtf(dot(tx, tx)));
    ty = cross(n, tx);
}

FR_HD float pdf_ggx(const Mat& m, V3 l, V3 v, V3 n)  // Material.h:258-280
{
    V3 hh = l + v;
    V3 h = div_each(hh, sqrtf(dot(hh, hh)));
    float ldoth = dot(l, h);
    float ndoth = dot(n, h);
    float alpha = m.roughness * m.roughness;
    float alpha_sq = alpha * alpha;
    float D = ggx_d(alpha_sq, ndoth);
    float pdf = D * ndoth / (4.0f * ldoth);
    return (pdf > 0.0f) ? pdf : 0.0f;
}

FR_HD float pdf_diffuse(V3 l, V3 n)  // Material.h:306-313
{
    float ndotl = dot(n, l);
    return (ndotl > 0.0f) ? ndotl / PI_F : 0.0f;
}

// --------------------------------------------------------------------------------------------
// lights in scene space (fresnel/common/Light.h:47-66)
// --------------------------------------------------------------------------------------------
struct LightsK {
    V3 dir[4];
    C3 color[4];
    float theta[4];
    float cos_theta[4];  // cos(theta), the cone test's threshold (taken before the clamp)
    float sin_half[4];   // sin(min(theta, pi/2)), the normalisation of the light's radiance
    uint32_t n;
};

// --------------------------------------------------------------------------------------------
// path tracing (fresnel/common/RayGen.h:110-186, TracerPathMethods.h:36-168)
// --------------------------------------------------------------------------------------------
// MISReflectionTransmission: returns the next direction; factor only changes on reflection.
FR_HD V3 mis_direction(float& factor, bool& transmit, V3 v, V3 n, uint32_t depth, uint32_t sample,
                       uint32_t key0, uint32_t key1, const Mat& m)
{
    U4 r = philox(0u, depth, sample, TAG_MIS, key0, key1);
    float xi0 = u01(r.x), xi1 = u01(r.y);
    float choice_mis = u01(r.z), choice_trans = u01(r.w);
    transmit = (choice_trans <= m.spec_trans);
    if (transmit)
        return -v;
    // Both samplers (sample_diffuse, sample_ggx) build a vector (rho cos a, rho sin a, z) in the
    // tangent frame of n; only rho, a and z differ.  Those are chosen per branch and the rest is
    // shared, so that lanes of a warp that chose different samplers run the sin/cos, the frame
    // and both pdfs together (the same operations in the same order as the two samplers).
    const bool diffuse = choice_mis <= 0.5f;
    float rho, a, z;
    if (diffuse) {  // sample_diffuse (Material.h:282-304)
        rho = sqrtf(xi0);
        a = 2 * PI_F * xi1;
        z = sqrtf(1.0f - xi0);
    } else {  // sample_ggx (Material.h:230-256)
        float alpha = m.roughness * m.roughness;
        a = 2.0f * PI_F * xi0;
        z = sqrtf((1.0f - xi1) / (1.0f + (alpha * alpha - 1.0f) * xi1));
        rho = sqrtf(1.0f - z * z);
    }
    float sa, ca;
    hsincos(a, sa, ca);
    const V3 vt = v3(rho * ca, rho * sa, z);
    V3 tx, ty;
    tangent_frame(n, tx, ty);
    const V3 w = tx * vt.x + ty * vt.y + n * vt.z;
    const V3 l = diffuse ? w : 2.0f * dot(v, w) * w - v;
    float pd = pdf_diffuse(l, n);
    float pg = pdf_ggx(m, l, v, n);
    factor = diffuse ? (pd / (pd + pg)) / (0.5f * pd) : (pg / (pd + pg)) / (0.5f * pg);
    return l;
}

// shouldTerminatePath
FR_HD bool russian_roulette(C3& att, uint32_t depth, uint32_t sample, uint32_t key0, uint32_t key1)
{
    U4 r = philox(0u, depth, sample, TAG_RR, key0, key1);
    float p = fmaxf(att.r, fmaxf(att.g, att.b));
    p = fminf(p, 1.0f);
    if (u01(r.x) > p)
        return true;
    att = c_div_each(att, p);
    return false;
}

// Per-path state (PRDpath, TracerPathMethods.h:24-34) without the fields the wavefront keeps
// elsewhere (the light-sample index and the alpha, which only a primary miss changes).
struct PathS {
    C3 result;
    C3 att;
    V3 origin, dir;
    uint32_t depth;
    bool done;
};

// path_tracer_miss for depth > 0 (TracerPathMethods.h:55-74); depth 0 is handled by the caller.
FR_HD void path_miss_lights(PathS& s, const LightsK& L, V3 ray_dir)
{
    for (uint32_t i = 0; i < L.n; ++i) {
        V3 l = L.dir[i];
        const float cos_half = L.cos_theta[i];
        float ldotd = dot(l, ray_dir);
        if (ldotd >= cos_half)
            s.result = s.result + c_div_recip(s.att * L.color[i], L.sin_half[i]);
    }
    s.done = true;
}

// path_tracer_hit (TracerPathMethods.h:79-168)
FR_HD void path_hit(PathS& s, const Mat& material, const Mat& outline, float shading_distance,
                    float outline_width, C3 shading_color, V3 shading_normal, V3 ray_o, V3 ray_d,
                    float t_hit, uint32_t key0, uint32_t key1, uint32_t sample)
{
    const Mat& m = (shading_distance >= outline_width) ? material : outline;
    V3 n = shading_normal * (1.0f / sqrtf(dot(shading_normal, shading_normal)));
    V3 v = -ray_d;
    if (is_solid(m)) {
        s.result = s.result + s.att * base_color(m, shading_color);
        s.done = true;
        return;
    }
    float factor = 1.0f;
    bool transmit = false;
    V3 l = mis_direction(factor, transmit, v, n, s.depth, sample, key0, key1, m);
    if (transmit) {
        C3 tc = base_color(m, shading_color);
        tc.r = sqrtf(tc.r);
        tc.g = sqrtf(tc.g);
        tc.b = sqrtf(tc.b);
        s.att = s.att * tc;
    } else {
        float ndotl = dot(n, l);
        if (dot(n, v) > 0.0f && ndotl > 0.0f) {
            s.att = s.att * (brdf(m, l, v, n, shading_color) * ndotl * factor);
        } else {
            s.att = c3(0, 0, 0);
            s.done = true;
        }
    }
    s.origin = ray_o + ray_d * t_hit;
    s.dir = l;
    if (russian_roulette(s.att, s.depth, sample, key0, key1))
        s.done = true;
}

// Camera constants for one render (Camera::Camera, Camera.h:129-157).
FR_HD CamK make_camera(V3 position, V3 look_at, V3 up, float h, float f, float f_stop,
                       float focus_distance, int model, uint32_t width, uint32_t height,
                       uint32_t seed, bool sample_aa)
{
    CamK k;
    k.p = position;
    camera_basis(position, look_at, up, k.u, k.v, k.w);
    k.focal_d = focus_distance;
    k.aperture = f / f_stop;
    k.model = model;
    k.width = width;
    k.height = height;
    k.seed = seed;
    k.sample_aa = sample_aa ? 1 : 0;
    k.focal_h = (model == 0) ? h : h / f * k.focal_d;
    return k;
}

// Lights::Lights(lights, cam) (Light.h:47-66): normalise, then camera space -> scene space.
FR_HD LightsK lights_to_world(const V3* dir_cam, const C3* color, const float* theta, uint32_t n,
                              const CamK& k)
{
    LightsK L;
    L.n = n;
    for (uint32_t i = 0; i < 4; ++i) {
        L.dir[i] = v3(0, 0, 0);
        L.color[i] = c3(0, 0, 0);
        L.theta[i] = 0.0f;
        L.cos_theta[i] = 1.0f;
        L.sin_half[i] = 0.0f;
    }
    for (uint32_t i = 0; i < n; ++i) {
        L.color[i] = color[i];
        V3 v = dir_cam[i];
        v = v * (1.0f / sqrtf(dot(v, v)));
        L.dir[i] = v.x * k.u + v.y * k.v + v.z * k.w;
        L.theta[i] = theta[i];
        // the miss program's per-light constants (TracerPathMethods.h:57-61), once per frame
        // instead of per escaping ray; on the host, with the C library's cosf/sinf
        L.cos_theta[i] = hcos(theta[i]);
        const float half = theta[i] > PI_F / 2.0f ? PI_F / 2.0f : theta[i];
        L.sin_half[i] = hsin(half);
    }
    return L;
}

// --------------------------------------------------------------------------------------------
// intersectors
// --------------------------------------------------------------------------------------------
constexpr float SPHERE_EPS = 1e-4f;

// t of intersect_ray_sphere (IntersectSphere.h:36-85) without the outputs only shading needs.
FR_HD bool sphere_t(V3 o, V3 d, V3 p, float r, float& t)
{
    V3 v = p - o;
    float b = dot(v, d);
    float det = b * b - dot(v, v) + r * r;
    if (det < 0)
        return false;
    det = sqrtf(det);
    t = b - det;
    if (t > SPHERE_EPS)
        return true;
    t = b + det;
    return t > SPHERE_EPS;
}

FR_HD bool isect_sphere(float& t, float& d_edge, V3& N, V3 o, V3 d, V3 p, float r)
{
    V3 v = p - o;
    float b = dot(v, d);
    float det = b * b - dot(v, v) + r * r;
    if (det < 0)
        return false;
    V3 w = cross(v, d);
    float Dsq = dot(w, w);
    d_edge = r - sqrtf(Dsq);
    det = sqrtf(det);
    t = b - det;
    if (t > SPHERE_EPS) {
        N = o + t * d - p;
        return true;
    }
    t = b + det;
    if (t > SPHERE_EPS) {
        N = -(o + t * d - p);
        return true;
    }
    return false;
}

// intersect_ray_cylinder (IntersectCylinder.h:35-113)
FR_HD bool isect_cylinder(float& t, V3& N, V3 o, V3 d, V3 A, V3 B, float r)
{
    const float eps = 1e-4f;
    const V3 Oa = o - A;
    const V3 C = B - A;
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
    V3 P = v3(0, 0, 0);
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
FR_HD bool isect_spherocylinder(float& t, float& d_edge, V3& N, uint32_t& color_index, V3 o, V3 d,
                                V3 A, V3 B, float r)
{
    t = HUGE_VALF;
    float t_sc = 0, de_sc = HUGE_VALF;
    V3 N_sc = v3(0, 0, 0);
    const V3 Oa = o - A;
    const V3 C = B - A;
    const float cdotc = dot(C, C);
    bool hit_cyl = isect_cylinder(t_sc, N_sc, o, d, A, B, r);
    if (hit_cyl && t_sc < t) {
        t = t_sc;
        N = N_sc;
    }
    bool hit_A = isect_sphere(t_sc, de_sc, N_sc, o, d, A, r);
    if (hit_A && (t_sc < t)) {
        const V3 PA = Oa + t_sc * d;
        if (dot(PA, C) <= 0) {
            t = t_sc;
            N = N_sc;
        } else {
            hit_A = false;
        }
    }
    bool hit_B = isect_sphere(t_sc, de_sc, N_sc, o, d, B, r);
    if (hit_B && (t_sc < t)) {
        const V3 PA = Oa + t_sc * d;
        if (dot(PA, C) >= cdotc) {
            t = t_sc;
            N = N_sc;
        } else {
            hit_B = false;
        }
    }
    const V3 P = Oa + t * d;
    const float pdotc = dot(P, C);
    color_index = (pdotc < cdotc / 2.0f) ? 0u : 1u;
    const V3 C_vp = C - dot(C, d) * d;
    const V3 Oa_vp = Oa - dot(Oa, d) * d;
    const float oc = dot(Oa_vp, C_vp);
    const float cc = dot(C_vp, C_vp);
    if (oc < 0) {
        d_edge = r - sqrtf(dot(Oa_vp, Oa_vp));
    } else if (oc > cc) {
        V3 e = Oa_vp - C_vp;
        d_edge = r - sqrtf(dot(e, e));
    } else {
        const V3 n_vp = Oa_vp - oc / cc * C_vp;
        d_edge = r - sqrtf(dot(n_vp, n_vp));
    }
    return hit_A || hit_B || hit_cyl;
}

// intersect_ray_triangle (IntersectTriangle.h:43-132)
FR_HD bool isect_triangle(float& u, float& v, float& w, float& t, float& d_edge, V3& n, V3 p, V3 q,
                          V3 a, V3 b, V3 c)
{
    V3 ab = b - a;
    V3 ac = c - a;
    V3 qp = p - q;
    n = cross(ab, ac);
    float d = dot(qp, n);
    if (d <= 0.0f)
        return false;
    V3 ap = p - a;
    t = dot(ap, n);
    if (t < 0.0f)
        return false;
    V3 e = cross(qp, ap);
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
    V3 edge, pt;
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
    V3 r_hit = p + t * (q - p);
    V3 vec = cross(edge, r_hit - pt);
    float dsq = dot(vec, vec) / dot(edge, edge);
    d_edge = sqrtf(dsq);
    return true;
}

// --------------------------------------------------------------------------------------------
// sRGB (fresnel/common/ColorMath.h:506-546)
// --------------------------------------------------------------------------------------------
FR_HD uint32_t srgb_pack(float r, float g, float b, float a)
{
    float x[3] = {r, g, b};
    uint32_t out = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float y = (x[k] < 0.0031308f) ? 12.92f * x[k]
                                      : (1.0f + 0.055f) * hpow(x[k], 1.0f / 2.4f) - 0.055f;
        if (y > 1.0f)
            y = 1.0f;
        out |= uint32_t((unsigned char)(y * 255.0f + 0.5f)) << (8 * k);
    }
    out |= uint32_t((unsigned char)(a * 255.0f + 0.5f)) << 24;
    return out;
}

}  // namespace fr

#endif
