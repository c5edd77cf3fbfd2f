// path_device.cuh -- device-side pieces shared by the single-render and the batched path
// tracer kernels: output writes, the Welford fold and the shading of one path vertex.
#ifndef FR_PATH_DEVICE_CUH
#define FR_PATH_DEVICE_CUH

#include "render.hpp"

namespace fr {
namespace {

constexpr float PATH_TNEAR = 1e-3f;  // fresnel/cpu/TracerPath.cc:121,167

__device__ __forceinline__ V3 xyz(float4 a) { return v3(a.x, a.y, a.z); }
__device__ __forceinline__ float4 f4(V3 a) { return make_float4(a.x, a.y, a.z, 0.0f); }
__device__ __forceinline__ float4 f4(C3 a) { return make_float4(a.r, a.g, a.b, 0.0f); }
__device__ __forceinline__ C3 rgb3(float4 a) { return c3(a.x, a.y, a.z); }

__device__ __forceinline__ void write_pixel(const FrameParams& P, uint32_t p, float r, float g,
                                            float b, float a)
{
    P.linear[p] = make_float4(r, g, b, a);
    if (!P.highlight || (r <= 1.0f && g <= 1.0f && b <= 1.0f))
        P.srgb[p] = srgb_pack(r, g, b, a);
    else
        P.srgb[p] = srgb_pack(P.hl_color.r, P.hl_color.g, P.hl_color.b, a);
}

// Welford update of one pixel with one sample (fresnel/cpu/TracerPath.cc:228-250), dropping
// non-finite samples as the GPU backend does (fresnel/gpu/path.cu:111-113).
__device__ __forceinline__ float4 welford(const FrameParams& P, float4 old, float4 x, uint32_t n)
{
    float q = 1.0f / float(n);
    float nr = old.x + (x.x - old.x) * q;
    float ng = old.y + (x.y - old.y) * q;
    float nb = old.z + (x.z - old.z) * q;
    float na = old.w + (x.w - old.w) * q;
    if (!(isfinite(nr) && isfinite(ng) && isfinite(nb))) {
        atomicAdd(P.stats + 2, 1ull);
        return old;
    }
    return make_float4(nr, ng, nb, na);
}

// Shade the current path vertex of one slot; returns true if the path needs another closest hit.
// p indexes the path state; local = k * w * h + pixel numbers the slot within its render (equal
// to p for a single render, p minus the render's first slot in a batch of renders).
__device__ __forceinline__ bool shade_pixel(const FrameParams& P, const PathState& S, uint32_t p,
                                            uint32_t local)
{
    const uint32_t wh = P.w * P.h;
    const uint32_t k = local / wh;
    const uint32_t pixel = local - k * wh;
    const uint32_t n_samples = P.n_samples + k;
    uint2 ld = S.ls_depth[p];
    uint32_t ls = ld.x;
    PathS s;
    s.result = rgb3(S.result[p]);
    s.att = rgb3(S.att[p]);
    s.depth = ld.y;
    s.origin = v3(0, 0, 0);
    s.dir = v3(0, 0, 0);
    const uint2 ph = S.prim_hit[p];
    const uint32_t key1 = P.cam.seed;
    while (true) {
        V3 ro, rd;
        uint2 h;
        if (s.depth == 0) {
            ro = xyz(S.prim_o[p]);
            rd = xyz(S.prim_d[p]);
            h = ph;
        } else {
            ro = xyz(S.ray_o[p]);
            rd = xyz(S.ray_d[p]);
            h = S.hit[p];
        }
        s.done = false;
        if (h.x != MISS) {
            const GeomDev& g = P.scene.geoms[h.x];
            Surface sf = hit_surface(g, h.y, ro, rd, PATH_TNEAR);
            uint32_t sample = (n_samples - 1u) * P.light_samples + ls;
            path_hit(s, g.material, g.outline, sf.d_edge, g.outline_width, sf.color, sf.Ng, ro, rd,
                     sf.t, pixel, key1, sample);
        } else if (s.depth == 0) {
            // a primary miss shows the background (fresnel/common/TracerPathMethods.h:44-50)
            s.result = P.bg * float(P.light_samples);
            s.done = true;
        } else {
            path_miss_lights(s, P.lights, rd);
        }
        if (!s.done) {
            s.depth += 1u;
            S.ray_o[p] = f4(s.origin);
            S.ray_d[p] = f4(s.dir);
            S.att[p] = f4(s.att);
            S.result[p] = f4(s.result);
            S.ls_depth[p] = make_uint2(ls, s.depth);
            return true;
        }
        if (ls + 1u < P.light_samples) {
            ++ls;
            s.depth = 0;
            s.att = c3(1.0f, 1.0f, 1.0f);
            continue;
        }
        // the pixel sample (fresnel/cpu/TracerPath.cc:228): radiance / L, alpha
        C3 out = c_div_recip(s.result, float(P.light_samples));
        S.sample[p] = make_float4(out.r, out.g, out.b, ph.x == MISS ? P.bg_alpha : 1.0f);
        return false;
    }
}

}  // namespace
}  // namespace fr

#endif
