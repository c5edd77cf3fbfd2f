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

// Work items of the primary pass: T x T-pixel tiles in row-major order (T = 2^tl, 8 by
// default), a tile's pixels in row-major order, and the K samples of a pixel innermost. A warp
// then traces two pixels' 16 samples (K = 16) or an 8x4 block of pixels (K = 1, T = 8): its
// rays start close together and point the same way, which keeps the warp's traversal steps and
// node loads shared. The path state is laid out in the same order: the slot of a render's item
// g is g itself, so the primary pass writes whole cache lines, and the queues it fills start
// out in slot order. Slots of pixels outside the image (edge tiles) stay unused.
struct PrimaryItem {
    uint32_t i, j, k;
    bool valid;
};

__host__ __device__ __forceinline__ uint32_t primary_tiles_x(uint32_t w, uint32_t tl)
{
    return (w + (1u << tl) - 1u) >> tl;
}

__host__ __device__ __forceinline__ uint32_t primary_items(uint32_t w, uint32_t h, uint32_t K,
                                                           uint32_t tl)
{
    return primary_tiles_x(w, tl) * primary_tiles_x(h, tl) * (1u << (2u * tl)) * K;
}

// Slot of sample 0 of pixel (i, j); its K samples follow it.
__device__ __forceinline__ uint32_t pixel_slot(uint32_t i, uint32_t j, uint32_t w, uint32_t K,
                                               uint32_t tl)
{
    const uint32_t m = (1u << tl) - 1u;
    return ((((j >> tl) * primary_tiles_x(w, tl) + (i >> tl)) << (2u * tl)) + ((j & m) << tl) +
            (i & m)) * K;
}

__device__ __forceinline__ PrimaryItem primary_item(uint32_t g, uint32_t w, uint32_t h, uint32_t K,
                                                    uint32_t tl)
{
    const uint32_t per_tile = (1u << (2u * tl)) * K;
    const uint32_t tile = g / per_tile;
    const uint32_t r = g - tile * per_tile;
    const uint32_t px = r / K;
    const uint32_t tiles_x = primary_tiles_x(w, tl);
    const uint32_t ty = tile / tiles_x;
    const uint32_t tx = tile - ty * tiles_x;
    const uint32_t m = (1u << tl) - 1u;
    PrimaryItem it;
    it.k = r - px * K;
    it.i = (tx << tl) + (px & m);
    it.j = (ty << tl) + (px >> tl);
    it.valid = it.i < w && it.j < h;
    return it;
}

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

// The shading loop of one slot from its current state (TracerPath's hit/miss programs,
// fresnel/common/TracerPathMethods.h:36-168, light samples in order): shade the vertex, then
// either store the continuing path (returns true: it needs another closest hit) or restart the
// next light sample from the cached primary hit, or store the finished pixel sample (returns
// false).  FIRST_IN_REGS: the first vertex's ray (ro0, rd0) and hit (h0) come from the
// caller's registers instead of the path state.  A light sample that ends at the primary vertex
// (an outline or solid hit, a killed or terminated path) hands the next one the same ray, hit
// and surface: those are kept in registers, not reloaded and recomputed.
template <bool FIRST_IN_REGS>
__device__ __forceinline__ bool shade_core(const FrameParams& P, const PathState& S, uint32_t p,
                                           uint32_t pixel, uint32_t n_samples, uint32_t ls,
                                           PathS s, uint2 ph, V3 ro0, V3 rd0, uint2 h0)
{
    const uint32_t key1 = P.cam.seed;
    V3 ro, rd;
    uint2 h;
    if (FIRST_IN_REGS) {
        ro = ro0;
        rd = rd0;
        h = h0;
    } else if (s.depth == 0) {
        ro = xyz(S.prim_o[p]);
        rd = xyz(S.prim_d[p]);
        h = ph;
    } else {
        ro = xyz(S.ray_o[p]);
        rd = xyz(S.ray_d[p]);
        h = S.hit[p];
    }
    Surface sf;
    bool have_sf = false;  // sf holds the surface of (ro, rd, h)
    while (true) {
        s.done = false;
        if (h.x != MISS) {
            const GeomDev& g = P.scene.geoms[h.x];
            if (!have_sf)
                sf = hit_surface(g, h.y, ro, rd, PATH_TNEAR);
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
            if (s.depth == 0) {  // the next light sample starts from this same vertex
                have_sf = true;
            } else {
                ro = xyz(S.prim_o[p]);
                rd = xyz(S.prim_d[p]);
                h = ph;
                have_sf = false;
            }
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

// Shade the current path vertex of one slot; returns true if the path needs another closest hit.
// p indexes the path state; local = k * w * h + pixel numbers the slot within its render (equal
// to p for a single render, p minus the render's first slot in a batch of renders).
__device__ __forceinline__ bool shade_pixel(const FrameParams& P, const PathState& S, uint32_t p,
                                            uint32_t local)
{
    const PrimaryItem pi = primary_item(local, P.w, P.h, P.batch, P.tile_log2);
    const uint32_t pixel = pi.j * P.w + pi.i;
    const uint32_t n_samples = P.n_samples + pi.k;
    const uint2 ld = S.ls_depth[p];
    PathS s;
    s.depth = ld.y;
    if (ld.x == 0u && s.depth == 0u) {  // a fresh primary hit (primary_finish)
        s.result = c3(0.0f, 0.0f, 0.0f);
        s.att = c3(1.0f, 1.0f, 1.0f);
    } else {
        s.result = rgb3(S.result[p]);
        s.att = rgb3(S.att[p]);
    }
    s.origin = v3(0, 0, 0);
    s.dir = v3(0, 0, 0);
    return shade_core<false>(P, S, p, pixel, n_samples, ld.x, s, S.prim_hit[p], v3(0, 0, 0),
                             v3(0, 0, 0), make_uint2(0u, 0u));
}

// Primary ray of one item: closest hit; a miss finishes its pixel sample (every light sample
// sees the background: radiance bg * L, fresnel/common/TracerPathMethods.h:44-50), a hit
// stores the ray and starts the path: (light sample, depth) = (0, 0), which tells the shade
// pass that the throughput is 1 and the radiance 0 (not stored).  Returns true for a hit (the
// slot is queued for shading).
__device__ __forceinline__ bool primary_finish(const FrameParams& P, const PathState& S,
                                               uint32_t slot, V3 o, V3 d, Hit h)
{
    S.prim_hit[slot] = make_uint2(h.geom, h.prim);
    if (h.geom == MISS) {
        C3 res = P.bg * float(P.light_samples);
        C3 out = c_div_recip(res, float(P.light_samples));
        S.sample[slot] = make_float4(out.r, out.g, out.b, P.bg_alpha);
        return false;
    }
    S.prim_o[slot] = f4(o);
    S.prim_d[slot] = f4(d);
    S.ls_depth[slot] = make_uint2(0u, 0u);
    return true;
}

template <int WIDTH, uint32_t MASK>
__device__ __forceinline__ bool primary_ray(const FrameParams& P, const PathState& S,
                                            const PrimaryItem& it, uint32_t slot, TraceCount& tc)
{
    V3 o, d;
    camera_ray(P.cam, it.i, it.j, P.n_samples + it.k, o, d);
    Hit h = trace_closest<WIDTH, MASK>(P.scene, o, d, PATH_TNEAR, tc);
    return primary_finish(P, S, slot, o, d, h);
}

// Primary ray of one item shaded at once (the first shade pass folded into the primary pass): a
// miss finishes its pixel sample as in primary_finish; a hit is shaded from registers, without
// storing the primary ray (unless a later light sample restarts from it) or reading anything
// back.  Returns true when the path continues (its extension ray is stored; queue it).
template <int WIDTH, uint32_t MASK>
__device__ __forceinline__ bool primary_shade(const FrameParams& P, const PathState& S,
                                              const PrimaryItem& it, uint32_t slot, TraceCount& tc)
{
    V3 o, d;
    camera_ray(P.cam, it.i, it.j, P.n_samples + it.k, o, d);
    Hit h = trace_closest<WIDTH, MASK>(P.scene, o, d, PATH_TNEAR, tc);
    const uint2 ph = make_uint2(h.geom, h.prim);
    S.prim_hit[slot] = ph;
    if (h.geom == MISS) {
        C3 res = P.bg * float(P.light_samples);
        C3 out = c_div_recip(res, float(P.light_samples));
        S.sample[slot] = make_float4(out.r, out.g, out.b, P.bg_alpha);
        return false;
    }
    if (P.light_samples > 1u) {  // later light samples restart from the primary ray
        S.prim_o[slot] = f4(o);
        S.prim_d[slot] = f4(d);
    }
    PathS s;
    s.result = c3(0.0f, 0.0f, 0.0f);
    s.att = c3(1.0f, 1.0f, 1.0f);
    s.depth = 0;
    s.origin = v3(0, 0, 0);
    s.dir = v3(0, 0, 0);
    return shade_core<true>(P, S, slot, it.j * P.w + it.i, P.n_samples + it.k, 0u, s, ph, o, d,
                            ph);
}

// Extension ray of slot p traced and its hit shaded at once (a bounce): the path state is read as
// the shade pass reads it, with the ray and the hit from registers.  local numbers the slot
// within its render (as for shade_pixel).  Returns true when the path continues (its next
// extension ray is stored; queue it).
template <int WIDTH, uint32_t MASK>
__device__ __forceinline__ bool bounce(const FrameParams& P, const PathState& S, uint32_t p,
                                       uint32_t local, TraceCount& tc)
{
    const V3 o = xyz(S.ray_o[p]);
    const V3 d = xyz(S.ray_d[p]);
    const Hit hit = trace_closest<WIDTH, MASK>(P.scene, o, d, PATH_TNEAR, tc);
    const PrimaryItem pi = primary_item(local, P.w, P.h, P.batch, P.tile_log2);
    const uint2 ld = S.ls_depth[p];
    PathS s;
    s.depth = ld.y;
    s.result = rgb3(S.result[p]);
    s.att = rgb3(S.att[p]);
    s.origin = v3(0, 0, 0);
    s.dir = v3(0, 0, 0);
    return shade_core<true>(P, S, p, pi.j * P.w + pi.i, P.n_samples + pi.k, ld.x, s,
                            S.prim_hit[p], o, d, make_uint2(hit.geom, hit.prim));
}

// Append the lanes with push set to queue q (one atomic per warp).
__device__ __forceinline__ void push_queue(const PathState& S, int q, bool push, uint32_t slot)
{
    const uint32_t lane = lane_id();
    const uint32_t m = __ballot_sync(0xffffffffu, push);
    if (m) {
        uint32_t at = 0;
        if (lane == 0)
            at = atomicAdd(S.ctr + q, uint32_t(__popc(m)));
        at = __shfl_sync(0xffffffffu, at, 0);
        if (push)
            S.queue[q][at + __popc(m & ((1u << lane) - 1u))] = slot;
    }
}

// Append the lanes with push set to queue 1 (one atomic per warp).
__device__ __forceinline__ void push_primary(const PathState& S, bool push, uint32_t slot)
{
    const uint32_t lane = lane_id();
    const uint32_t m = __ballot_sync(0xffffffffu, push);
    if (m) {
        uint32_t at = 0;
        if (lane == 0)
            at = atomicAdd(S.ctr + 1, uint32_t(__popc(m)));
        at = __shfl_sync(0xffffffffu, at, 0);
        if (push)
            S.queue[1][at + __popc(m & ((1u << lane) - 1u))] = slot;
    }
}

}  // namespace
}  // namespace fr

#endif
