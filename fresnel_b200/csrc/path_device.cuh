// path_device.cuh -- device-side pieces shared by the single-render and the batched path
// tracer kernels: output writes, the Welford fold and the shading of one path vertex.
#ifndef FR_PATH_DEVICE_CUH
#define FR_PATH_DEVICE_CUH

#include "render.hpp"

namespace fr {
namespace {

constexpr float PATH_TNEAR = 1e-3f;  // fresnel/cpu/TracerPath.cc:121,167

// Bound on the bounces a tail kernel follows one path for (never reached: Russian roulette ends
// paths long before); a path cut there sets ERR_ITERATION_CAP.
constexpr uint32_t TAIL_MAX_DEPTH = 1u << 16;

__device__ __forceinline__ V3 xyz(float4 a) { return v3(a.x, a.y, a.z); }
__device__ __forceinline__ float4 f4(V3 a) { return make_float4(a.x, a.y, a.z, 0.0f); }
__device__ __forceinline__ float4 f4(C3 a) { return make_float4(a.r, a.g, a.b, 0.0f); }
__device__ __forceinline__ C3 rgb3(float4 a) { return c3(a.x, a.y, a.z); }

// Path-state and queue accesses are streamed: each slot's values are read and written once per
// pass, and the wavefront (gigabytes) is far larger than L2, so they are loaded and stored with
// the evict-first (.cs) policy, which leaves L2 to the scene and its acceleration structure.
template <class T>
__device__ __forceinline__ T ld_cs(const T* a)
{
    return __ldcs(a);
}
template <class T>
__device__ __forceinline__ void st_cs(T* a, T v)
{
    __stcs(a, v);
}

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

// One slot being shaded: its path state in registers, with the vertex to shade next (the ray
// ro, rd and its hit h).  sf caches the surface of that vertex once computed (have_sf): a light
// sample that ends at the primary vertex (an outline or solid hit, a killed or terminated path)
// hands the next one the same ray, hit and surface, which are then neither reloaded nor
// recomputed.
struct ShadeLane {
    uint32_t p;          // path-state slot
    uint32_t pixel;      // j * w + i
    uint32_t n_samples;  // 1-based sample number of the slot's pixel sample
    uint32_t ls;         // light sample
    PathS s;
    uint2 ph;            // primary hit
    uint2 h;             // hit of the vertex to shade
    V3 ro, rd;           // its ray
    Surface sf;
    bool have_sf;
};

// Outcome of one shade_step.
enum ShadeStep : int {
    STEP_CONTINUE = 0,  // the path continues: its extension ray is stored, queue the slot
    STEP_FINISHED = 1,  // the pixel sample is stored in S.sample
    STEP_RESTART = 2    // the light sample ended; the lane now holds the next one's first vertex
};

// The lane state of slot p from the path state (the shade pass's view of a queued slot); local
// numbers the slot within its render (equal to p for a single render, p minus the render's
// first slot in a batch of renders).  A fresh primary hit, (light sample, depth) = (0, 0), has
// throughput 1 and radiance 0, which are not stored.
__device__ __forceinline__ void shade_load(const FrameParams& P, const PathState& S, uint32_t p,
                                           uint32_t local, ShadeLane& L)
{
    const PrimaryItem pi = primary_item(local, P.w, P.h, P.batch, P.tile_log2);
    L.p = p;
    L.pixel = pi.j * P.w + pi.i;
    L.n_samples = P.n_samples + pi.k;
    const uint2 ld = ld_cs(S.ls_depth + (p));
    L.ls = ld.x;
    L.s.depth = ld.y;
    if (ld.x == 0u && ld.y == 0u) {
        L.s.result = c3(0.0f, 0.0f, 0.0f);
        L.s.att = c3(1.0f, 1.0f, 1.0f);
    } else {
        L.s.result = rgb3(ld_cs(S.result + (p)));
        L.s.att = rgb3(ld_cs(S.att + (p)));
    }
    L.s.origin = v3(0, 0, 0);
    L.s.dir = v3(0, 0, 0);
    L.ph = ld_cs(S.prim_hit + (p));
    if (ld.y == 0u) {
        L.ro = xyz(ld_cs(S.prim_o + (p)));
        L.rd = xyz(ld_cs(S.prim_d + (p)));
        L.h = L.ph;
    } else {
        L.ro = xyz(ld_cs(S.ray_o + (p)));
        L.rd = xyz(ld_cs(S.ray_d + (p)));
        L.h = ld_cs(S.hit + (p));
    }
    L.have_sf = false;
}

// Shade the lane's current vertex (TracerPath's hit/miss programs,
// fresnel/common/TracerPathMethods.h:36-168, light samples in order), then store the continuing
// path, or move to the next light sample from the cached primary hit, or store the finished
// pixel sample (fresnel/cpu/TracerPath.cc:228: radiance / L, alpha).
__device__ __forceinline__ ShadeStep shade_step(const FrameParams& P, const PathState& S,
                                                ShadeLane& L)
{
    PathS& s = L.s;
    s.done = false;
    if (L.h.x != MISS) {
        const GeomDev& g = P.scene.geoms[L.h.x];
        if (!L.have_sf)
            L.sf = hit_surface(g, L.h.y, L.ro, L.rd, PATH_TNEAR);
        const uint32_t sample = (L.n_samples - 1u) * P.light_samples + L.ls;
        path_hit(s, g.material, g.outline, L.sf.d_edge, g.outline_width, L.sf.color, L.sf.Ng,
                 L.ro, L.rd, L.sf.t, L.pixel, P.cam.seed, sample);
    } else if (s.depth == 0) {
        // a primary miss shows the background (fresnel/common/TracerPathMethods.h:44-50)
        s.result = P.bg * float(P.light_samples);
        s.done = true;
    } else {
        path_miss_lights(s, P.lights, L.rd);
    }
    const uint32_t p = L.p;
    if (!s.done) {
        s.depth += 1u;
        st_cs(S.ray_o + (p), f4(s.origin));
        st_cs(S.ray_d + (p), f4(s.dir));
        st_cs(S.att + (p), f4(s.att));
        st_cs(S.result + (p), f4(s.result));
        st_cs(S.ls_depth + (p), make_uint2(L.ls, s.depth));
        return STEP_CONTINUE;
    }
    if (L.ls + 1u < P.light_samples) {
        ++L.ls;
        if (s.depth == 0) {  // the next light sample starts from this same vertex
            L.have_sf = true;
        } else {
            L.ro = xyz(ld_cs(S.prim_o + (p)));
            L.rd = xyz(ld_cs(S.prim_d + (p)));
            L.h = L.ph;
            L.have_sf = false;
        }
        s.depth = 0;
        s.att = c3(1.0f, 1.0f, 1.0f);
        return STEP_RESTART;
    }
    C3 out = c_div_recip(s.result, float(P.light_samples));
    st_cs(S.sample + (p), make_float4(out.r, out.g, out.b, L.ph.x == MISS ? P.bg_alpha : 1.0f));
    return STEP_FINISHED;
}

// Shade a lane until its path needs another closest hit (returns true) or its pixel sample is
// finished (returns false).
__device__ __forceinline__ bool shade_run(const FrameParams& P, const PathState& S, ShadeLane& L)
{
    while (true) {
        const ShadeStep r = shade_step(P, S, L);
        if (r != STEP_RESTART)
            return r == STEP_CONTINUE;
    }
}

// Shade the current path vertex of one slot; returns true if the path needs another closest hit.
// p indexes the path state; local = k * w * h + pixel numbers the slot within its render.
__device__ __forceinline__ bool shade_pixel(const FrameParams& P, const PathState& S, uint32_t p,
                                            uint32_t local)
{
    ShadeLane L;
    shade_load(P, S, p, local, L);
    return shade_run(P, S, L);
}

// Primary ray of one item: closest hit; a miss finishes its pixel sample (every light sample
// sees the background: radiance bg * L, fresnel/common/TracerPathMethods.h:44-50), a hit
// stores the ray and starts the path: (light sample, depth) = (0, 0), which tells the shade
// pass that the throughput is 1 and the radiance 0 (not stored).  Returns true for a hit (the
// slot is queued for shading).
__device__ __forceinline__ bool primary_finish(const FrameParams& P, const PathState& S,
                                               uint32_t slot, V3 o, V3 d, Hit h)
{
    st_cs(S.prim_hit + (slot), make_uint2(h.geom, h.prim));
    if (h.geom == MISS) {
        C3 res = P.bg * float(P.light_samples);
        C3 out = c_div_recip(res, float(P.light_samples));
        st_cs(S.sample + (slot), make_float4(out.r, out.g, out.b, P.bg_alpha));
        return false;
    }
    st_cs(S.prim_o + (slot), f4(o));
    st_cs(S.prim_d + (slot), f4(d));
    st_cs(S.ls_depth + (slot), make_uint2(0u, 0u));
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
    st_cs(S.prim_hit + (slot), ph);
    if (h.geom == MISS) {
        C3 res = P.bg * float(P.light_samples);
        C3 out = c_div_recip(res, float(P.light_samples));
        st_cs(S.sample + (slot), make_float4(out.r, out.g, out.b, P.bg_alpha));
        return false;
    }
    if (P.light_samples > 1u) {  // later light samples restart from the primary ray
        st_cs(S.prim_o + (slot), f4(o));
        st_cs(S.prim_d + (slot), f4(d));
    }
    ShadeLane L;
    L.p = slot;
    L.pixel = it.j * P.w + it.i;
    L.n_samples = P.n_samples + it.k;
    L.ls = 0;
    L.s.result = c3(0.0f, 0.0f, 0.0f);
    L.s.att = c3(1.0f, 1.0f, 1.0f);
    L.s.depth = 0;
    L.s.origin = v3(0, 0, 0);
    L.s.dir = v3(0, 0, 0);
    L.ph = ph;
    L.h = ph;
    L.ro = o;
    L.rd = d;
    L.have_sf = false;
    return shade_run(P, S, L);
}

// Extension ray of slot p traced and its hit shaded at once (a bounce): the path state is read as
// the shade pass reads it, with the ray and the hit from registers.  local numbers the slot
// within its render (as for shade_pixel).  Returns true when the path continues (its next
// extension ray is stored; queue it).
template <int WIDTH, uint32_t MASK>
__device__ __forceinline__ bool bounce(const FrameParams& P, const PathState& S, uint32_t p,
                                       uint32_t local, TraceCount& tc)
{
    const V3 o = xyz(ld_cs(S.ray_o + (p)));
    const V3 d = xyz(ld_cs(S.ray_d + (p)));
    const Hit hit = trace_closest<WIDTH, MASK>(P.scene, o, d, PATH_TNEAR, tc);
    const PrimaryItem pi = primary_item(local, P.w, P.h, P.batch, P.tile_log2);
    const uint2 ld = ld_cs(S.ls_depth + (p));
    ShadeLane L;
    L.p = p;
    L.pixel = pi.j * P.w + pi.i;
    L.n_samples = P.n_samples + pi.k;
    L.ls = ld.x;
    L.s.depth = ld.y;
    L.s.result = rgb3(ld_cs(S.result + (p)));
    L.s.att = rgb3(ld_cs(S.att + (p)));
    L.s.origin = v3(0, 0, 0);
    L.s.dir = v3(0, 0, 0);
    L.ph = ld_cs(S.prim_hit + (p));
    L.h = make_uint2(hit.geom, hit.prim);
    L.ro = o;
    L.rd = d;
    L.have_sf = false;
    return shade_run(P, S, L);
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
            st_cs(S.queue[q] + (at + __popc(m & ((1u << lane) - 1u))), slot);
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
            st_cs(S.queue[1] + (at + __popc(m & ((1u << lane) - 1u))), slot);
    }
}

}  // namespace
}  // namespace fr

#endif
