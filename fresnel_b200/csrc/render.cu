// render.cu -- wavefront path tracer and preview tracer kernels.
//
// Path tracer (replaces path_ray_gen/path_closest_hit/path_miss, fresnel/gpu/path.cu:70-171,
// with the CPU loop order of fresnel/cpu/TracerPath.cc:78-255).  A batch traces K samples of
// every pixel at once, one path slot per (pixel, sample):
//   primary  one thread per slot, the K samples of a pixel in neighbouring lanes: camera ray,
//            closest hit (shared by all light samples of the pixel sample, as the CPU path
//            caches it); a miss finishes its sample, a hit is queued
//   shade    per queued slot: hit or miss program of the current light sample; a finished
//            light sample restarts the next one from the cached primary hit in the same thread,
//            so each pixel's radiance accumulates in the reference's order; a finished slot
//            stores its pixel sample; a continuing path is appended to the extension queue
//            (warp-aggregated atomics)
//   extend   warps pull 32 queued rays at a time and find their closest hits
//   fold     per pixel: the batch's K samples, in sample order, into the running mean
//            (Welford), then the sRGB output
// The host alternates shade/extend until the queue is empty.
//
// Preview (replaces direct_ray_gen/direct_closest_hit, fresnel/gpu/direct.cu, with the CPU
// arithmetic of fresnel/cpu/TracerDirect.cc:59-220): aa_n^2 samples per pixel, a group of 32 or
// 16 lanes per pixel when that count is a multiple of 16, else one thread per pixel.
#include "path_device.cuh"

namespace fr {

namespace {

// Primary rays of every slot of the batch, one thread per work item (primary_item order).
template <int WIDTH, uint32_t MASK, bool PACKET = false>
__global__ void __launch_bounds__(256) k_path_primary(FrameParams P, PathState S)
{
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n_items = primary_items(P.w, P.h, P.batch, P.tile_log2);
    PrimaryItem it;
    it.valid = false;
    if (g < n_items)
        it = primary_item(g, P.w, P.h, P.batch, P.tile_log2);
    bool push = false;
    uint32_t slot = 0;
    TraceCount tc;
    if constexpr (PACKET) {
        // a warp's rays are neighbouring samples of the same pixels: trace them as a packet
        __shared__ uint32_t stk_node[8][TRAVERSAL_STACK];
        __shared__ float stk_t[8][TRAVERSAL_STACK];
        const uint32_t w = threadIdx.x >> 5;
        V3 o = v3(0.0f, 0.0f, 0.0f), d = v3(0.0f, 0.0f, 1.0f);
        if (it.valid)
            camera_ray(P.cam, it.i, it.j, P.n_samples + it.k, o, d);
        Hit h = trace_closest_packet<MASK>(P.scene, o, d, it.valid, PATH_TNEAR, tc, stk_node[w],
                                           stk_t[w]);
        if (it.valid) {
            slot = g;
            push = primary_finish(P, S, slot, o, d, h);
        }
    } else if (it.valid) {
        slot = g;
        push = primary_ray<WIDTH, MASK>(P, S, it, slot, tc);
    }
    flush_counts(tc, P.stats + 3);
    push_primary(S, push, slot);
    const uint32_t mv = __ballot_sync(0xffffffffu, it.valid);
    if (lane_id() == 0 && mv) {
        atomicAdd(P.stats + 0, (unsigned long long)__popc(mv));
        atomicAdd(P.stats + 1, (unsigned long long)__popc(mv) * P.light_samples);
    }
}

// Primary rays with their first shading (device option "fuse_shade"): one thread per work item
// as k_path_primary; continuing paths go straight to the extension queue (queue 0), so the
// frame's first shade pass is not launched.  Limited to fused_blocks<MASK> blocks of 256 threads
// per SM.
template <int WIDTH, uint32_t MASK>
__global__ void __launch_bounds__(256, fused_blocks(MASK)) k_path_primary_shade(FrameParams P, PathState S)
{
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n_items = primary_items(P.w, P.h, P.batch, P.tile_log2);
    PrimaryItem it;
    it.valid = false;
    if (g < n_items)
        it = primary_item(g, P.w, P.h, P.batch, P.tile_log2);
    bool push = false;
    TraceCount tc;
    if (it.valid)
        push = primary_shade<WIDTH, MASK>(P, S, it, g, tc);
    flush_counts(tc, P.stats + 3);
    push_queue(S, 0, push, g);
    const uint32_t mv = __ballot_sync(0xffffffffu, it.valid);
    if (lane_id() == 0 && mv) {
        atomicAdd(P.stats + 0, (unsigned long long)__popc(mv));
        atomicAdd(P.stats + 1, (unsigned long long)__popc(mv) * P.light_samples);
    }
}

// ---------------------------------------------------------------------------------------------
// Persistent traversal with per-lane refill (4-wide trees): a warp steps one node visit at a
// time; whenever at least REFILL lanes are idle, they claim new work items with one atomic, so
// lanes stay busy although rays need very different numbers of steps.
// ---------------------------------------------------------------------------------------------
constexpr uint32_t REFILL = 8;

template <uint32_t MASK, class Src>
__device__ __forceinline__ void persistent_trace(const FrameParams& P, Src& src, uint32_t count,
                                                 uint32_t* work, TraceCount& tc, uint32_t& n_rays)
{
    uint32_t stack_node[TRAVERSAL_STACK];
    float stack_t[TRAVERSAL_STACK];
    LaneRay L;
    L.gi = 0;
    L.cur = NEED_GEOM;
    bool active = false;
    uint32_t item = 0;
    bool exhausted = false;  // warp-uniform
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt = (1u << lane) - 1u;
    while (true) {
        uint32_t idle = __ballot_sync(0xffffffffu, !active);
        if (!exhausted && (__popc(idle) >= REFILL || idle == 0xffffffffu)) {
            uint32_t n = uint32_t(__popc(idle));
            uint32_t base = 0;
            if (lane == 0)
                base = atomicAdd(work, n);
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base >= count || count - base <= n)
                exhausted = true;
            if (!active) {
                item = base + uint32_t(__popc(idle & lt));
                if (item < count && src.begin(item, L)) {
                    active = true;
                    ++n_rays;
                }
            }
        }
        if (__ballot_sync(0xffffffffu, active) == 0u) {
            if (exhausted)
                break;
            continue;
        }
        bool done = false;
        if (active && !step4<MASK>(P.scene, L, stack_node, stack_t, tc)) {
            done = true;
            active = false;
        }
        if (__any_sync(0xffffffffu, done))
            src.finish(done, item, L);
    }
}

struct PrimarySource {
    const FrameParams& P;
    const PathState& S;
    uint32_t slot;
    __device__ bool begin(uint32_t item, LaneRay& L)
    {
        const PrimaryItem it = primary_item(item, P.w, P.h, P.batch, P.tile_log2);
        if (!it.valid)
            return false;
        slot = item;
        V3 o, d;
        camera_ray(P.cam, it.i, it.j, P.n_samples + it.k, o, d);
        lane_begin(L, o, d, PATH_TNEAR);
        return true;
    }
    // warp-collective: every lane calls it after each step, `done` marks finished rays
    __device__ void finish(bool done, uint32_t, const LaneRay& L)
    {
        bool push = false;
        if (done) {
            uint32_t prim = L.hit_geom == MISS ? 0u : __ldg(P.scene.geoms[L.hit_geom].order + L.hit_slot);
            st_cs(S.prim_hit + (slot), make_uint2(L.hit_geom, prim));
            if (L.hit_geom == MISS) {
                C3 res = P.bg * float(P.light_samples);
                C3 out = c_div_recip(res, float(P.light_samples));
                st_cs(S.sample + (slot), make_float4(out.r, out.g, out.b, P.bg_alpha));
            } else {
                st_cs(S.prim_o + (slot), f4(L.ray.o));
                st_cs(S.prim_d + (slot), f4(L.ray.d));
                st_cs(S.ls_depth + (slot), make_uint2(0u, 0u));  // see primary_finish
                push = true;
            }
        }
        uint32_t m = __ballot_sync(0xffffffffu, push);
        if (m) {
            const uint32_t lane = threadIdx.x & 31u;
            uint32_t at = 0;
            if (lane == 0)
                at = atomicAdd(S.ctr + 1, uint32_t(__popc(m)));
            at = __shfl_sync(0xffffffffu, at, 0);
            if (push)
                st_cs(S.queue[1] + (at + __popc(m & ((1u << lane) - 1u))), slot);
        }
    }
};

struct ExtendSource {
    const FrameParams& P;
    const PathState& S;
    const uint32_t* queue;
    uint32_t slot;
    __device__ bool begin(uint32_t item, LaneRay& L)
    {
        slot = ld_cs(queue + (item));
        lane_begin(L, xyz(ld_cs(S.ray_o + (slot))), xyz(ld_cs(S.ray_d + (slot))), PATH_TNEAR);
        return true;
    }
    __device__ void finish(bool done, uint32_t, const LaneRay& L)
    {
        if (done) {
            uint32_t prim = L.hit_geom == MISS ? 0u : __ldg(P.scene.geoms[L.hit_geom].order + L.hit_slot);
            st_cs(S.hit + (slot), make_uint2(L.hit_geom, prim));
        }
    }
};

__device__ __forceinline__ void flush_rays(const FrameParams& P, uint32_t n_rays, bool paths)
{
    unsigned long long r = n_rays;
    for (int off = 16; off > 0; off >>= 1)
        r += __shfl_xor_sync(0xffffffffu, r, off);
    if (lane_id() == 0u && r) {
        atomicAdd(P.stats + 0, r);
        if (paths)
            atomicAdd(P.stats + 1, r * P.light_samples);
    }
}

template <uint32_t MASK>
__global__ void __launch_bounds__(256) k_path_primary_persistent(FrameParams P, PathState S)
{
    PrimarySource src{P, S, 0u};
    TraceCount tc;
    uint32_t n_rays = 0;
    persistent_trace<MASK>(P, src, primary_items(P.w, P.h, P.batch, P.tile_log2), S.ctr + 3, tc, n_rays);
    flush_counts(tc, P.stats + 3);
    flush_rays(P, n_rays, true);
}

template <uint32_t MASK>
__global__ void __launch_bounds__(256) k_path_extend_persistent(FrameParams P, PathState S, int q)
{
    if (blockIdx.x == 0 && threadIdx.x == 0)
        S.ctr[q ^ 1] = 0;  // the other queue was consumed by the shade pass that produced q
    ExtendSource src{P, S, S.queue[q], 0u};
    TraceCount tc;
    uint32_t n_rays = 0;
    persistent_trace<MASK>(P, src, S.ctr[q], S.ctr + 2, tc, n_rays);
    flush_counts(tc, P.stats + 3);
    flush_rays(P, n_rays, false);
}

// Fold the batch's samples into the running mean of each pixel, in sample order, then write
// the sRGB output once.
__global__ void __launch_bounds__(256) k_path_fold(FrameParams P, PathState S)
{
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P.w * P.h)
        return;
    const uint32_t j = p / P.w;
    const uint32_t base = pixel_slot(p - j * P.w, j, P.w, P.batch, P.tile_log2);
    float4 mean = P.linear[p];
    for (uint32_t k = 0; k < P.batch; ++k)
        mean = welford(P, mean, S.sample[base + k], P.n_samples + k);
    write_pixel(P, p, mean.x, mean.y, mean.z, mean.w);
}

// Tracer.histogram (fresnel/tracer.py:79-108) over the linear output, with numpy's float32
// arithmetic: for every pixel with alpha > 0, the lightness l = (0.21 r + 0.72 g) + 0.07 b
// (each product and sum rounded to float32) and r, g, b are raised to float32(1/2.2) and
// counted in HIST_BINS equal bins over [0, 1]; 1 falls in the last bin, values outside
// [0, 1] and NaN in none.  The power is evaluated in double and rounded once to float32.
// counts[bin * 4 + channel], channels (l, r, g, b); counts must be zero on entry.
__global__ void __launch_bounds__(256) k_histogram(const float4* linear, uint32_t n,
                                                   uint32_t* counts)
{
    __shared__ uint32_t h[HIST_BINS * 4];
    for (uint32_t i = threadIdx.x; i < HIST_BINS * 4; i += blockDim.x)
        h[i] = 0;
    __syncthreads();
    const double e = double(float(1.0 / 2.2));
    auto count = [&](float x, uint32_t c) {
        const float v = __double2float_rn(pow(double(x), e));
        if (v >= 0.0f && v <= 1.0f) {
            const uint32_t b = min(uint32_t(v * float(HIST_BINS)), HIST_BINS - 1u);
            atomicAdd(&h[b * 4u + c], 1u);
        }
    };
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const float4 a = ldg4(linear + p);
        if (!(a.w > 0.0f))
            continue;
        const float l = __fadd_rn(__fadd_rn(__fmul_rn(float(0.21), a.x), __fmul_rn(float(0.72), a.y)),
                                  __fmul_rn(float(0.07), a.z));
        count(l, 0);
        count(a.x, 1);
        count(a.y, 2);
        count(a.z, 3);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < HIST_BINS * 4; i += blockDim.x)
        if (h[i])
            atomicAdd(counts + i, h[i]);
}

// Shade pass: the slots of queue in_q, continuing paths appended to queue out_q.  A slot's
// light samples that end at the primary vertex are shaded one after another by the same lane, so
// lanes finish their slots after different numbers of steps (up to the light-sample count); a
// lane whose slot is done takes the next slot of its warp's share of the queue (groups of 32
// slots, warp w owning groups w, w + n_warps, ...) while the others carry on, so the warp's lanes
// stay busy until the share runs out.  The continuing slots are staged per warp in shared memory
// and appended to out_q 32 at a time: the extension pass takes its rays 32 per warp in queue
// order, and a run of one warp's slots (a few neighbouring pixel samples, whose rays start from
// about the same point) traces more coherently than slots interleaved from many warps.
template <int MINB = 1>
__global__ void __launch_bounds__(256, MINB) k_path_shade(FrameParams P, PathState S, int in_q,
                                                          int out_q)
{
    if (blockIdx.x == 0 && threadIdx.x == 0)
        S.ctr[2] = 0;  // work counter of the extend kernel that follows
    const uint32_t count = S.ctr[in_q];
    const uint32_t* inq = S.queue[in_q];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t below = (1u << lane) - 1u;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t n_warps = (gridDim.x * blockDim.x) >> 5;
    __shared__ uint32_t stage[8][64];  // blocks of 256 threads: 8 warps
    uint32_t* staged = stage[threadIdx.x >> 5];
    uint32_t n_staged = 0;  // warp-uniform, below 32 between iterations
    uint32_t* outq = S.queue[out_q];
    uint32_t* outc = S.ctr + out_q;
    uint32_t taken = 0;  // positions of the warp's share handed out so far (warp-uniform)
    bool busy = false;
    ShadeLane L;
    L.p = 0;
    while (true) {
        const uint32_t idle = __ballot_sync(0xffffffffu, !busy);
        if (idle) {
            if (!busy) {
                const uint32_t k = taken + __popc(idle & below);
                const uint32_t idx = (warp + (k >> 5) * n_warps) * 32u + (k & 31u);
                if (idx < count) {
                    const uint32_t p = ld_cs(inq + (idx));
                    shade_load(P, S, p, p, L);
                    busy = true;
                }
            }
            taken += __popc(idle);
        }
        if (!__any_sync(0xffffffffu, busy))
            break;
        bool push = false;
        if (busy) {
            const ShadeStep r = shade_step(P, S, L);
            if (r != STEP_RESTART) {
                busy = false;
                push = r == STEP_CONTINUE;
            }
        }
        const uint32_t m = __ballot_sync(0xffffffffu, push);
        if (push)
            staged[n_staged + __popc(m & below)] = L.p;
        n_staged += __popc(m);
        if (n_staged >= 32u) {
            __syncwarp();
            uint32_t at = 0;
            if (lane == 0)
                at = atomicAdd(outc, 32u);
            at = __shfl_sync(0xffffffffu, at, 0);
            outq[at + lane] = staged[lane];
            const uint32_t rest = staged[32u + lane];
            __syncwarp();
            n_staged -= 32u;
            if (lane < n_staged)
                staged[lane] = rest;
            __syncwarp();
        }
    }
    if (n_staged) {
        __syncwarp();
        uint32_t at = 0;
        if (lane == 0)
            at = atomicAdd(outc, n_staged);
        at = __shfl_sync(0xffffffffu, at, 0);
        if (lane < n_staged)
            outq[at + lane] = staged[lane];
    }
}

template <int WIDTH, uint32_t MASK>
__global__ void __launch_bounds__(256) k_path_extend(FrameParams P, PathState S, int q)
{
    if (blockIdx.x == 0 && threadIdx.x == 0)
        S.ctr[q ^ 1] = 0;  // the other queue was consumed by the shade pass that produced q
    const uint32_t count = S.ctr[q];
    const uint32_t* queue = S.queue[q];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t CHUNK = 32;  // rays claimed per atomic: one per lane keeps every warp busy
    TraceCount tc;
    while (true) {
        uint32_t base = 0;
        if (lane == 0)
            base = atomicAdd(S.ctr + 2, CHUNK);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= count)
            break;
        for (uint32_t sub = 0; sub < CHUNK; sub += 32) {
            uint32_t idx = base + sub + lane;
            if (idx < count) {
                uint32_t p = ld_cs(queue + (idx));
                V3 o = xyz(ld_cs(S.ray_o + (p)));
                V3 d = xyz(ld_cs(S.ray_d + (p)));
                Hit h = trace_closest<WIDTH, MASK>(P.scene, o, d, PATH_TNEAR, tc);
                st_cs(S.hit + (p), make_uint2(h.geom, h.prim));
            }
        }
        if (lane == 0)
            atomicAdd(P.stats + 0, (unsigned long long)min(CHUNK, count - base));
    }
    flush_counts(tc, P.stats + 3);
}

// Extension rays traced and shaded at once (device option "fuse_shade"): the rays of queue q are
// taken 32 per warp as in k_path_extend; the continuing paths go to queue q ^ 1, whose length
// and the work counter (ctr[2]) must be zero at launch.  Limited to fused_blocks<MASK> blocks per
// SM.
template <int WIDTH, uint32_t MASK>
__global__ void __launch_bounds__(256, fused_blocks(MASK)) k_path_bounce(FrameParams P, PathState S, int q)
{
    const uint32_t count = S.ctr[q];
    const uint32_t* queue = S.queue[q];
    const uint32_t lane = threadIdx.x & 31u;
    TraceCount tc;
    while (true) {
        uint32_t base = 0;
        if (lane == 0)
            base = atomicAdd(S.ctr + 2, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= count)
            break;
        const uint32_t idx = base + lane;
        bool push = false;
        uint32_t p = 0;
        if (idx < count) {
            p = ld_cs(queue + (idx));
            push = bounce<WIDTH, MASK>(P, S, p, p, tc);
        }
        push_queue(S, q ^ 1, push, p);
        if (lane == 0)
            atomicAdd(P.stats + 0, (unsigned long long)min(32u, count - base));
    }
    flush_counts(tc, P.stats + 3);
}

// The tail of a wavefront's bounces in one launch (sphere-grid scenes): once the early bounces
// have retired most paths, the launches of later bounces carry few rays each and every launch
// lasts as long as its longest grid walk.  Here each lane follows its path bounce after bounce
// (trace, shade, store, read back) until the path finishes, then takes the next path of queue q
// (lanes that are idle together share one atomic), so the walks of different bounces overlap
// instead of being serialised launch by launch.  Every path runs the same per-bounce arithmetic
// as in k_path_bounce.  The work counter (ctr[2]) must be zero at launch; no queue is written.
// A path longer than TAIL_MAX_DEPTH further bounces is cut and reported.

template <int WIDTH, uint32_t MASK>
__global__ void __launch_bounds__(256, fused_blocks(MASK)) k_path_tail(FrameParams P, PathState S, int q)
{
    const uint32_t count = S.ctr[q];
    const uint32_t* queue = S.queue[q];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t below = (1u << lane) - 1u;
    TraceCount tc;
    bool active = false, exhausted = false;
    uint32_t p = 0, guard = 0;
    unsigned long long rays = 0;
    while (true) {
        const uint32_t idle = __ballot_sync(0xffffffffu, !active);
        if (idle && !exhausted) {
            const uint32_t n = uint32_t(__popc(idle));
            uint32_t base = 0;
            if (lane == 0)
                base = atomicAdd(S.ctr + 2, n);
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base + n >= count)
                exhausted = true;
            if (!active) {
                const uint32_t item = base + uint32_t(__popc(idle & below));
                if (item < count) {
                    p = ld_cs(queue + item);
                    active = true;
                    guard = TAIL_MAX_DEPTH;
                }
            }
        }
        if (__ballot_sync(0xffffffffu, active) == 0u)
            break;
        if (active) {
            ++rays;
            if (!bounce<WIDTH, MASK>(P, S, p, p, tc)) {
                active = false;
            } else if (--guard == 0u) {
                atomicOr(P.scene.status, ERR_ITERATION_CAP);
                active = false;
            }
        }
    }
    for (int off = 16; off > 0; off >>= 1)
        rays += __shfl_xor_sync(0xffffffffu, rays, off);
    if (lane == 0 && rays)
        atomicAdd(P.stats + 0, rays);
    flush_counts(tc, P.stats + 3);
}

// ---------------------------------------------------------------------------------------------
// Extension rays with per-lane refill: a lane whose ray is finished takes the next queued ray as
// soon as at least REFILL_MIN lanes of its warp are idle (one atomic per refill), so the lanes of
// a warp do not wait for the warp's slowest ray.  Each lane runs the same node visits (visit4)
// as the one-ray-per-thread kernel.  Scenes with a combined tree or a single enabled geometry
// (P.refill_geom: -2 combined, else the geometry's index).
// ---------------------------------------------------------------------------------------------
constexpr uint32_t REFILL_MIN = 8;

template <uint32_t MASK>
__global__ void __launch_bounds__(256) k_path_extend_refill(FrameParams P, PathState S, int q)
{
    if (blockIdx.x == 0 && threadIdx.x == 0)
        S.ctr[q ^ 1] = 0;  // the other queue was consumed by the shade pass that produced q
    const uint32_t count = S.ctr[q];
    const uint32_t* queue = S.queue[q];
    const uint32_t lane = lane_id();
    const uint32_t below = (1u << lane) - 1u;
    const SceneDev& sc = P.scene;
    const bool combined = P.refill_geom < 0;
    const uint32_t gi = combined ? 0u : uint32_t(P.refill_geom);
    const GeomDev& g = sc.geoms[gi];
    const float4* nodes4 = combined ? sc.nodes4 : g.nodes4;
    const uint32_t n_nodes4 = combined ? sc.n_nodes4 : g.n_nodes4;
    const uint32_t n_prims = combined ? sc.n_prims : g.n_prims;
    const int type = combined ? -1 : g.type;
    uint32_t stack_node[TRAVERSAL_STACK];
    float stack_t[TRAVERSAL_STACK];
    TraceCount tc;
    bool active = false, exhausted = false;
    uint32_t p = 0, cur = 0, guard = 0, hg = MISS, hs = 0;
    int sp = 0;
    float tmax = 0.0f;
    RayK ray;
    NearFar nf{0, 2, 4};
    unsigned long long rays = 0;
    auto leaf = [&](uint32_t first, uint32_t n) {
        if (combined) {
            leaf_test_mixed<MASK>(sc, ray, first, n, PATH_TNEAR, tmax, hg, hs, tc);
            return;
        }
#define FR_LEAF(T)                                                                       \
    if ((MASK & (1u << T)) && type == T) {                                               \
        leaf_test<T>(g, gi, ray, first, n, PATH_TNEAR, tmax, hg, hs, tc);                 \
        return;                                                                          \
    }
        FR_LEAF(FR_GEOM_SPHERE)
        FR_LEAF(FR_GEOM_CYLINDER)
        FR_LEAF(FR_GEOM_POLYHEDRON)
        FR_LEAF(FR_GEOM_MESH)
        FR_LEAF(FR_GEOM_POLYGON)
#undef FR_LEAF
    };
    while (true) {
        const uint32_t idle = __ballot_sync(0xffffffffu, !active);
        if (!exhausted && (__popc(idle) >= int(REFILL_MIN) || idle == 0xffffffffu)) {
            const uint32_t n = uint32_t(__popc(idle));
            uint32_t base = 0;
            if (lane == 0)
                base = atomicAdd(S.ctr + 2, n);
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base + n >= count)
                exhausted = true;
            if (!active) {
                const uint32_t item = base + uint32_t(__popc(idle & below));
                if (item < count) {
                    p = ld_cs(queue + (item));
                    ray = make_rayk(xyz(ld_cs(S.ray_o + (p))), xyz(ld_cs(S.ray_d + (p))));
                    nf = near_far(ray);
                    tmax = __int_as_float(0x7f800000);
                    hg = MISS;
                    hs = 0;
                    cur = 0;
                    sp = 0;
                    guard = n_nodes4 + 8u;
                    active = n_nodes4 != 0;
                    if (!active)
                        st_cs(S.hit + (p), make_uint2(MISS, 0u));
                    ++rays;
                }
            }
        }
        if (__ballot_sync(0xffffffffu, active) == 0u) {
            if (exhausted)
                break;
            continue;
        }
        if (active) {
            bool more = false;
            if (--guard == 0u)
                atomicOr(sc.status, ERR_ITERATION_CAP);
            else
                more = visit4(nodes4, n_nodes4, n_prims, ray, nf, tmax, cur, sp, stack_node,
                              stack_t, sc.status, tc, leaf);
            if (!more) {
                uint32_t prim = 0;
                if (hg != MISS)
                    prim = __ldg((combined ? sc.order : sc.geoms[hg].order) + hs);
                st_cs(S.hit + (p), make_uint2(hg, prim));
                active = false;
            }
        }
    }
    for (int off = 16; off > 0; off >>= 1)
        rays += __shfl_xor_sync(0xffffffffu, rays, off);
    if (lane == 0 && rays)
        atomicAdd(P.stats + 0, rays);
    flush_counts(tc, P.stats + 3);
}

// Extension rays through the sphere grid with per-lane refill (device option "refill"): a lane
// walks one cell of its ray per iteration, and a lane whose walk is over stores the hit and
// takes the next queued ray as soon as REFILL_MIN lanes of its warp are idle, so the warp is not
// held by its longest walk.  The hits are shaded by the separate shade pass.
__global__ void __launch_bounds__(256) k_path_extend_grid_refill(FrameParams P, PathState S, int q)
{
    if (blockIdx.x == 0 && threadIdx.x == 0)
        S.ctr[q ^ 1] = 0;  // the other queue was consumed by the shade pass that produced q
    const uint32_t count = S.ctr[q];
    const uint32_t* queue = S.queue[q];
    const uint32_t lane = lane_id();
    const uint32_t below = (1u << lane) - 1u;
    const GridDev& G = P.scene.grid;
    TraceCount tc;
    bool active = false, exhausted = false;
    uint32_t p = 0, slot = MISS;
    float tmax = 0.0f;
    RayK ray;
    GridWalk W;
    unsigned long long rays = 0;
    while (true) {
        const uint32_t idle = __ballot_sync(0xffffffffu, !active);
        if (!exhausted && (__popc(idle) >= int(REFILL_MIN) || idle == 0xffffffffu)) {
            const uint32_t n = uint32_t(__popc(idle));
            uint32_t base = 0;
            if (lane == 0)
                base = atomicAdd(S.ctr + 2, n);
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base + n >= count)
                exhausted = true;
            if (!active) {
                const uint32_t item = base + uint32_t(__popc(idle & below));
                if (item < count) {
                    p = ld_cs(queue + (item));
                    ray = make_rayk(xyz(ld_cs(S.ray_o + (p))), xyz(ld_cs(S.ray_d + (p))));
                    tmax = __int_as_float(0x7f800000);
                    slot = MISS;
                    active = grid_walk_begin(G, ray, W);
                    if (!active)
                        st_cs(S.hit + (p), make_uint2(MISS, 0u));
                    ++rays;
                }
            }
        }
        if (__ballot_sync(0xffffffffu, active) == 0u) {
            if (exhausted)
                break;
            continue;
        }
        if (active && !grid_walk_step(G, ray, PATH_TNEAR, tmax, slot, W, tc)) {
            st_cs(S.hit + (p), slot == MISS ? make_uint2(MISS, 0u)
                                            : make_uint2(G.geom, __ldg(G.ref_prim + slot)));
            active = false;
        }
    }
    for (int off = 16; off > 0; off >>= 1)
        rays += __shfl_xor_sync(0xffffffffu, rays, off);
    if (lane == 0 && rays)
        atomicAdd(P.stats + 0, rays);
    flush_counts(tc, P.stats + 3);
}

// Representative-point area-light shading of one preview sample
// (fresnel/cpu/TracerDirect.cc:120-200).
__device__ __forceinline__ C3 preview_shade(const FrameParams& P, const GeomDev& g,
                                            const Surface& sf, V3 dir)
{
    V3 n = div_each(sf.Ng, sqrtf(dot(sf.Ng, sf.Ng)));
    V3 v = div_recip(-dir, sqrtf(dot(dir, dir)));
    const Mat& m = (sf.d_edge >= g.outline_width) ? g.material : g.outline;
    if (is_solid(m))
        return base_color(m, sf.color);
    C3 c = c3(0, 0, 0);
    for (uint32_t li = 0; li < P.lights.n; ++li) {
        V3 l = P.lights.dir[li];
        V3 r = -v + (2.0f * n * dot(n, v));
        float half = P.lights.theta[li];
        const float cos_half = P.lights.cos_theta[li];
        float ldotr = dot(l, r);
        if (ldotr < cos_half) {
            V3 ax = cross(l, r);
            ax = div_recip(ax, sqrtf(dot(ax, ax)));
            Qt q = from_axis_angle(ax, -hacos(ldotr) + half);
            r = rotate(q, r);
        }
        C3 f_d = c3(0, 0, 0), f_s = c3(0, 0, 0);
        float ndotl = dot(n, l);
        if (ndotl >= 0.0f)
            f_d = brdf_diffuse(m, l, v, n, sf.color) * ndotl;
        if (dot(n, r) >= 0.0f)
            f_s = brdf_specular(m, r, v, n, sf.color, half) * dot(n, r);
        c = c + (f_d + f_s) * PI_F * P.lights.color[li];
    }
    return c;
}

template <int WIDTH, uint32_t MASK>
__global__ void __launch_bounds__(256) k_preview(FrameParams P, uint32_t aa_n, uint2* hits)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t j = blockIdx.y * blockDim.y + threadIdx.y;
    bool valid = (i < P.w) && (j < P.h);
    const uint32_t ns = aa_n * aa_n;
    TraceCount tc;
    if (valid) {
        uint32_t p = j * P.w + i;
        float avg[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        for (uint32_t sample = 0; sample < ns; ++sample) {
            V3 o, d;
            camera_ray(P.cam, i, j, sample, o, d);
            Hit h = trace_closest<WIDTH, MASK>(P.scene, o, d, 0.0f, tc);  // CPU preview: tnear 0
            C3 c = P.bg;
            float a = P.bg_alpha;
            if (h.geom != MISS) {
                const GeomDev& g = P.scene.geoms[h.geom];
                Surface sf = hit_surface(g, h.prim, o, d, 0.0f);
                c = preview_shade(P, g, sf, d);
                a = 1.0f;
            }
            if (hits)
                hits[size_t(p) * ns + sample] =
                    make_uint2(h.geom == MISS ? 0u : h.geom + 1u, h.geom == MISS ? 0u : h.prim);
            avg[0] += c.r;
            avg[1] += c.g;
            avg[2] += c.b;
            avg[3] += a;
        }
        float q = 1.0f / float(ns);
        write_pixel(P, p, avg[0] * q, avg[1] * q, avg[2] * q, avg[3] * q);
    }
    flush_counts(tc, P.stats + 3);
    uint32_t m = __ballot_sync(0xffffffffu, valid);
    if ((threadIdx.x + threadIdx.y * blockDim.x) % 32 == 0 && m) {
        atomicAdd(P.stats + 0, (unsigned long long)__popc(m) * ns);
        atomicAdd(P.stats + 1, (unsigned long long)__popc(m) * ns);
    }
}

// Preview with a group of G lanes per pixel (G = 32 or 16 dividing the samples per pixel: 4x4
// and 8x8 anti-aliasing): lane l of a group traces samples l, l + G, ... of its pixel,
// so that a warp's rays are a few pixels' own jittered samples, which walk the same cells and
// nodes, where k_preview's warp holds 32 pixels whose sample loops run side by side.  Each round
// of G samples is summed in sample order (every lane reads its group's G colours by shuffles), so
// the pixel is the same float sum as k_preview's; the hit ids go to the same places.
template <int WIDTH, uint32_t MASK, uint32_t G>
__global__ void __launch_bounds__(256) k_preview_warp(FrameParams P, uint32_t aa_n, uint2* hits)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t gl = lane & (G - 1u);  // lane within the pixel's group
    const uint32_t first = lane - gl;     // the group's first lane
    const uint32_t gmask = (G == 32u ? 0xffffffffu : ((1u << G) - 1u)) << first;
    const uint32_t p = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    const bool valid = p < P.w * P.h;  // uniform within a group
    const uint32_t ns = aa_n * aa_n;   // a multiple of G
    TraceCount tc;
    if (valid) {
        const uint32_t j = p / P.w, i = p - j * P.w;
        float avg[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        for (uint32_t base = 0; base < ns; base += G) {
            const uint32_t sample = base + gl;
            V3 o, d;
            camera_ray(P.cam, i, j, sample, o, d);
            Hit h = trace_closest<WIDTH, MASK>(P.scene, o, d, 0.0f, tc);  // CPU preview: tnear 0
            C3 c = P.bg;
            float a = P.bg_alpha;
            if (h.geom != MISS) {
                const GeomDev& g = P.scene.geoms[h.geom];
                Surface sf = hit_surface(g, h.prim, o, d, 0.0f);
                c = preview_shade(P, g, sf, d);
                a = 1.0f;
            }
            if (hits)
                hits[size_t(p) * ns + sample] =
                    make_uint2(h.geom == MISS ? 0u : h.geom + 1u, h.geom == MISS ? 0u : h.prim);
            for (uint32_t k = 0; k < G; ++k) {
                avg[0] += __shfl_sync(gmask, c.r, first + k);
                avg[1] += __shfl_sync(gmask, c.g, first + k);
                avg[2] += __shfl_sync(gmask, c.b, first + k);
                avg[3] += __shfl_sync(gmask, a, first + k);
            }
        }
        if (gl == 0u) {
            const float q = 1.0f / float(ns);
            write_pixel(P, p, avg[0] * q, avg[1] * q, avg[2] * q, avg[3] * q);
        }
    }
    flush_counts(tc, P.stats + 3);
    if (valid && gl == 0u) {
        atomicAdd(P.stats + 0, (unsigned long long)ns);
        atomicAdd(P.stats + 1, (unsigned long long)ns);
    }
}

// Diagnostic: trace rays[i] = (o, d) with both 4-wide traversal forms (one ray per thread, and
// the step-wise form stepped to completion by one lane); out[i] = (geom, prim, box tests) of
// each, six words per ray.
__global__ void k_traversal_compare(SceneDev sc, const float* rays, uint32_t n, uint32_t* out)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    V3 o = v3(rays[6 * i], rays[6 * i + 1], rays[6 * i + 2]);
    V3 d = v3(rays[6 * i + 3], rays[6 * i + 4], rays[6 * i + 5]);
    TraceCount a;
    Hit h = trace_closest<4, MASK_SPHERES>(sc, o, d, PATH_TNEAR, a);
    LaneRay L;
    lane_begin(L, o, d, PATH_TNEAR);
    uint32_t stack_node[TRAVERSAL_STACK];
    float stack_t[TRAVERSAL_STACK];
    TraceCount b;
    for (int guard = 0; guard < 100000 && step4<MASK_SPHERES>(sc, L, stack_node, stack_t, b); ++guard) {
    }
    uint32_t prim = L.hit_geom == MISS ? 0u : __ldg(sc.geoms[L.hit_geom].order + L.hit_slot);
    uint32_t* r = out + 6 * size_t(i);
    r[0] = h.geom;
    r[1] = h.prim;
    r[2] = a.box;
    r[3] = L.hit_geom;
    r[4] = prim;
    r[5] = b.box;
}

}  // namespace

void launch_traversal_compare(const SceneDev& sc, const float* rays, uint32_t n, uint32_t* out,
                              cudaStream_t st)
{
    k_traversal_compare<<<(n + 127) / 128, 128, 0, st>>>(sc, rays, n, out);
}

// Pick the kernel instantiation for the frame's BVH width and geometry mix.
template <class F> F pick(const FrameParams& P, F w2s, F w2a, F w4s, F w4a)
{
    bool spheres_only = (P.type_mask & ~MASK_SPHERES) == 0u;
    if (P.bvh_width == 4)
        return spheres_only ? w4s : w4a;
    return spheres_only ? w2s : w2a;
}

template <class K> int blocks_per_sm(K kernel)
{
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, 256, 0);
    return n > 0 ? n : 1;
}

LaunchShape path_launch_shape(int num_sms)
{
    LaunchShape s;
    s.shade_grid = num_sms * blocks_per_sm(k_path_shade<>);
    s.shade_grid_occ[0] = num_sms * blocks_per_sm(k_path_shade<3>);
    s.refill_grid[0] = num_sms * blocks_per_sm(k_path_extend_refill<MASK_SPHERES>);
    s.refill_grid[1] = num_sms * blocks_per_sm(k_path_extend_refill<MASK_ALL>);
    s.shade_grid_occ[1] = num_sms * blocks_per_sm(k_path_shade<4>);
    s.extend_grid[0] = num_sms * blocks_per_sm(k_path_extend<2, MASK_SPHERES>);
    s.extend_grid[1] = num_sms * blocks_per_sm(k_path_extend<2, MASK_ALL>);
    s.extend_grid[2] = num_sms * blocks_per_sm(k_path_extend<4, MASK_SPHERES>);
    s.extend_grid[3] = num_sms * blocks_per_sm(k_path_extend<4, MASK_ALL>);
    s.extend_grid_sphere_grid = num_sms * blocks_per_sm(k_path_extend<4, MASK_GRID>);
    s.refill_grid_sphere_grid = num_sms * blocks_per_sm(k_path_extend_grid_refill);
    s.extend_grid_parts_grid[0] = num_sms * blocks_per_sm(k_path_extend<4, MASK_GRID_PARTS>);
    s.extend_grid_parts_grid[1] =
        num_sms * blocks_per_sm(k_path_extend<4, MASK_GRID_PARTS_NO_MESH>);
    s.bounce_grid[0] = num_sms * fused_blocks(MASK_ALL);
    s.bounce_grid[1] = num_sms * fused_blocks(MASK_GRID);
    s.bounce_grid[2] = num_sms * fused_blocks(MASK_GRID_PARTS);
    s.bounce_grid[3] = num_sms * fused_blocks(MASK_GRID_PARTS_NO_MESH);
    s.persistent_grid[0] = num_sms * blocks_per_sm(k_path_extend_persistent<MASK_SPHERES>);
    s.persistent_grid[1] = num_sms * blocks_per_sm(k_path_extend_persistent<MASK_ALL>);
    s.primary_grid[0] = num_sms * blocks_per_sm(k_path_primary_persistent<MASK_SPHERES>);
    s.primary_grid[1] = num_sms * blocks_per_sm(k_path_primary_persistent<MASK_ALL>);
    return s;
}

// The kernels a frame runs: 0 for BVH scenes, 1 for a sphere grid, 2 for a grid over parts, 3
// for a grid over parts none of which is a mesh.
static int grid_kind(const FrameParams& P)
{
    if (P.scene.grid.n_cells == 0)
        return 0;
    if (!P.scene.grid.parts)
        return 1;
    return (P.type_mask & (1u << FR_GEOM_MESH)) ? 2 : 3;
}

// The kernel K<4, mask> for grid kind gk (1-3).
#define FR_GRID_KERNEL(K, gk)                                                                  \
    ((gk) == 1 ? K<4, MASK_GRID> : (gk) == 2 ? K<4, MASK_GRID_PARTS> : K<4, MASK_GRID_PARTS_NO_MESH>)

void launch_path_primary(const FrameParams& P, const PathState& S, const LaunchShape& shape,
                         cudaStream_t st)
{
    bool spheres_only = (P.type_mask & ~MASK_SPHERES) == 0u;
    if (const int gk = grid_kind(P)) {
        const uint32_t n = primary_items(P.w, P.h, P.batch, P.tile_log2);
        auto k = gk == 1 ? k_path_primary<4, MASK_GRID>
                 : gk == 2 ? k_path_primary<4, MASK_GRID_PARTS>
                           : k_path_primary<4, MASK_GRID_PARTS_NO_MESH>;
        k<<<(n + 255) / 256, 256, 0, st>>>(P, S);
        return;
    }
    if (P.bvh_width == 4 && P.persistent) {
        if (spheres_only)
            k_path_primary_persistent<MASK_SPHERES><<<shape.primary_grid[0], 256, 0, st>>>(P, S);
        else
            k_path_primary_persistent<MASK_ALL><<<shape.primary_grid[1], 256, 0, st>>>(P, S);
        return;
    }
    const uint32_t n_items = primary_items(P.w, P.h, P.batch, P.tile_log2);
    auto k = pick(P, k_path_primary<2, MASK_SPHERES>, k_path_primary<2, MASK_ALL>,
                  k_path_primary<4, MASK_SPHERES>, k_path_primary<4, MASK_ALL>);
    if (P.bvh_width == 4 && P.packet)
        k = spheres_only ? k_path_primary<4, MASK_SPHERES, true> : k_path_primary<4, MASK_ALL, true>;
    k<<<(n_items + 255) / 256, 256, 0, st>>>(P, S);
}

void launch_path_primary_shade(const FrameParams& P, const PathState& S, cudaStream_t st)
{
    const uint32_t n_items = primary_items(P.w, P.h, P.batch, P.tile_log2);
    auto k = pick(P, k_path_primary_shade<2, MASK_SPHERES>, k_path_primary_shade<2, MASK_ALL>,
                  k_path_primary_shade<4, MASK_SPHERES>, k_path_primary_shade<4, MASK_ALL>);
    if (const int gk = grid_kind(P))
        k = FR_GRID_KERNEL(k_path_primary_shade, gk);
    k<<<(n_items + 255) / 256, 256, 0, st>>>(P, S);
}

void launch_path_fold(const FrameParams& P, const PathState& S, cudaStream_t st)
{
    k_path_fold<<<(P.w * P.h + 255) / 256, 256, 0, st>>>(P, S);
}

void launch_path_shade(const FrameParams& P, const PathState& S, int iteration,
                       const LaunchShape& shape, cudaStream_t st)
{
    // iteration 0 reads the primary hits (queue 1); then the queues alternate
    const int in_q = (iteration + 1) & 1, out_q = iteration & 1;
    if (P.shade_blocks == 3)
        k_path_shade<3><<<shape.shade_grid_occ[0], 256, 0, st>>>(P, S, in_q, out_q);
    else if (P.shade_blocks == 4)
        k_path_shade<4><<<shape.shade_grid_occ[1], 256, 0, st>>>(P, S, in_q, out_q);
    else
        k_path_shade<><<<shape.shade_grid, 256, 0, st>>>(P, S, in_q, out_q);
}

void launch_path_extend(const FrameParams& P, const PathState& S, int iteration,
                        const LaunchShape& shape, cudaStream_t st)
{
    bool spheres_only = (P.type_mask & ~MASK_SPHERES) == 0u;
    int q = iteration & 1;
    if (const int gk = grid_kind(P)) {
        if (gk == 2)
            k_path_extend<4, MASK_GRID_PARTS><<<shape.extend_grid_parts_grid[0], 256, 0, st>>>(P, S, q);
        else if (gk == 3)
            k_path_extend<4, MASK_GRID_PARTS_NO_MESH>
                <<<shape.extend_grid_parts_grid[1], 256, 0, st>>>(P, S, q);
        else if (P.refill)
            k_path_extend_grid_refill<<<shape.refill_grid_sphere_grid, 256, 0, st>>>(P, S, q);
        else
            k_path_extend<4, MASK_GRID><<<shape.extend_grid_sphere_grid, 256, 0, st>>>(P, S, q);
        return;
    }
    if (P.bvh_width == 4 && P.persistent) {
        if (spheres_only)
            k_path_extend_persistent<MASK_SPHERES><<<shape.persistent_grid[0], 256, 0, st>>>(P, S, q);
        else
            k_path_extend_persistent<MASK_ALL><<<shape.persistent_grid[1], 256, 0, st>>>(P, S, q);
        return;
    }
    if (P.bvh_width == 4 && P.refill && P.refill_geom != -1) {
        if (spheres_only)
            k_path_extend_refill<MASK_SPHERES><<<shape.refill_grid[0], 256, 0, st>>>(P, S, q);
        else
            k_path_extend_refill<MASK_ALL><<<shape.refill_grid[1], 256, 0, st>>>(P, S, q);
        return;
    }
    int grid = shape.extend_grid[(P.bvh_width == 4 ? 2 : 0) + (spheres_only ? 0 : 1)];
    auto k = pick(P, k_path_extend<2, MASK_SPHERES>, k_path_extend<2, MASK_ALL>,
                  k_path_extend<4, MASK_SPHERES>, k_path_extend<4, MASK_ALL>);
    k<<<grid, 256, 0, st>>>(P, S, q);
}

void launch_path_bounce(const FrameParams& P, const PathState& S, int iteration,
                        const LaunchShape& shape, cudaStream_t st)
{
    const int q = iteration & 1;
    auto k = pick(P, k_path_bounce<2, MASK_SPHERES>, k_path_bounce<2, MASK_ALL>,
                  k_path_bounce<4, MASK_SPHERES>, k_path_bounce<4, MASK_ALL>);
    const int gk = grid_kind(P);
    if (gk)
        k = FR_GRID_KERNEL(k_path_bounce, gk);
    k<<<shape.bounce_grid[gk], 256, 0, st>>>(P, S, q);
}

void launch_path_tail(const FrameParams& P, const PathState& S, int iteration,
                      const LaunchShape& shape, cudaStream_t st)
{
    const int q = iteration & 1;
    auto k = pick(P, k_path_tail<2, MASK_SPHERES>, k_path_tail<2, MASK_ALL>,
                  k_path_tail<4, MASK_SPHERES>, k_path_tail<4, MASK_ALL>);
    const int gk = grid_kind(P);
    if (gk)
        k = FR_GRID_KERNEL(k_path_tail, gk);
    k<<<shape.bounce_grid[gk], 256, 0, st>>>(P, S, q);
}

void launch_histogram(const float4* linear, uint32_t n, uint32_t* counts, int num_sms,
                      cudaStream_t st)
{
    const uint32_t blocks = (n + 255u) / 256u;
    const uint32_t cap = uint32_t(num_sms > 0 ? num_sms : 1) * 4u;
    k_histogram<<<blocks < cap ? (blocks ? blocks : 1u) : cap, 256, 0, st>>>(linear, n, counts);
}

void launch_preview(const FrameParams& P, uint32_t aa_n, uint2* hits, cudaStream_t st)
{
    // a group of 32 or 16 lanes per pixel when that divides the samples per pixel (with 2x2
    // anti-aliasing, 4 lanes per pixel were no faster than one thread on the 1M-sphere scene)
    const uint32_t ns = aa_n * aa_n;
    if (P.preview_warp && ns % 16u == 0u) {
        const bool g32 = ns % 32u == 0u;
        const uint64_t threads = uint64_t(P.w) * P.h * (g32 ? 32u : 16u);
        auto k = g32 ? pick(P, k_preview_warp<2, MASK_SPHERES, 32>, k_preview_warp<2, MASK_ALL, 32>,
                            k_preview_warp<4, MASK_SPHERES, 32>, k_preview_warp<4, MASK_ALL, 32>)
                     : pick(P, k_preview_warp<2, MASK_SPHERES, 16>, k_preview_warp<2, MASK_ALL, 16>,
                            k_preview_warp<4, MASK_SPHERES, 16>, k_preview_warp<4, MASK_ALL, 16>);
        if (const int gk = grid_kind(P))
            k = g32 ? (gk == 1   ? k_preview_warp<4, MASK_GRID, 32>
                       : gk == 2 ? k_preview_warp<4, MASK_GRID_PARTS, 32>
                                 : k_preview_warp<4, MASK_GRID_PARTS_NO_MESH, 32>)
                    : (gk == 1   ? k_preview_warp<4, MASK_GRID, 16>
                       : gk == 2 ? k_preview_warp<4, MASK_GRID_PARTS, 16>
                                 : k_preview_warp<4, MASK_GRID_PARTS_NO_MESH, 16>);
        k<<<uint32_t((threads + 255u) / 256u), 256, 0, st>>>(P, aa_n, hits);
        return;
    }
    dim3 block(16, 16);
    dim3 grid((P.w + 15) / 16, (P.h + 15) / 16);
    auto k = pick(P, k_preview<2, MASK_SPHERES>, k_preview<2, MASK_ALL>,
                  k_preview<4, MASK_SPHERES>, k_preview<4, MASK_ALL>);
    if (const int gk = grid_kind(P))
        k = FR_GRID_KERNEL(k_preview, gk);
    k<<<grid, block, 0, st>>>(P, aa_n, hits);
}

}  // namespace fr
