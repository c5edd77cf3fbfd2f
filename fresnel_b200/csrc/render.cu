// render.cu -- wavefront path tracer and preview tracer kernels.
//
// Path tracer (replaces path_ray_gen/path_closest_hit/path_miss, fresnel/gpu/path.cu:70-171,
// with the CPU loop order of fresnel/cpu/TracerPath.cc:78-255):
//   primary  one thread per pixel: camera ray for this sample, closest hit (shared by all light
//            samples of the pixel, as the CPU path caches it)
//   shade    per queued pixel: hit or miss program of the current light sample; a finished
//            light sample restarts the next one from the cached primary hit in the same thread,
//            so each pixel's radiance accumulates in the reference's order; a finished pixel
//            folds its sample into the running mean (Welford) and writes sRGB; a continuing path
//            is appended to the extension queue (warp-aggregated atomics)
//   extend   persistent warps pull 32 queued rays at a time and find their closest hits
// The host alternates shade/extend until the queue is empty.
//
// Preview (replaces direct_ray_gen/direct_closest_hit, fresnel/gpu/direct.cu, with the CPU
// arithmetic of fresnel/cpu/TracerDirect.cc:59-220): one thread per pixel, aa_n^2 samples.
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

__global__ void __launch_bounds__(256) k_path_primary(FrameParams P, PathState S)
{
    if (blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0 &&
        threadIdx.y == 0) {
        S.ctr[0] = 0;
        S.ctr[1] = 0;
        S.ctr[2] = 0;
    }
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t j = blockIdx.y * blockDim.y + threadIdx.y;
    uint32_t k = blockIdx.z;
    bool valid = (i < P.w) && (j < P.h);
    TraceCount tc;
    if (valid) {
        uint32_t p = j * P.w + i;
        size_t slot = size_t(k) * P.w * P.h + p;
        V3 o, d;
        camera_ray(P.cam, i, j, P.n_samples + k, o, d);
        Hit h = trace_closest(P.scene, o, d, PATH_TNEAR, tc);
        S.prim_o[slot] = f4(o);
        S.prim_d[slot] = f4(d);
        S.prim_hit[slot] = make_uint2(h.geom, h.prim);
        S.ls_depth[slot] = make_uint2(0u, 0u);
        S.att[slot] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
        S.result[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    flush_counts(tc, P.stats + 3);
    uint32_t m = __ballot_sync(0xffffffffu, valid);
    if ((threadIdx.x + threadIdx.y * blockDim.x) % 32 == 0 && m) {
        atomicAdd(P.stats + 0, (unsigned long long)__popc(m));
        atomicAdd(P.stats + 1, (unsigned long long)__popc(m) * P.light_samples);
    }
}

// Fold the batch's samples into the running mean of each pixel, in sample order, then write
// the sRGB output once.
__global__ void __launch_bounds__(256) k_path_fold(FrameParams P, PathState S)
{
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t wh = P.w * P.h;
    if (p >= wh)
        return;
    float4 mean = P.linear[p];
    for (uint32_t k = 0; k < P.batch; ++k)
        mean = welford(P, mean, S.sample[size_t(k) * wh + p], P.n_samples + k);
    write_pixel(P, p, mean.x, mean.y, mean.z, mean.w);
}

// Shade the current path vertex of one slot; returns true if the path needs another closest hit.
__device__ __forceinline__ bool shade_pixel(const FrameParams& P, const PathState& S, uint32_t p)
{
    const uint32_t wh = P.w * P.h;
    const uint32_t k = p / wh;
    const uint32_t pixel = p - k * wh;
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

__global__ void __launch_bounds__(256) k_path_shade(FrameParams P, PathState S, int in_q, int out_q)
{
    if (blockIdx.x == 0 && threadIdx.x == 0)
        S.ctr[2] = 0;  // work counter of the extend kernel that follows
    const uint32_t count = (in_q < 0) ? P.w * P.h * P.batch : S.ctr[in_q];
    const uint32_t* inq = (in_q < 0) ? nullptr : S.queue[in_q];
    uint32_t* outq = S.queue[out_q];
    uint32_t* outc = S.ctr + out_q;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t n_warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t base = warp * 32u; base < count; base += n_warps * 32u) {
        uint32_t idx = base + lane;
        bool push = false;
        uint32_t p = 0;
        if (idx < count) {
            p = inq ? inq[idx] : idx;
            push = shade_pixel(P, S, p);
        }
        uint32_t m = __ballot_sync(0xffffffffu, push);
        if (m) {
            uint32_t at = 0;
            if (lane == 0)
                at = atomicAdd(outc, uint32_t(__popc(m)));
            at = __shfl_sync(0xffffffffu, at, 0);
            if (push)
                outq[at + __popc(m & ((1u << lane) - 1u))] = p;
        }
    }
}

__global__ void __launch_bounds__(256) k_path_extend(FrameParams P, PathState S, int q)
{
    if (blockIdx.x == 0 && threadIdx.x == 0)
        S.ctr[q ^ 1] = 0;  // the other queue was consumed by the shade pass that produced q
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
        uint32_t idx = base + lane;
        if (idx < count) {
            uint32_t p = queue[idx];
            V3 o = xyz(S.ray_o[p]);
            V3 d = xyz(S.ray_d[p]);
            Hit h = trace_closest(P.scene, o, d, PATH_TNEAR, tc);
            S.hit[p] = make_uint2(h.geom, h.prim);
        }
        if (lane == 0)
            atomicAdd(P.stats + 0, (unsigned long long)min(32u, count - base));
    }
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
        float cos_half = cosf(half);
        float ldotr = dot(l, r);
        if (ldotr < cos_half) {
            V3 ax = cross(l, r);
            ax = div_recip(ax, sqrtf(dot(ax, ax)));
            Qt q = from_axis_angle(ax, -acosf(ldotr) + half);
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
            Hit h = trace_closest(P.scene, o, d, 0.0f, tc);  // preview tnear is 0 on the CPU path
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

}  // namespace

LaunchShape path_launch_shape(int num_sms)
{
    int per_sm_shade = 0, per_sm_extend = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_shade, k_path_shade, 256, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_extend, k_path_extend, 256, 0);
    LaunchShape s;
    s.shade_grid = num_sms * (per_sm_shade > 0 ? per_sm_shade : 1);
    s.extend_grid = num_sms * (per_sm_extend > 0 ? per_sm_extend : 1);
    return s;
}

void launch_path_primary(const FrameParams& P, const PathState& S, cudaStream_t st)
{
    dim3 block(16, 16);
    dim3 grid((P.w + 15) / 16, (P.h + 15) / 16, P.batch);
    k_path_primary<<<grid, block, 0, st>>>(P, S);
}

void launch_path_fold(const FrameParams& P, const PathState& S, cudaStream_t st)
{
    k_path_fold<<<(P.w * P.h + 255) / 256, 256, 0, st>>>(P, S);
}

void launch_path_shade(const FrameParams& P, const PathState& S, int iteration,
                       const LaunchShape& shape, cudaStream_t st)
{
    int in_q = iteration == 0 ? -1 : ((iteration - 1) & 1);
    k_path_shade<<<shape.shade_grid, 256, 0, st>>>(P, S, in_q, iteration & 1);
}

void launch_path_extend(const FrameParams& P, const PathState& S, int iteration,
                        const LaunchShape& shape, cudaStream_t st)
{
    k_path_extend<<<shape.extend_grid, 256, 0, st>>>(P, S, iteration & 1);
}

void launch_preview(const FrameParams& P, uint32_t aa_n, uint2* hits, cudaStream_t st)
{
    dim3 block(16, 16);
    dim3 grid((P.w + 15) / 16, (P.h + 15) / 16);
    k_preview<<<grid, block, 0, st>>>(P, aa_n, hits);
}

}  // namespace fr
