// batch.cu -- kernels and CUDA graph of the batched path tracer (see batch.hpp).
//
// The per-slot work is the single-render path tracer's (path_device.cuh: shade_pixel, welford,
// write_pixel; engine.cuh: trace_closest), so a render gives the same image alone or in a
// batch. What changes is how a thread finds its render: primary work items, queued slots and fold
// pixels carry indices into the current wave, and a binary search over the wave's render table
// maps them to the render (its scene, camera, lights, outputs and sample numbers).
#include "batch.hpp"
#include "path_device.cuh"

namespace fr {

namespace {

// The render of [lo, hi) whose base (member M) is the largest one <= key (bases ascend and
// jobs[lo].*M <= key).
template <uint32_t WaveJob::*M>
__device__ __forceinline__ uint32_t find_job(const WaveJob* jobs, uint32_t lo, uint32_t hi,
                                             uint32_t key)
{
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (jobs[mid].*M <= key)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

__global__ void k_batch_start(BatchCtl* ctl, cudaGraphConditionalHandle outer)
{
    ctl->wave = 0;
    ctl->inner = 0;
    ctl->error = 0;
    ctl->pairs = 0;
    ctl->box_tests = 0;
    ctl->prim_tests = 0;
    cudaGraphSetConditional(outer, ctl->n_waves > 0u ? 1u : 0u);
}

__global__ void k_wave_begin(BatchDev B, cudaGraphConditionalHandle inner)
{
    B.S.ctr[0] = 0;
    B.S.ctr[1] = 0;
    B.S.ctr[2] = 0;
    B.S.ctr[3] = 0;
    B.ctl->inner = 0;
    cudaGraphSetConditional(inner, 1u);
}

// Primary rays of the wave, grid-stride over its work items (each render's items in
// primary_item order; a render has a multiple of 64 items, so a warp never spans two renders).
template <int WIDTH, uint32_t MASK>
__global__ void __launch_bounds__(256) k_batch_primary(BatchDev B)
{
    const PathState& S = B.S;
    const uint32_t w = B.ctl->wave;
    const uint32_t f0 = B.wave_first[w], f1 = B.wave_first[w + 1];
    const uint32_t n_items = B.wave_items[w];
    TraceCount tc;
    const uint32_t stride = gridDim.x * blockDim.x;
    // n_items is a multiple of 64, so whole warps enter and leave the loop together
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g - lane_id() < n_items;
         g += stride) {
        const WaveJob& J = B.jobs[find_job<&WaveJob::item_base>(B.jobs, f0, f1, g)];
        const FrameParams& P = J.P;
        const PrimaryItem it = primary_item(g - J.item_base, P.w, P.h, P.batch, P.tile_log2);
        bool push = false;
        uint32_t slot = 0;
        if (it.valid) {
            slot = J.slot_base + (g - J.item_base);
            push = primary_ray<WIDTH, MASK>(P, S, it, slot, tc);
        }
        push_primary(S, push, slot);
        const uint32_t mv = __ballot_sync(0xffffffffu, it.valid);
        if (lane_id() == 0 && mv) {
            atomicAdd(P.stats + 0, (unsigned long long)__popc(mv));
            atomicAdd(P.stats + 1, (unsigned long long)__popc(mv) * P.light_samples);
        }
    }
    flush_counts(tc, &B.ctl->box_tests);
}

__global__ void __launch_bounds__(256) k_batch_shade(BatchDev B, int in_q, int out_q)
{
    const PathState& S = B.S;
    if (blockIdx.x == 0 && threadIdx.x == 0)
        S.ctr[2] = 0;  // work counter of the extend kernel that follows
    const uint32_t w = B.ctl->wave;
    const uint32_t f0 = B.wave_first[w], f1 = B.wave_first[w + 1];
    const uint32_t count = S.ctr[in_q];
    const uint32_t* inq = S.queue[in_q];
    uint32_t* outq = S.queue[out_q];
    uint32_t* outc = S.ctr + out_q;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t n_warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t base = warp * 32u; base < count; base += n_warps * 32u) {
        const uint32_t idx = base + lane;
        bool push = false;
        uint32_t p = 0;
        if (idx < count) {
            p = ld_cs(inq + (idx));
            const WaveJob& J = B.jobs[find_job<&WaveJob::slot_base>(B.jobs, f0, f1, p)];
            push = shade_pixel(J.P, S, p, p - J.slot_base);
        }
        const uint32_t m = __ballot_sync(0xffffffffu, push);
        if (m) {
            uint32_t at = 0;
            if (lane == 0)
                at = atomicAdd(outc, uint32_t(__popc(m)));
            at = __shfl_sync(0xffffffffu, at, 0);
            if (push)
                st_cs(outq + (at + __popc(m & ((1u << lane) - 1u))), p);
        }
    }
}

template <int WIDTH, uint32_t MASK>
__global__ void __launch_bounds__(256) k_batch_extend(BatchDev B, int q)
{
    const PathState& S = B.S;
    if (blockIdx.x == 0 && threadIdx.x == 0)
        S.ctr[q ^ 1] = 0;  // the other queue was consumed by the shade pass that produced q
    const uint32_t w = B.ctl->wave;
    const uint32_t f0 = B.wave_first[w], f1 = B.wave_first[w + 1];
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
        const bool act = idx < count;
        uint32_t jb = 0;
        if (act) {
            const uint32_t p = ld_cs(queue + (idx));
            jb = find_job<&WaveJob::slot_base>(B.jobs, f0, f1, p);
            const V3 o = xyz(ld_cs(S.ray_o + (p)));
            const V3 d = xyz(ld_cs(S.ray_d + (p)));
            Hit h = trace_closest<WIDTH, MASK>(B.jobs[jb].P.scene, o, d, PATH_TNEAR, tc);
            st_cs(S.hit + (p), make_uint2(h.geom, h.prim));
        }
        // rays per render, one atomic per render present in the warp
        const uint32_t am = __ballot_sync(0xffffffffu, act);
        if (act) {
            const uint32_t same = __match_any_sync(am, jb);
            if (lane == uint32_t(__ffs(same) - 1))
                atomicAdd(B.jobs[jb].P.stats + 0, (unsigned long long)__popc(same));
        }
    }
    flush_counts(tc, &B.ctl->box_tests);
}

// Primary rays of the wave shaded at once (k_path_primary_shade), continuing paths into queue 0.
template <int WIDTH, uint32_t MASK>
__global__ void __launch_bounds__(256, fused_blocks(MASK)) k_batch_primary_shade(BatchDev B)
{
    const PathState& S = B.S;
    const uint32_t w = B.ctl->wave;
    const uint32_t f0 = B.wave_first[w], f1 = B.wave_first[w + 1];
    const uint32_t n_items = B.wave_items[w];
    TraceCount tc;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g - lane_id() < n_items;
         g += stride) {
        const WaveJob& J = B.jobs[find_job<&WaveJob::item_base>(B.jobs, f0, f1, g)];
        const FrameParams& P = J.P;
        const PrimaryItem it = primary_item(g - J.item_base, P.w, P.h, P.batch, P.tile_log2);
        bool push = false;
        uint32_t slot = 0;
        if (it.valid) {
            slot = J.slot_base + (g - J.item_base);
            push = primary_shade<WIDTH, MASK>(P, S, it, slot, tc);
        }
        push_queue(S, 0, push, slot);
        const uint32_t mv = __ballot_sync(0xffffffffu, it.valid);
        if (lane_id() == 0 && mv) {
            atomicAdd(P.stats + 0, (unsigned long long)__popc(mv));
            atomicAdd(P.stats + 1, (unsigned long long)__popc(mv) * P.light_samples);
        }
    }
    flush_counts(tc, &B.ctl->box_tests);
}

// One bounce of the wave (k_path_bounce): the rays of queue q traced and shaded, continuing paths
// into queue q ^ 1, whose length and the work counter are cleared before the launch.
template <int WIDTH, uint32_t MASK>
__global__ void __launch_bounds__(256, fused_blocks(MASK)) k_batch_bounce(BatchDev B, int q)
{
    const PathState& S = B.S;
    const uint32_t w = B.ctl->wave;
    const uint32_t f0 = B.wave_first[w], f1 = B.wave_first[w + 1];
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
        const bool act = idx < count;
        uint32_t jb = 0, p = 0;
        bool push = false;
        if (act) {
            p = ld_cs(queue + (idx));
            jb = find_job<&WaveJob::slot_base>(B.jobs, f0, f1, p);
            push = bounce<WIDTH, MASK>(B.jobs[jb].P, S, p, p - B.jobs[jb].slot_base, tc);
        }
        push_queue(S, q ^ 1, push, p);
        // rays per render, one atomic per render present in the warp
        const uint32_t am = __ballot_sync(0xffffffffu, act);
        if (act) {
            const uint32_t same = __match_any_sync(am, jb);
            if (lane == uint32_t(__ffs(same) - 1))
                atomicAdd(B.jobs[jb].P.stats + 0, (unsigned long long)__popc(same));
        }
    }
    flush_counts(tc, &B.ctl->box_tests);
}

// The remaining bounces of every path of queue q in one launch (k_path_tail): each lane follows
// its path to the end, then takes the next one (idle lanes share one atomic); a path's rays are
// added to its render's count when it ends.  The work counter must be zero at launch; no queue is
// written.
template <int WIDTH, uint32_t MASK>
__global__ void __launch_bounds__(256, fused_blocks(MASK)) k_batch_tail(BatchDev B, int q)
{
    const PathState& S = B.S;
    const uint32_t w = B.ctl->wave;
    const uint32_t f0 = B.wave_first[w], f1 = B.wave_first[w + 1];
    const uint32_t count = S.ctr[q];
    const uint32_t* queue = S.queue[q];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t below = (1u << lane) - 1u;
    TraceCount tc;
    bool active = false, exhausted = false;
    uint32_t p = 0, jb = 0, guard = 0;
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
                    jb = find_job<&WaveJob::slot_base>(B.jobs, f0, f1, p);
                    active = true;
                    guard = TAIL_MAX_DEPTH;
                    rays = 0;
                }
            }
        }
        if (__ballot_sync(0xffffffffu, active) == 0u)
            break;
        if (active) {
            ++rays;
            const FrameParams& P = B.jobs[jb].P;
            bool more = bounce<WIDTH, MASK>(P, S, p, p - B.jobs[jb].slot_base, tc);
            if (more && --guard == 0u) {
                atomicOr(P.scene.status, ERR_ITERATION_CAP);
                more = false;
            }
            if (!more) {
                atomicAdd(P.stats + 0, rays);
                active = false;
            }
        }
    }
    flush_counts(tc, &B.ctl->box_tests);
}

__global__ void k_wave_begin_flat(BatchDev B)
{
    B.S.ctr[0] = 0;
    B.S.ctr[1] = 0;
    B.S.ctr[2] = 0;
    B.S.ctr[3] = 0;
    B.ctl->inner = 0;
}

// Before a fused bounce: the output queue q and the work counter start at zero.
__global__ void k_clear_queue(BatchDev B, int q)
{
    B.S.ctr[q] = 0;
    B.S.ctr[2] = 0;
}

__global__ void k_inner_cond(BatchDev B, cudaGraphConditionalHandle inner, int q_next)
{
    BatchCtl* c = B.ctl;
    c->inner += 1u;
    c->pairs += 1u;
    bool more = B.S.ctr[q_next] != 0u;
    if (more && c->inner >= BATCH_MAX_PAIRS) {
        c->error = 1u;
        more = false;
    }
    cudaGraphSetConditional(inner, more ? 1u : 0u);
}

// Fold each render's samples of the wave into its running mean, in sample order (k_path_fold).
__global__ void __launch_bounds__(256) k_batch_fold(BatchDev B)
{
    const PathState& S = B.S;
    const uint32_t w = B.ctl->wave;
    const uint32_t f0 = B.wave_first[w], f1 = B.wave_first[w + 1];
    const uint32_t n = B.wave_pixels[w];
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const WaveJob& J = B.jobs[find_job<&WaveJob::pixel_base>(B.jobs, f0, f1, q)];
        const FrameParams& P = J.P;
        const uint32_t lp = q - J.pixel_base;
        const uint32_t j = lp / P.w;
        const uint32_t base = J.slot_base + pixel_slot(lp - j * P.w, j, P.w, P.batch, P.tile_log2);
        float4 mean = P.linear[lp];
        for (uint32_t k = 0; k < P.batch; ++k)
            mean = welford(P, mean, S.sample[base + k], P.n_samples + k);
        write_pixel(P, lp, mean.x, mean.y, mean.z, mean.w);
    }
}

__global__ void k_wave_end(BatchDev B, cudaGraphConditionalHandle outer)
{
    BatchCtl* c = B.ctl;
    c->wave += 1u;
    cudaGraphSetConditional(outer, (c->wave < c->n_waves && c->error == 0u) ? 1u : 0u);
}

template <class K> int grid_for(K kernel, int num_sms, int threads)
{
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, 0);
    return num_sms * (n > 0 ? n : 1);
}

template <int WIDTH, uint32_t MASK> struct Kernels {
    static void primary(const BatchDev& B, int grid, cudaStream_t s)
    {
        k_batch_primary<WIDTH, MASK><<<grid, 256, 0, s>>>(B);
    }
    static void extend(const BatchDev& B, int q, int grid, cudaStream_t s)
    {
        k_batch_extend<WIDTH, MASK><<<grid, 256, 0, s>>>(B, q);
    }
    static int primary_grid(int sms) { return grid_for(k_batch_primary<WIDTH, MASK>, sms, 256); }
    static int extend_grid(int sms) { return grid_for(k_batch_extend<WIDTH, MASK>, sms, 256); }
};

// Appends a `while` node after the capture's current leaves and returns its body graph.
cudaError_t add_while(cudaStream_t s, cudaGraphConditionalHandle h, cudaGraph_t* body)
{
    cudaStreamCaptureStatus status;
    cudaGraph_t graph = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t n_deps = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(s, &status, nullptr, &graph, &deps, &n_deps);
    if (e != cudaSuccess)
        return e;
    if (status != cudaStreamCaptureStatusActive)
        return cudaErrorStreamCaptureInvalidated;
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    if ((e = cudaGraphAddNode(&node, graph, deps, n_deps, &cp)) != cudaSuccess)
        return e;
    *body = cp.conditional.phGraph_out[0];
    return cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies);
}

cudaGraph_t capturing_graph(cudaStream_t s)
{
    cudaStreamCaptureStatus status;
    cudaGraph_t graph = nullptr;
    if (cudaStreamGetCaptureInfo(s, &status, nullptr, &graph, nullptr, nullptr) != cudaSuccess)
        return nullptr;
    return graph;
}

// FUSED: shading folded into the tracing kernels (k_batch_primary_shade, k_batch_bounce), as the
// single-render path does for sphere-grid scenes.
template <int WIDTH, uint32_t MASK, bool FUSED = false>
cudaError_t capture(const BatchDev& B, int num_sms, cudaStream_t s0, cudaGraphExec_t* exec)
{
    using KS = Kernels<WIDTH, MASK>;
    const int g_primary = FUSED ? grid_for(k_batch_primary_shade<WIDTH, MASK>, num_sms, 256)
                                : KS::primary_grid(num_sms);
    const int g_extend = FUSED ? grid_for(k_batch_bounce<WIDTH, MASK>, num_sms, 256)
                               : KS::extend_grid(num_sms);
    const int g_shade = grid_for(k_batch_shade, num_sms, 256);
    const int g_fold = num_sms * 8;

    cudaStream_t s1 = nullptr, s2 = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&s1, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking);
    cudaGraph_t top = nullptr;
    bool c0 = false, c1 = false, c2 = false;
    auto keep = [&](cudaError_t x) {
        if (e == cudaSuccess)
            e = x;
        return e == cudaSuccess;
    };
    if (e == cudaSuccess && keep(cudaStreamBeginCapture(s0, cudaStreamCaptureModeRelaxed))) {
        c0 = true;
        cudaGraph_t g = capturing_graph(s0);
        cudaGraphConditionalHandle h_outer;
        cudaGraph_t outer_body = nullptr;
        if (keep(g ? cudaGraphConditionalHandleCreate(&h_outer, g, 0, 0) : cudaErrorUnknown)) {
            k_batch_start<<<1, 1, 0, s0>>>(B.ctl, h_outer);
            if (keep(cudaGetLastError()) && keep(add_while(s0, h_outer, &outer_body))) {
                cudaGraphConditionalHandle h_inner;
                cudaGraph_t inner_body = nullptr;
                if (FUSED &&
                    keep(cudaStreamBeginCaptureToGraph(s1, outer_body, nullptr, nullptr, 0,
                                                       cudaStreamCaptureModeRelaxed))) {
                    // a wave without a bounce loop: two bounce launches while the queues are
                    // long (queue 0 -> 1 -> 0; the fused primary kernel fills queue 0), then
                    // every path's remaining bounces in one launch (k_batch_tail).  (One bounce
                    // launch before the tail, the single-render default, was slower here: the
                    // 64-frame set 151.7 against 143.0 ms.)
                    c1 = true;
                    k_wave_begin_flat<<<1, 1, 0, s1>>>(B);
                    k_batch_primary_shade<WIDTH, MASK><<<g_primary, 256, 0, s1>>>(B);
                    k_clear_queue<<<1, 1, 0, s1>>>(B, 1);
                    k_batch_bounce<WIDTH, MASK><<<g_extend, 256, 0, s1>>>(B, 0);
                    k_clear_queue<<<1, 1, 0, s1>>>(B, 0);
                    k_batch_bounce<WIDTH, MASK><<<g_extend, 256, 0, s1>>>(B, 1);
                    k_clear_queue<<<1, 1, 0, s1>>>(B, 1);
                    k_batch_tail<WIDTH, MASK><<<g_extend, 256, 0, s1>>>(B, 0);
                    k_batch_fold<<<g_fold, 256, 0, s1>>>(B);
                    k_wave_end<<<1, 1, 0, s1>>>(B, h_outer);
                    keep(cudaGetLastError());
                } else if (!FUSED &&
                           keep(cudaGraphConditionalHandleCreate(&h_inner, outer_body, 0, 0)) &&
                           keep(cudaStreamBeginCaptureToGraph(s1, outer_body, nullptr, nullptr, 0,
                                                              cudaStreamCaptureModeRelaxed))) {
                    c1 = true;
                    k_wave_begin<<<1, 1, 0, s1>>>(B, h_inner);
                    KS::primary(B, g_primary, s1);
                    if (keep(cudaGetLastError()) && keep(add_while(s1, h_inner, &inner_body)) &&
                        keep(cudaStreamBeginCaptureToGraph(s2, inner_body, nullptr, nullptr, 0,
                                                           cudaStreamCaptureModeRelaxed))) {
                        c2 = true;
                        // two iterations per pass: queue 1 -> 0, then 0 -> 1 (the primary
                        // kernel fills queue 1)
                        k_batch_shade<<<g_shade, 256, 0, s2>>>(B, 1, 0);
                        KS::extend(B, 0, g_extend, s2);
                        k_batch_shade<<<g_shade, 256, 0, s2>>>(B, 0, 1);
                        KS::extend(B, 1, g_extend, s2);
                        k_inner_cond<<<1, 1, 0, s2>>>(B, h_inner, 1);
                        keep(cudaGetLastError());
                    }
                    if (c2) {
                        keep(cudaStreamEndCapture(s2, &inner_body));
                        c2 = false;
                    }
                    k_batch_fold<<<g_fold, 256, 0, s1>>>(B);
                    k_wave_end<<<1, 1, 0, s1>>>(B, h_outer);
                    keep(cudaGetLastError());
                }
                if (c1) {
                    keep(cudaStreamEndCapture(s1, &outer_body));
                    c1 = false;
                }
            }
        }
    }
    if (c0)
        keep(cudaStreamEndCapture(s0, &top));
    if (e == cudaSuccess)
        e = cudaGraphInstantiate(exec, top, 0);
    if (top)
        cudaGraphDestroy(top);
    if (s1)
        cudaStreamDestroy(s1);
    if (s2)
        cudaStreamDestroy(s2);
    return e;
}

}  // namespace

cudaError_t batch_graph_create(const BatchDev& B, int width, uint32_t type_mask, int num_sms,
                               cudaStream_t capture_stream, cudaGraphExec_t* exec)
{
    if (type_mask == MASK_GRID_FUSED)  // every render traces a sphere grid, shading fused
        return capture<4, MASK_GRID, true>(B, num_sms, capture_stream, exec);
    if (type_mask == MASK_GRID)  // every render of the batch traces a sphere grid
        return capture<4, MASK_GRID>(B, num_sms, capture_stream, exec);
    if (type_mask == MASK_GRID_PARTS_FUSED)  // every render traces a grid over its parts
        return capture<4, MASK_GRID_PARTS, true>(B, num_sms, capture_stream, exec);
    if (type_mask == MASK_GRID_PARTS_NO_MESH_FUSED)  // the same, no mesh among the parts
        return capture<4, MASK_GRID_PARTS_NO_MESH, true>(B, num_sms, capture_stream, exec);
    // renders tracing trees, sphere grids or grids over parts (MASK_MAY_PARTS)
    const bool spheres_only = (type_mask & ~MASK_SPHERES) == 0u;
    constexpr uint32_t SPH = MASK_SPHERES | MASK_MAY_PARTS, ALL = MASK_ALL | MASK_MAY_PARTS;
    if (width == 4)
        return spheres_only ? capture<4, SPH>(B, num_sms, capture_stream, exec)
                            : capture<4, ALL>(B, num_sms, capture_stream, exec);
    return spheres_only ? capture<2, SPH>(B, num_sms, capture_stream, exec)
                        : capture<2, ALL>(B, num_sms, capture_stream, exec);
}

}  // namespace fr
