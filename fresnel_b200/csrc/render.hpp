// render.hpp -- host interface of the path-tracing and preview kernels.
#ifndef FR_RENDER_HPP
#define FR_RENDER_HPP

#include <cstdint>

#include <cuda_runtime.h>

#include "engine.cuh"

namespace fr {

// Everything one render reads, passed by value to every kernel of that render.
struct FrameParams {
    SceneDev scene;
    int bvh_width;       // 2 or 4 (selects the kernel instantiation)
    int persistent;      // 4-wide trees: persistent warps with per-lane refill (1) or not (0)
    uint32_t type_mask;  // geometry types enabled in the scene (selects the instantiation)
    CamK cam;
    LightsK lights;
    C3 bg;
    float bg_alpha;
    uint32_t w, h;
    uint32_t n_samples;      // 1-based sample number of the batch's first render
    uint32_t batch;          // samples traced together (slot = k * w * h + pixel)
    uint32_t light_samples;  // light paths per primary ray
    uint32_t tile_log2;      // primary work in 2^tile_log2-pixel square tiles (path_device.cuh)
    int shade_blocks;        // 0: shade kernel as compiled; 3 or 4: register-limited variants
    int packet;              // 1: primary rays traced warp-cooperatively (4-wide trees)
    int refill;              // 1: extension rays with per-lane refill where refill_geom != -1
    int preview_warp;        // 1: Preview with 32k samples per pixel traces one pixel per warp
    int refill_geom;         // -2: the scene's combined tree; >= 0: its one enabled geometry;
                             // -1: several per-geometry trees (refill not available)
    int highlight;
    C3 hl_color;
    float4* linear;     // [h][w] running mean, linear RGBA
    uint32_t* srgb;     // [h][w] RGBA8
    unsigned long long* stats;  // [0] rays, [1] paths, [2] dropped, [3] box tests, [4] prim tests
};

// Wavefront state of the path tracer (structure of arrays, one entry per path slot; a batch of
// K samples uses K * w * h slots, slot = k * w * h + pixel).
struct PathState {
    float4* prim_o;     // primary ray, shared by the light samples of a pixel sample
    float4* prim_d;
    uint2* prim_hit;    // (geometry or MISS, primitive)
    float4* ray_o;      // next extension ray
    float4* ray_d;
    float4* att;        // path throughput
    float4* result;     // radiance summed over the pixel's light samples so far
    uint2* ls_depth;    // (light sample, depth)
    uint2* hit;         // closest hit of the last extension ray
    float4* sample;     // the finished pixel sample of each slot (folded in order at the end)
    uint32_t* queue[2];
    uint32_t* ctr;      // [0], [1] queue lengths, [2] extend and [3] primary work counters
};

struct LaunchShape {
    int shade_grid;
    int shade_grid_occ[2];   // shade kernel compiled for 3|4 blocks per SM
    int refill_grid[2];      // extension kernel with per-lane refill [spheres only|all types]
    int extend_grid[4];      // [width 2|4][spheres only|all types]
    int extend_grid_sphere_grid;  // scenes traced through a uniform sphere grid
    int extend_grid_parts_grid[2];  // k_path_extend over a grid of parts [with|without meshes]
    int refill_grid_sphere_grid;  // the same with per-lane refill
    int bounce_grid[4];           // fused extension and shading (k_path_bounce)
                                  // [BVH|sphere grid|parts grid|parts grid without meshes]
    int persistent_grid[2];  // 4-wide persistent extend kernel [spheres only|all types]
    int primary_grid[2];     // 4-wide persistent primary kernel [spheres only|all types]
};

LaunchShape path_launch_shape(int num_sms);

// One batch of P.batch TracerPath::render samples: primary rays for every slot ...
void launch_path_primary(const FrameParams& P, const PathState& S, const LaunchShape& shape,
                         cudaStream_t st);
// ... then iteration i of shade (queue in = q[(i+1)&1], out = q[i&1]; the primary kernel fills
// q[1] with the slots whose primary ray hit) and extend (q[i&1]) until the output queue is
// empty; both queue lengths are zero between batches ...
void launch_path_shade(const FrameParams& P, const PathState& S, int iteration,
                       const LaunchShape& shape, cudaStream_t st);
void launch_path_extend(const FrameParams& P, const PathState& S, int iteration,
                        const LaunchShape& shape, cudaStream_t st);
// Or, instead of the primary pass and the first shade pass: primary rays shaded at once, the
// continuing paths in queue 0 (all four counters must be zero); the loop then starts with the
// extend of iteration 0.
void launch_path_primary_shade(const FrameParams& P, const PathState& S, cudaStream_t st);
// With the primary pass shaded at once, iteration i may instead be one fused bounce: the rays of
// q[i&1] traced and shaded, continuing paths into q[(i&1)^1] (whose length and ctr[2] must be
// zero).
void launch_path_bounce(const FrameParams& P, const PathState& S, int iteration,
                        const LaunchShape& shape, cudaStream_t st);
// The remaining bounces of every path in queue (iteration & 1) in one launch (k_path_tail).
void launch_path_tail(const FrameParams& P, const PathState& S, int iteration,
                      const LaunchShape& shape, cudaStream_t st);
// ... then fold the batch's samples into each pixel's running mean, in sample order.
void launch_path_fold(const FrameParams& P, const PathState& S, cudaStream_t st);
// Diagnostic comparison of the two 4-wide traversal forms (sphere scenes).
void launch_traversal_compare(const SceneDev& sc, const float* rays, uint32_t n, uint32_t* out,
                              cudaStream_t st);
// Tracer.histogram: counts[HIST_BINS][4] (lightness, R, G, B) of the visible pixels of a
// linear RGBA image of n pixels; counts must be zeroed first.
constexpr uint32_t HIST_BINS = 512;
void launch_histogram(const float4* linear, uint32_t n, uint32_t* counts, int num_sms,
                      cudaStream_t st);
// TracerDirect::render
void launch_preview(const FrameParams& P, uint32_t aa_n, uint2* hits, cudaStream_t st);

}  // namespace fr

#endif
