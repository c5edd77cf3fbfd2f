// batch.hpp -- many path renders (frames, scenes, resolutions) traced in shared wavefronts.
//
// A batch is cut into waves. A wave holds whole renders (one tracer's next K samples of every
// pixel) and fits the path state. The kernels find a slot's render by binary search over the
// wave's render table, so the renders of one wave share their queues and launches. The whole
// batch runs as one CUDA graph launch. A graph `while` node steps through the waves. In each
// wave, a nested `while` node alternates shade and extend until the wave's queue is empty.
// Loop state lives in device memory, so the graph is captured once and relaunched for any plan
// that fits its buffers.
#ifndef FR_BATCH_HPP
#define FR_BATCH_HPP

#include <cstdint>

#include <cuda_runtime.h>

#include "render.hpp"

namespace fr {

// One render of a wave: P.batch samples of every pixel, starting at sample P.n_samples.
struct WaveJob {
    FrameParams P;
    uint32_t slot_base;   // first path-state slot of this render in its wave (slots follow the
                          // render's primary work items, so item g has slot slot_base + g)
    uint32_t item_base;   // first primary work item of this render in its wave
    uint32_t pixel_base;  // first fold pixel in its wave
};

// Loop state of one batch launch (device memory).
struct BatchCtl {
    uint32_t n_waves;              // set by the host before each launch
    uint32_t wave;                 // wave being traced
    uint32_t inner;                // shade/extend pairs of the current wave
    uint32_t error;                // 1: a wave reached the iteration cap
    unsigned long long pairs;      // shade/extend pairs over the whole launch
    unsigned long long box_tests;  // traversal counters over the whole launch
    unsigned long long prim_tests;
};

struct BatchDev {
    const WaveJob* jobs;          // renders of all waves; wave w's are [wave_first[w], wave_first[w+1])
    const uint32_t* wave_first;   // [n_waves + 1]
    const uint32_t* wave_items;   // [n_waves] primary work items of each wave
    const uint32_t* wave_pixels;  // [n_waves] fold pixels of each wave
    BatchCtl* ctl;
    PathState S;
};

// Shade/extend pairs after which a wave stops with BatchCtl::error = 1 (a path ends by Russian
// roulette long before; the cap bounds the graph's loop).
constexpr uint32_t BATCH_MAX_PAIRS = 1u << 16;

// Capture the whole-batch graph for trees of `width` (2 or 4) and the geometry types in
// `type_mask` (MASK_GRID: every render traces a sphere grid; MASK_GRID_FUSED: the same with the
// shading folded into the tracing kernels; MASK_GRID_PARTS_FUSED: every render traces a grid over
// its parts, shading folded in; MASK_GRID_PARTS_NO_MESH_FUSED: the same without a mesh), grids
// sized for num_sms. The buffers behind B must outlive the
// graph.
constexpr uint32_t MASK_GRID_FUSED = (1u << 31) | (1u << 30);
constexpr uint32_t MASK_GRID_PARTS_FUSED = MASK_GRID_PARTS | (1u << 30);
constexpr uint32_t MASK_GRID_PARTS_NO_MESH_FUSED = MASK_GRID_PARTS_NO_MESH | (1u << 30);
cudaError_t batch_graph_create(const BatchDev& B, int width, uint32_t type_mask, int num_sms,
                               cudaStream_t capture_stream, cudaGraphExec_t* exec);

}  // namespace fr

#endif
