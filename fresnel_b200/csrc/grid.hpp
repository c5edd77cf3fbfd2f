// grid.hpp -- uniform grids, the acceleration structure the renderers use instead of a BVH for
// evenly spread primitives (device option "accel"): over the spheres of a scene's one geometry,
// or over the primitives of all its enabled geometries (the parts a combined tree would hold).
#ifndef FR_GRID_HPP
#define FR_GRID_HPP

#include "bvh.hpp"

namespace fr {

struct GridBuffers {
    DevArray<uint32_t> cell_start;   // n_cells + 1 offsets into the references
    DevArray<float4> ref_sphere;     // sphere grid, per reference: the sphere (x, y, z, r)
    DevArray<uint32_t> ref_prim;     // per reference: the primitive's index in its geometry
    DevArray<float4> ref_data;       // parts grid, per reference: 2 float4 of the primitive's
                                     // record (laid out as a combined tree's leaf slot)
    DevArray<uint32_t> ref_geom;     // parts grid, per reference: scene geometry index
    DevArray<uint32_t> prim_count;   // build temporaries kept between builds: cells per primitive
    DevArray<uint32_t> prim_offset;  // and their exclusive prefix sum
    DevArray<float4> box_lo;         // parts grid build temporaries: primitive boxes
    DevArray<float4> box_hi;
    uint32_t n_cells = 0;            // 0: no grid
    uint32_t n_refs = 0;
    bool parts = false;              // built over parts (ref_data, ref_geom) or spheres
    uint32_t dims[3] = {0, 0, 0};
    float lo[3] = {0, 0, 0};
    float hi[3] = {0, 0, 0};
    float cell[3] = {0, 0, 0};
};

struct GridParams {
    float cells_per_prim = 1.5f;         // cells per primitive (sets the cell size)
    int mode = 2;                        // 1: build whenever the primitives allow; 2: only when
                                         //    the grid is expected to beat the BVH
    // Mode 2 thresholds.  Measured on sphere scenes of 100 to 1M spheres at densities from the
    // 1M-sphere scene's down to one sphere per 4e5 volume units, the grid traced every one of
    // them faster than the BVH (1.4x to 2x), and scenes of spheres and bonds of 1e4 to 2e6
    // primitives 1.5x to 1.9x faster and the mixed scene 1.15x faster; what keeps the BVH is
    // clustering.
    uint32_t min_prims = 1;              // mode 2: fewer primitives keep the BVH
    float max_cells_per_ray = 1024.0f;   // mode 2: estimated cells a ray crosses before a hit
                                         //    or before it leaves the grid
    uint32_t max_refs_per_cell = 64;     // mode 2: a fuller cell means clustered primitives
    uint32_t max_cells_per_prim = 4096;  // any mode: a primitive spanning more stops the build
};

// Outcome of one build attempt.
struct GridReport {
    bool built = false;
    const char* reason = "";   // why the grid was not built
    uint32_t n_valid = 0;      // spheres with a finite, non-empty box
    double cells_per_ray = 0;  // estimated cells crossed per ray before a hit or the grid's exit
    uint32_t max_refs = 0;     // fullest cell
};

// Builds the grid of the n spheres (positions [n][3], radii [n]) on `st` and waits for it.
// Returns a CUDA error only for device failures; a grid that should not be used (mode 2 rules,
// a sphere spanning too many cells, no valid sphere) leaves out.n_cells == 0 with
// report.built == false and report.reason set.
cudaError_t build_grid(const float* position, const float* radius, uint32_t n,
                       const GridParams& gp, GridBuffers& out, Scratch& scratch, cudaStream_t st,
                       GridReport& report);

// Builds the grid over the n = in.first[in.n_parts] primitives of the parts of `in` (their boxes
// as the tree builds compute them), with the same rules; the references hold leaf-slot records
// (out.parts = true).
cudaError_t build_grid(const PartsInput& in, uint32_t n, const GridParams& gp, GridBuffers& out,
                       Scratch& scratch, cudaStream_t st, GridReport& report);

}  // namespace fr

#endif
