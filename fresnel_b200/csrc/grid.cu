// grid.cu -- construction of the uniform grids traced by trace_grid and trace_grid_parts
// (engine.cuh): over the spheres of one geometry, or over the primitives of the scene's parts.
//
// Steps, all on the stream of the build:
//   1. bounding box of every primitive (a sphere's centre +- radius, as the reference computes
//      it, padded as the BVH builder pads its boxes; a part's primitive box as the tree builds
//      compute it), their union, the number of valid primitives and the sum of their mean
//      cross-sections / pi (r^2 for a sphere, surface / (4 pi) for a box) (one pass with warp
//      reductions and atomics);
//   2. on the host: the cell size (cells_per_prim cells per primitive over the union's volume)
//      and, in automatic mode, the estimated number of cells a ray crosses before it meets a
//      primitive or leaves the grid, min(mean free path / cell size, nx + ny + nz) with mean
//      free path = volume / (n pi <r^2>);
//   3. cells per primitive, their prefix sum, then one (cell, primitive) pair per covered cell
//      written in primitive order and radix-sorted by cell (stable, so each cell lists its
//      primitives in index order and the build is deterministic);
//   4. references per cell, their prefix sum (cell_start), the fullest cell, and the reference
//      records: for spheres a copy of the sphere (x, y, z, r) and its index; for parts the
//      record, geometry and index of a combined tree's leaf slot.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "grid.hpp"

namespace fr {

namespace {

__device__ __forceinline__ uint32_t f2o(float f)
{
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

float o2f_host(uint32_t u)
{
    uint32_t v = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
    float f;
    std::memcpy(&f, &v, sizeof(f));
    return f;
}

struct SBox {
    float lo[3], hi[3];
    bool ok;
};

// The sphere's bounding box (fresnel/cpu/GeometrySphere.cc:60-73: centre - r to centre + r); a
// box that is not finite or has lower > upper (negative radius) is not valid, as for the BVH.
// Valid boxes get the BVH builder's padding.
__device__ __forceinline__ SBox sphere_box(const float* pos, const float* rad, uint32_t i)
{
    SBox b;
    const float r = rad[i];
    for (int k = 0; k < 3; ++k) {
        const float c = pos[3 * size_t(i) + k];
        b.lo[k] = c - r;
        b.hi[k] = c + r;
    }
    b.ok = true;
    for (int k = 0; k < 3; ++k)
        b.ok = b.ok && isfinite(b.lo[k]) && isfinite(b.hi[k]) && b.lo[k] <= b.hi[k];
    if (b.ok) {
        float scale = 0.0f, ext = 0.0f;
        for (int k = 0; k < 3; ++k) {
            scale = fmaxf(scale, fmaxf(fabsf(b.lo[k]), fabsf(b.hi[k])));
            ext += b.hi[k] - b.lo[k];
        }
        const float pad = 1e-5f * scale + 1e-6f * ext + 1e-30f;
        for (int k = 0; k < 3; ++k) {
            b.lo[k] -= pad;
            b.hi[k] += pad;
        }
    }
    return b;
}

// The primitives a grid is built over: a box per primitive (ok = false: left out) and its mean
// cross-section / pi.
struct SphereSource {
    const float* pos;
    const float* rad;
    __device__ __forceinline__ SBox box(uint32_t i) const { return sphere_box(pos, rad, i); }
    __device__ __forceinline__ double xsec(uint32_t i) const
    {
        const double r = double(rad[i]);
        return r * r;
    }
};

struct BoxSource {
    const float4* lo;
    const float4* hi;
    __device__ __forceinline__ SBox box(uint32_t i) const
    {
        const float4 a = lo[i], b = hi[i];
        SBox r;
        r.lo[0] = a.x;
        r.lo[1] = a.y;
        r.lo[2] = a.z;
        r.hi[0] = b.x;
        r.hi[1] = b.y;
        r.hi[2] = b.z;
        r.ok = a.x <= b.x && a.y <= b.y && a.z <= b.z;  // the tree builds' empty box fails this
        return r;
    }
    // a convex body's mean projected area is a quarter of its surface (Cauchy)
    __device__ __forceinline__ double xsec(uint32_t i) const
    {
        const float4 a = lo[i], b = hi[i];
        const double ex = double(b.x) - a.x, ey = double(b.y) - a.y, ez = double(b.z) - a.z;
        return 2.0 * (ex * ey + ey * ez + ez * ex) / (4.0 * 3.14159265358979323846);
    }
};

struct Shape {
    float lo[3], ih[3];
    uint32_t n[3];
};

__device__ __forceinline__ int cell_index(float x, const Shape& g, int k)
{
    const float u = floorf((x - g.lo[k]) * g.ih[k]);
    return int(fminf(fmaxf(u, 0.0f), float(g.n[k] - 1u)));
}

// words: [0..2] min lo (order-preserving), [3..5] max hi, [6] valid primitives
template <class Src>
__global__ void k_grid_bounds(Src src, uint32_t n, uint32_t* words, double* r2sum)
{
    uint32_t mn[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, mx[3] = {0u, 0u, 0u}, cnt = 0;
    double r2 = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const SBox b = src.box(i);
        if (!b.ok)
            continue;
        for (int k = 0; k < 3; ++k) {
            mn[k] = min(mn[k], f2o(b.lo[k]));
            mx[k] = max(mx[k], f2o(b.hi[k]));
        }
        r2 += src.xsec(i);
        ++cnt;
    }
    for (int off = 16; off > 0; off >>= 1) {
        for (int k = 0; k < 3; ++k) {
            mn[k] = min(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], off));
            mx[k] = max(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], off));
        }
        cnt += __shfl_xor_sync(0xffffffffu, cnt, off);
        r2 += __shfl_xor_sync(0xffffffffu, r2, off);
    }
    if ((threadIdx.x & 31u) == 0u && cnt) {
        for (int k = 0; k < 3; ++k) {
            atomicMin(words + k, mn[k]);
            atomicMax(words + 3 + k, mx[k]);
        }
        atomicAdd(words + 6, cnt);
        atomicAdd(r2sum, r2);
    }
}

// cells covered by each primitive (0 for invalid ones); flag bit 0: one covers too many
template <class Src>
__global__ void k_grid_count(Src src, uint32_t n, Shape g, uint32_t max_per_prim,
                             uint32_t* counts, uint32_t* flag)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const SBox b = src.box(i);
    uint32_t c = 0;
    if (b.ok) {
        unsigned long long m = 1;
        for (int k = 0; k < 3; ++k)
            m *= (unsigned long long)(cell_index(b.hi[k], g, k) - cell_index(b.lo[k], g, k) + 1);
        if (m > max_per_prim)
            atomicOr(flag, 1u);
        else
            c = uint32_t(m);
    }
    counts[i] = c;
}

template <class Src>
__global__ void k_grid_emit(Src src, uint32_t n, Shape g, const uint32_t* counts,
                            const uint32_t* offsets, uint32_t* keys, uint32_t* vals)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || counts[i] == 0)
        return;
    const SBox b = src.box(i);
    int i0[3], i1[3];
    for (int k = 0; k < 3; ++k) {
        i0[k] = cell_index(b.lo[k], g, k);
        i1[k] = cell_index(b.hi[k], g, k);
    }
    uint32_t o = offsets[i];
    const uint32_t end = o + counts[i];
    for (int z = i0[2]; z <= i1[2]; ++z)
        for (int y = i0[1]; y <= i1[1]; ++y)
            for (int x = i0[0]; x <= i1[0]; ++x) {
                if (o >= end)
                    return;  // cannot happen: the counts come from the same ranges
                keys[o] = (uint32_t(z) * g.n[1] + uint32_t(y)) * g.n[0] + uint32_t(x);
                vals[o] = i;
                ++o;
            }
}

__global__ void k_grid_cell_counts(const uint32_t* keys, uint32_t total, uint32_t n_cells,
                                   uint32_t* cell_counts)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < total && keys[i] < n_cells)
        atomicAdd(cell_counts + keys[i], 1u);
}

__global__ void k_grid_max(const uint32_t* cell_counts, uint32_t n_cells, uint32_t* word)
{
    uint32_t m = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_cells;
         i += gridDim.x * blockDim.x)
        m = max(m, cell_counts[i]);
    for (int off = 16; off > 0; off >>= 1)
        m = max(m, __shfl_xor_sync(0xffffffffu, m, off));
    if ((threadIdx.x & 31u) == 0u && m)
        atomicMax(word, m);
}

__global__ void k_grid_gather(const uint32_t* vals, uint32_t total, const float* pos,
                              const float* rad, float4* ref_sphere, uint32_t* ref_prim)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total)
        return;
    const uint32_t s = vals[i];
    ref_sphere[i] = make_float4(pos[3 * size_t(s)], pos[3 * size_t(s) + 1],
                                pos[3 * size_t(s) + 2], rad[s]);
    ref_prim[i] = s;
}

// blocks of 256 threads for one thread per item (cap: for grid-stride kernels only)
uint32_t blocks_for(size_t n, uint32_t cap = 0x7fffffffu)
{
    size_t b = (n + 255) / 256;
    return uint32_t(std::max<size_t>(1, std::min<size_t>(b, cap)));
}

}  // namespace

namespace {

// Why a grid was not built, in the words of its primitives.
struct Reasons {
    const char *none, *no_valid, *few, *sparse, *spans, *refs, *clustered;
};
const Reasons SPHERE_REASONS = {"no spheres",
                                "no valid sphere",
                                "too few spheres",
                                "spheres too sparse",
                                "a sphere spans too many cells",
                                "too many sphere references",
                                "spheres too clustered"};
const Reasons PART_REASONS = {"no primitives",
                              "no valid primitive",
                              "too few primitives",
                              "primitives too sparse",
                              "a primitive spans too many cells",
                              "too many primitive references",
                              "primitives too clustered"};

// Steps 1-4 but the reference records: cell_start, the shape, and the primitive of every
// reference in *vals_sorted (scratch memory, valid until the scratch is next reserved).  A grid
// that should not be used leaves out.n_cells == 0 with rep.built false and rep.reason set.
template <class Src>
cudaError_t build_cells(const Src& src, uint32_t n, const Reasons& why, const GridParams& gp,
                        GridBuffers& out, Scratch& scratch, cudaStream_t st, GridReport& rep,
                        const uint32_t*& vals_out, uint32_t& total_out)
{
    rep = GridReport();
    out.n_cells = 0;
    out.n_refs = 0;
    vals_out = nullptr;
    total_out = 0;
    if (n == 0) {
        rep.reason = why.none;
        return cudaSuccess;
    }
    cudaError_t e;
    // ---- 1. bounds, valid count, sum of r^2
    size_t scan_n_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_n_bytes, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                  int(n), st);
    ScratchLayout L1;
    uint32_t* words = L1.take<uint32_t>(16);
    double* r2sum = L1.take<double>(1);
    void* scan_tmp = L1.take<unsigned char>(scan_n_bytes);
    if ((e = scratch.reserve(L1.bytes)) != cudaSuccess)
        return e;
    L1.bind(scratch.ptr);
    words = L1.at(words);
    r2sum = L1.at(r2sum);
    scan_tmp = L1.at(scan_tmp);
    const uint32_t init[16] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0, 0, 0, 0, 0,
                               0,           0,           0,           0, 0, 0, 0, 0};
    if ((e = cudaMemcpyAsync(words, init, sizeof(init), cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return e;
    if ((e = cudaMemsetAsync(r2sum, 0, sizeof(double), st)) != cudaSuccess)
        return e;
    k_grid_bounds<<<blocks_for(n, 148u * 8u), 256, 0, st>>>(src, n, words, r2sum);
    uint32_t hw[16];
    double hr2 = 0.0;
    if ((e = cudaMemcpyAsync(hw, words, sizeof(hw), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&hr2, r2sum, sizeof(double), cudaMemcpyDeviceToHost, st)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return e;
    rep.n_valid = hw[6];
    if (rep.n_valid == 0) {
        rep.reason = why.no_valid;
        return cudaSuccess;
    }
    // ---- 2. cell size and the automatic choice
    double lo[3], ext[3];
    double scale = 1.0;
    for (int k = 0; k < 3; ++k) {
        lo[k] = o2f_host(hw[k]);
        ext[k] = double(o2f_host(hw[3 + k])) - lo[k];
        scale = std::max(scale, std::max(std::fabs(lo[k]), std::fabs(lo[k] + ext[k])));
    }
    for (int k = 0; k < 3; ++k)
        ext[k] = std::max(ext[k], 1e-6 * scale);
    const double volume = ext[0] * ext[1] * ext[2];
    double h = std::cbrt(volume / (double(gp.cells_per_prim) * rep.n_valid));
    uint32_t dims[3] = {1, 1, 1};
    for (int pass = 0; pass < 64; ++pass) {
        double cells = 1.0;
        for (int k = 0; k < 3; ++k) {
            dims[k] = uint32_t(std::min(1024.0, std::max(1.0, std::ceil(ext[k] / h))));
            cells *= dims[k];
        }
        if (cells <= double(1u << 26))
            break;
        h *= 1.25;
    }
    const uint64_t n_cells = uint64_t(dims[0]) * dims[1] * dims[2];
    float cell[3], ih[3], flo[3], fhi[3];
    for (int k = 0; k < 3; ++k) {
        flo[k] = float(lo[k]);
        cell[k] = float(ext[k] / dims[k]) * (1.0f + 4e-7f);  // the cells cover the whole union
        ih[k] = 1.0f / cell[k];
        fhi[k] = flo[k] + float(dims[k]) * cell[k];
    }
    const double mean_r2 = hr2 / rep.n_valid;
    const double h_mean = std::cbrt(double(cell[0]) * cell[1] * cell[2]);
    const double pi = 3.14159265358979323846;
    rep.cells_per_ray =
        mean_r2 > 0.0 ? volume / (rep.n_valid * pi * mean_r2) / h_mean + 1.0 : 1e30;
    // a ray leaves the grid after at most nx + ny + nz cells
    rep.cells_per_ray = std::min(rep.cells_per_ray, double(dims[0]) + dims[1] + dims[2]);
    if (gp.mode == 2) {
        if (rep.n_valid < gp.min_prims) {
            rep.reason = why.few;
            return cudaSuccess;
        }
        if (rep.cells_per_ray > gp.max_cells_per_ray) {
            rep.reason = why.sparse;
            return cudaSuccess;
        }
    }
    Shape g;
    for (int k = 0; k < 3; ++k) {
        g.lo[k] = flo[k];
        g.ih[k] = ih[k];
        g.n[k] = dims[k];
    }
    // ---- 3. cells per sphere, offsets, pairs
    if ((e = out.prim_count.reserve(n)) != cudaSuccess ||
        (e = out.prim_offset.reserve(n)) != cudaSuccess)
        return e;
    k_grid_count<<<blocks_for(n), 256, 0, st>>>(src, n, g, gp.max_cells_per_prim,
                                                 out.prim_count.ptr, words + 8);
    if ((e = cub::DeviceScan::ExclusiveSum(scan_tmp, scan_n_bytes, out.prim_count.ptr,
                                           out.prim_offset.ptr, int(n), st)) != cudaSuccess)
        return e;
    uint32_t last[2] = {0, 0}, flag = 0;
    if ((e = cudaMemcpyAsync(&last[0], out.prim_offset.ptr + (n - 1), 4, cudaMemcpyDeviceToHost,
                             st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&last[1], out.prim_count.ptr + (n - 1), 4, cudaMemcpyDeviceToHost,
                             st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&flag, words + 8, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return e;
    if (flag) {
        rep.reason = why.spans;
        return cudaSuccess;
    }
    const uint64_t total64 = uint64_t(last[0]) + last[1];
    if (total64 == 0 || total64 > uint64_t(1u << 30) ||
        total64 > 32 * uint64_t(rep.n_valid) + (uint64_t(1) << 20)) {
        rep.reason = why.refs;
        return cudaSuccess;
    }
    const uint32_t total = uint32_t(total64);
    const uint32_t nc = uint32_t(n_cells);
    int end_bit = 1;
    while (end_bit < 32 && (uint64_t(1) << end_bit) < n_cells)
        ++end_bit;
    size_t sort_bytes = 0, scan_c_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                    (uint32_t*)nullptr, (uint32_t*)nullptr, int(total), 0, end_bit,
                                    st);
    cub::DeviceScan::ExclusiveSum(nullptr, scan_c_bytes, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                  int(nc + 1), st);
    ScratchLayout L2;
    uint32_t* keys = L2.take<uint32_t>(total);
    uint32_t* keys_sorted = L2.take<uint32_t>(total);
    uint32_t* vals = L2.take<uint32_t>(total);
    uint32_t* vals_sorted = L2.take<uint32_t>(total);
    uint32_t* cell_counts = L2.take<uint32_t>(size_t(nc) + 1);
    uint32_t* max_word = L2.take<uint32_t>(1);
    void* tmp = L2.take<unsigned char>(std::max(sort_bytes, scan_c_bytes));
    if ((e = scratch.reserve(L2.bytes)) != cudaSuccess)
        return e;
    L2.bind(scratch.ptr);
    keys = L2.at(keys);
    keys_sorted = L2.at(keys_sorted);
    vals = L2.at(vals);
    vals_sorted = L2.at(vals_sorted);
    cell_counts = L2.at(cell_counts);
    max_word = L2.at(max_word);
    tmp = L2.at(tmp);
    if ((e = out.cell_start.reserve(size_t(nc) + 1)) != cudaSuccess)
        return e;
    k_grid_emit<<<blocks_for(n), 256, 0, st>>>(src, n, g, out.prim_count.ptr, out.prim_offset.ptr,
                                                keys, vals);
    if ((e = cub::DeviceRadixSort::SortPairs(tmp, sort_bytes, keys, keys_sorted, vals,
                                             vals_sorted, int(total), 0, end_bit, st)) !=
        cudaSuccess)
        return e;
    // ---- 4. cell offsets, fullest cell, reference records
    if ((e = cudaMemsetAsync(cell_counts, 0, (size_t(nc) + 1) * sizeof(uint32_t), st)) !=
            cudaSuccess ||
        (e = cudaMemsetAsync(max_word, 0, sizeof(uint32_t), st)) != cudaSuccess)
        return e;
    k_grid_cell_counts<<<blocks_for(total), 256, 0, st>>>(keys_sorted, total, nc, cell_counts);
    k_grid_max<<<blocks_for(nc, 148u * 8u), 256, 0, st>>>(cell_counts, nc, max_word);
    if ((e = cub::DeviceScan::ExclusiveSum(tmp, scan_c_bytes, cell_counts, out.cell_start.ptr,
                                           int(nc + 1), st)) != cudaSuccess)
        return e;
    uint32_t max_refs = 0;
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cudaMemcpyAsync(&max_refs, max_word, 4, cudaMemcpyDeviceToHost, st)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return e;
    rep.max_refs = max_refs;
    if (gp.mode == 2 && max_refs > gp.max_refs_per_cell) {
        rep.reason = why.clustered;
        return cudaSuccess;
    }
    for (int k = 0; k < 3; ++k) {
        out.dims[k] = dims[k];
        out.lo[k] = flo[k];
        out.hi[k] = fhi[k];
        out.cell[k] = cell[k];
    }
    vals_out = vals_sorted;
    total_out = total;
    return cudaSuccess;
}

}  // namespace

cudaError_t build_grid(const float* position, const float* radius, uint32_t n,
                       const GridParams& gp, GridBuffers& out, Scratch& scratch, cudaStream_t st,
                       GridReport& rep)
{
    const uint32_t* vals = nullptr;
    uint32_t total = 0;
    cudaError_t e = build_cells(SphereSource{position, radius}, n, SPHERE_REASONS, gp, out,
                                scratch, st, rep, vals, total);
    if (e != cudaSuccess || vals == nullptr)
        return e;
    if ((e = out.ref_sphere.reserve(total)) != cudaSuccess ||
        (e = out.ref_prim.reserve(total)) != cudaSuccess)
        return e;
    k_grid_gather<<<blocks_for(total), 256, 0, st>>>(vals, total, position, radius,
                                                      out.ref_sphere.ptr, out.ref_prim.ptr);
    if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return e;
    out.parts = false;
    out.n_cells = uint32_t(uint64_t(out.dims[0]) * out.dims[1] * out.dims[2]);
    out.n_refs = total;
    rep.built = true;
    rep.reason = "";
    return cudaSuccess;
}

cudaError_t build_grid(const PartsInput& in, uint32_t n, const GridParams& gp, GridBuffers& out,
                       Scratch& scratch, cudaStream_t st, GridReport& rep)
{
    cudaError_t e;
    if (n != 0 && ((e = out.box_lo.reserve(n)) != cudaSuccess ||
                   (e = out.box_hi.reserve(n)) != cudaSuccess ||
                   (e = parts_boxes(in, n, out.box_lo.ptr, out.box_hi.ptr, st)) != cudaSuccess))
        return e;
    const uint32_t* vals = nullptr;
    uint32_t total = 0;
    e = build_cells(BoxSource{out.box_lo.ptr, out.box_hi.ptr}, n, PART_REASONS, gp, out, scratch,
                    st, rep, vals, total);
    if (e != cudaSuccess || vals == nullptr)
        return e;
    if ((e = out.ref_data.reserve(2 * size_t(total))) != cudaSuccess ||
        (e = out.ref_prim.reserve(total)) != cudaSuccess ||
        (e = out.ref_geom.reserve(total)) != cudaSuccess ||
        (e = gather_parts(in, vals, total, out.ref_data.ptr, out.ref_prim.ptr, out.ref_geom.ptr,
                          st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return e;
    out.parts = true;
    out.n_cells = uint32_t(uint64_t(out.dims[0]) * out.dims[1] * out.dims[2]);
    out.n_refs = total;
    rep.built = true;
    rep.reason = "";
    return cudaSuccess;
}

}  // namespace fr
