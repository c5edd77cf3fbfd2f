// bvh.cu -- GPU LBVH construction for one geometry.
//
// Replaces the acceleration structure the reference gets from OptiX ("Trbvh",
// fresnel/gpu/Scene.cc:19) or Embree (RTC_BUILD_QUALITY_LOW, fresnel/cpu/Scene.cc:18-19),
// built over the per-primitive bounds of fresnel/gpu/Geometry*.cu / fresnel/cpu/Geometry*.cc.
// Method (published): Karras, "Maximizing parallelism in the construction of BVHs, octrees,
// and k-d trees", HPG 2012 -- 63-bit Morton codes of the box centroids, radix sort (CUB),
// one thread per internal node to find its key range and split, then a bottom-up pass with
// per-node arrival counters that unions child boxes and evaluates the surface-area cost of
// turning each subtree into a leaf (collapse when count <= leaf_max and the leaf is cheaper).
// The surviving interior nodes are compacted so that the two children of every interior node
// are adjacent (one 64-byte load per traversal step).
#include <cub/cub.cuh>

#include "bvh.hpp"
#include "engine.cuh"

namespace fr {

namespace {

struct Box {
    float3 lo, hi;
};

__device__ __forceinline__ float3 f3min(float3 a, float3 b)
{
    return make_float3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z));
}
__device__ __forceinline__ float3 f3max(float3 a, float3 b)
{
    return make_float3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z));
}

__device__ __forceinline__ bool finite3(float3 a)
{
    return isfinite(a.x) && isfinite(a.y) && isfinite(a.z);
}

// Pad a box outward so that rounding in the traversal's slab test (one fused multiply-add per
// plane) can never reject a ray that the exact intersector would accept.
__device__ __forceinline__ Box inflate(Box b)
{
    float scale = fmaxf(fmaxf(fmaxf(fabsf(b.lo.x), fabsf(b.hi.x)), fmaxf(fabsf(b.lo.y), fabsf(b.hi.y))),
                        fmaxf(fabsf(b.lo.z), fabsf(b.hi.z)));
    float ext = (b.hi.x - b.lo.x) + (b.hi.y - b.lo.y) + (b.hi.z - b.lo.z);
    float pad = 1e-5f * scale + 1e-6f * ext + 1e-30f;
    b.lo = make_float3(b.lo.x - pad, b.lo.y - pad, b.lo.z - pad);
    b.hi = make_float3(b.hi.x + pad, b.hi.y + pad, b.hi.z + pad);
    return b;
}

__device__ __forceinline__ void grow(Box& b, V3 p)
{
    b.lo = f3min(b.lo, make_float3(p.x, p.y, p.z));
    b.hi = f3max(b.hi, make_float3(p.x, p.y, p.z));
}

__device__ __forceinline__ Box empty_box()
{
    const float inf = __int_as_float(0x7f800000);
    return Box{make_float3(inf, inf, inf), make_float3(-inf, -inf, -inf)};
}

__device__ __forceinline__ float std_min(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float std_max(float a, float b) { return (a < b) ? b : a; }

// Bounds of one primitive, with the reference's formulas (fresnel/cpu/GeometrySphere.cc:60-73,
// GeometryCylinder.cc:55-70, GeometryConvexPolyhedron.cc:119-132, GeometryMesh.cc:81-113,
// GeometryPolygon.cc:89-104).  A box that is not finite or has lower > upper (e.g. a negative or
// infinite radius) is empty, so no ray enters it: Embree leaves such primitives out of its
// tree.
__device__ Box prim_bounds(const BuildInput& in, uint32_t i)
{
    Box b = empty_box();
    switch (in.type) {
    case FR_GEOM_SPHERE: {
        V3 p = load3(in.position, i);
        float r = in.radius[i];
        b.lo = make_float3(p.x - r, p.y - r, p.z - r);
        b.hi = make_float3(p.x + r, p.y + r, p.z + r);
        break;
    }
    case FR_GEOM_CYLINDER: {
        V3 A = load3(in.points, 2 * i), B = load3(in.points, 2 * i + 1);
        float r = in.radius[i];
        b.lo = make_float3(std_min(A.x - r, B.x - r), std_min(A.y - r, B.y - r),
                           std_min(A.z - r, B.z - r));
        b.hi = make_float3(std_max(A.x + r, B.x + r), std_max(A.y + r, B.y + r),
                           std_max(A.z + r, B.z + r));
        break;
    }
    case FR_GEOM_POLYHEDRON: {
        V3 p = load3(in.position, i);
        float r = in.poly_radius;
        b.lo = make_float3(p.x - r, p.y - r, p.z - r);
        b.hi = make_float3(p.x + r, p.y + r, p.z + r);
        break;
    }
    case FR_GEOM_MESH: {
        if (in.instances) {  // the whole instance: every face's vertices
            V3 p = load3(in.position, i);
            Qt q = loadq(in.orientation, i);
            for (uint32_t k = 0; k < 3 * in.n_faces; ++k)
                grow(b, rotate(q, load3(in.vertices, k)) + p);
            break;
        }
        uint32_t inst = i / in.n_faces, face = i - inst * in.n_faces;
        V3 p = load3(in.position, inst);
        Qt q = loadq(in.orientation, inst);
        for (int k = 0; k < 3; ++k)
            grow(b, rotate(q, load3(in.vertices, 3 * face + k)) + p);
        break;
    }
    default: {  // polygon in the z = 0 plane
        const float x = in.position[2 * size_t(i)], y = in.position[2 * size_t(i) + 1];
        const float r = in.poly_radius;
        b.lo = make_float3(x - r, y - r, 0.0f - 1e-5f);
        b.hi = make_float3(x + r, y + r, 0.0f + 1e-5f);
        break;
    }
    }
    if (!finite3(b.lo) || !finite3(b.hi) || b.lo.x > b.hi.x || b.lo.y > b.hi.y || b.lo.z > b.hi.z)
        return empty_box();
    return inflate(b);
}

// Part of combined primitive i (the last part whose first index is <= i).
__device__ __forceinline__ uint32_t part_of(const PartsInput& in, uint32_t i)
{
    uint32_t p = 0;
    while (p + 1u < in.n_parts && i >= in.first[p + 1])
        ++p;
    return p;
}

__device__ Box prim_bounds(const PartsInput& in, uint32_t i)
{
    const uint32_t p = part_of(in, i);
    return prim_bounds(in.part[p], i - in.first[p]);
}

// float <-> order-preserving uint32 for atomic min/max of the centroid bounds
__device__ __forceinline__ uint32_t f2o(float f)
{
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float o2f(uint32_t u)
{
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

template <class In>
__global__ void k_bounds(In in, uint32_t n, float4* box_lo, float4* box_hi, uint32_t* cbounds)
{
    uint32_t lmin[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, lmax[3] = {0u, 0u, 0u};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        Box b = prim_bounds(in, i);
        box_lo[i] = make_float4(b.lo.x, b.lo.y, b.lo.z, 0.0f);
        box_hi[i] = make_float4(b.hi.x, b.hi.y, b.hi.z, 0.0f);
        if (b.lo.x <= b.hi.x) {
            float c[3] = {0.5f * (b.lo.x + b.hi.x), 0.5f * (b.lo.y + b.hi.y), 0.5f * (b.lo.z + b.hi.z)};
            for (int k = 0; k < 3; ++k) {
                lmin[k] = min(lmin[k], f2o(c[k]));
                lmax[k] = max(lmax[k], f2o(c[k]));
            }
        }
    }
    for (int k = 0; k < 3; ++k) {
        for (int off = 16; off > 0; off >>= 1) {
            lmin[k] = min(lmin[k], __shfl_xor_sync(0xffffffffu, lmin[k], off));
            lmax[k] = max(lmax[k], __shfl_xor_sync(0xffffffffu, lmax[k], off));
        }
    }
    if ((threadIdx.x & 31) == 0) {
        for (int k = 0; k < 3; ++k) {
            atomicMin(cbounds + k, lmin[k]);
            atomicMax(cbounds + 3 + k, lmax[k]);
        }
    }
}

__device__ __forceinline__ uint64_t spread21(uint32_t x)
{
    uint64_t v = x & 0x1fffffu;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

__global__ void k_morton(uint32_t n, const float4* box_lo, const float4* box_hi,
                         const uint32_t* cbounds, uint64_t* keys, uint32_t* vals)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    float4 lo = box_lo[i], hi = box_hi[i];
    uint64_t key = ~0ull;
    if (lo.x <= hi.x) {
        float c[3] = {0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y), 0.5f * (lo.z + hi.z)};
        uint32_t q[3];
        for (int k = 0; k < 3; ++k) {
            float mn = o2f(cbounds[k]), mx = o2f(cbounds[3 + k]);
            float ext = mx - mn;
            float u = ext > 0.0f ? (c[k] - mn) / ext : 0.5f;
            u = fminf(fmaxf(u, 0.0f), 1.0f);
            q[k] = min(uint32_t(u * 2097152.0f), 2097151u);
        }
        key = (spread21(q[0]) << 2) | (spread21(q[1]) << 1) | spread21(q[2]);
    }
    keys[i] = key;
    vals[i] = i;
}

// common-prefix length of sorted keys i and j, with the index breaking ties (Karras 2012 sec 4)
__device__ __forceinline__ int delta(const uint64_t* keys, uint32_t n, int i, int j)
{
    if (j < 0 || j >= int(n))
        return -1;
    uint64_t a = keys[i], b = keys[j];
    if (a == b)
        return 64 + __clz(uint32_t(i) ^ uint32_t(j));
    return __clzll(a ^ b);
}

__global__ void k_karras(uint32_t n, const uint64_t* keys, int2* range, uint32_t* split,
                         uint32_t* parent_int, uint32_t* parent_leaf)
{
    int i = int(blockIdx.x * blockDim.x + threadIdx.x);
    if (i >= int(n) - 1)
        return;
    int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    int dmin = delta(keys, n, i, i - d);
    int lmax = 2;
    while (delta(keys, n, i, i + lmax * d) > dmin)
        lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (delta(keys, n, i, i + (l + t) * d) > dmin)
            l += t;
    int j = i + l * d;
    int dnode = delta(keys, n, i, j);
    int s = 0;
    for (int div = 2;; div <<= 1) {
        int t = (l + div - 1) / div;
        if (delta(keys, n, i, i + (s + t) * d) > dnode)
            s += t;
        if (t == 1)
            break;
    }
    int gamma = i + s * d + min(d, 0);
    int first = min(i, j), last = max(i, j);
    range[i] = make_int2(first, last);
    split[i] = uint32_t(gamma);
    // children: gamma (leaf if first == gamma) and gamma + 1 (leaf if last == gamma + 1)
    if (first == gamma)
        parent_leaf[gamma] = uint32_t(i);
    else
        parent_int[gamma] = uint32_t(i);
    if (last == gamma + 1)
        parent_leaf[gamma + 1] = uint32_t(i);
    else
        parent_int[gamma + 1] = uint32_t(i);
}

__device__ __forceinline__ float half_area(float3 lo, float3 hi)
{
    float dx = hi.x - lo.x, dy = hi.y - lo.y, dz = hi.z - lo.z;
    if (!(dx >= 0.0f) || !(dy >= 0.0f) || !(dz >= 0.0f))
        return 0.0f;
    return dx * dy + dy * dz + dz * dx;
}

struct NodeInfo {  // per internal node, written by the refit pass
    float4 lo, hi;  // lo.w = SAH cost, hi.w = primitive count (as float)
};

// Bottom-up: one thread per leaf; the second thread to arrive at a node unions its children.
__global__ void k_refit(uint32_t n, const uint32_t* sorted_vals, const float4* box_lo,
                        const float4* box_hi, const int2* range, const uint32_t* split,
                        const uint32_t* parent_int, const uint32_t* parent_leaf, uint32_t* arrive,
                        NodeInfo* info, uint8_t* collapse, int leaf_max, float c_trav,
                        float c_isect, uint32_t* status)
{
    uint32_t leaf = blockIdx.x * blockDim.x + threadIdx.x;
    if (leaf >= n || n < 2)
        return;
    uint32_t node = parent_leaf[leaf];
    for (int guard = 0;; ++guard) {
        if (node >= n - 1 || guard > 200) {  // unset parent or a cycle: report, never follow
            atomicOr(status, ERR_BUILD);
            return;
        }
        __threadfence();
        if (atomicAdd(arrive + node, 1u) == 0u)
            return;
        __threadfence();
        uint32_t g = split[node];
        int2 rg = range[node];
        if (g + 1u >= n) {
            atomicOr(status, ERR_BUILD);
            return;
        }
        float4 lo[2], hi[2];
        float cost[2];
        float cnt[2];
        for (int c = 0; c < 2; ++c) {
            uint32_t idx = g + uint32_t(c);
            bool is_leaf = (c == 0) ? (uint32_t(rg.x) == g) : (uint32_t(rg.y) == g + 1);
            if (is_leaf) {
                uint32_t p = sorted_vals[idx];
                lo[c] = box_lo[p];
                hi[c] = box_hi[p];
                float a = half_area(make_float3(lo[c].x, lo[c].y, lo[c].z),
                                    make_float3(hi[c].x, hi[c].y, hi[c].z));
                cost[c] = c_isect * a;
                cnt[c] = 1.0f;
            } else {
                NodeInfo ci;
                ci.lo = __ldcg(&info[idx].lo);
                ci.hi = __ldcg(&info[idx].hi);
                lo[c] = ci.lo;
                hi[c] = ci.hi;
                cost[c] = ci.lo.w;
                cnt[c] = ci.hi.w;
            }
        }
        float3 ulo = f3min(make_float3(lo[0].x, lo[0].y, lo[0].z), make_float3(lo[1].x, lo[1].y, lo[1].z));
        float3 uhi = f3max(make_float3(hi[0].x, hi[0].y, hi[0].z), make_float3(hi[1].x, hi[1].y, hi[1].z));
        float a = half_area(ulo, uhi);
        float count = cnt[0] + cnt[1];
        float split_cost = c_trav * a + cost[0] + cost[1];
        float leaf_cost = c_isect * a * count;
        bool col = (count <= float(leaf_max)) && (leaf_cost <= split_cost);
        NodeInfo out;
        out.lo = make_float4(ulo.x, ulo.y, ulo.z, col ? leaf_cost : split_cost);
        out.hi = make_float4(uhi.x, uhi.y, uhi.z, count);
        __stcg(&info[node].lo, out.lo);
        __stcg(&info[node].hi, out.hi);
        collapse[node] = col ? 1 : 0;
        if (node == 0)
            return;
        node = parent_int[node];
    }
}

// An internal node survives as an interior node of the output tree iff it is not collapsed
// and no ancestor is collapsed.  keep[gamma] marks the child pair owned by that node.
__global__ void k_mark(uint32_t n, const uint32_t* split, const uint32_t* parent_int,
                       const uint8_t* collapse, uint32_t* keep, uint32_t* removed)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1)
        return;
    bool rem = false;
    uint32_t a = i;
    for (int guard = 0; a != 0 && guard < 4096; ++guard) {
        a = parent_int[a];
        if (a >= n - 1)
            break;  // unset parent: reported by the refit pass
        if (collapse[a]) {
            rem = true;
            break;
        }
    }
    removed[i] = rem ? 1u : 0u;
    keep[split[i]] = (!rem && !collapse[i]) ? 1u : 0u;
}

__device__ __forceinline__ void write_node(float4* nodes, uint32_t slot, float4 lo, float4 hi,
                                           uint32_t a, uint32_t b)
{
    nodes[2 * size_t(slot)] = make_float4(lo.x, lo.y, lo.z, __uint_as_float(a));
    nodes[2 * size_t(slot) + 1] = make_float4(hi.x, hi.y, hi.z, __uint_as_float(b));
}

__global__ void k_emit(uint32_t n, const int2* range, const uint32_t* split,
                       const uint8_t* collapse, const uint32_t* removed, const uint32_t* pair_index,
                       const NodeInfo* info, const uint32_t* sorted_vals, const float4* box_lo,
                       const float4* box_hi, float4* nodes)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1 || removed[i])
        return;
    if (i == 0) {  // root
        int2 rg = range[0];
        if (collapse[0])
            write_node(nodes, 0, info[0].lo, info[0].hi, uint32_t(rg.x), uint32_t(rg.y - rg.x + 1));
        else
            write_node(nodes, 0, info[0].lo, info[0].hi, 1u + 2u * pair_index[split[0]], 0u);
    }
    if (collapse[i])
        return;
    uint32_t g = split[i];
    int2 rg = range[i];
    uint32_t base = 1u + 2u * pair_index[g];
    if (base + 1u >= 2u * n - 1u)  // both children must fit in the 2n-1 node slots
        return;
    for (int c = 0; c < 2; ++c) {
        uint32_t idx = g + uint32_t(c);
        bool is_leaf = (c == 0) ? (uint32_t(rg.x) == g) : (uint32_t(rg.y) == g + 1);
        if (is_leaf) {
            uint32_t p = sorted_vals[idx];
            write_node(nodes, base + c, box_lo[p], box_hi[p], idx, 1u);
        } else if (collapse[idx]) {
            int2 cr = range[idx];
            write_node(nodes, base + c, info[idx].lo, info[idx].hi, uint32_t(cr.x),
                       uint32_t(cr.y - cr.x + 1));
        } else {
            write_node(nodes, base + c, info[idx].lo, info[idx].hi, 1u + 2u * pair_index[split[idx]],
                       0u);
        }
    }
}

__global__ void k_single_leaf(const float4* box_lo, const float4* box_hi, float4* nodes)
{
    write_node(nodes, 0, box_lo[0], box_hi[0], 0u, 1u);
}

// The record the intersection loop reads for primitive p, written at r (1 float4 for a sphere,
// 2 for the other types).
__device__ __forceinline__ void write_record(const BuildInput& in, uint32_t p, float4* r)
{
    switch (in.type) {
    case FR_GEOM_SPHERE: {
        V3 c = load3(in.position, p);
        r[0] = make_float4(c.x, c.y, c.z, in.radius[p]);
        break;
    }
    case FR_GEOM_CYLINDER: {
        V3 A = load3(in.points, 2 * p), B = load3(in.points, 2 * p + 1);
        r[0] = make_float4(A.x, A.y, A.z, in.radius[p]);
        r[1] = make_float4(B.x, B.y, B.z, 0.0f);
        break;
    }
    case FR_GEOM_POLYHEDRON: {
        V3 c = load3(in.position, p);
        Qt q = loadq(in.orientation, p);
        r[0] = make_float4(c.x, c.y, c.z, 0.0f);
        r[1] = make_float4(q.s, q.v.x, q.v.y, q.v.z);
        break;
    }
    case FR_GEOM_MESH: {  // (an instance record when in.instances: face 0)
        uint32_t inst = in.instances ? p : p / in.n_faces;
        uint32_t face = in.instances ? 0u : p - inst * in.n_faces;
        V3 c = load3(in.position, inst);
        Qt q = loadq(in.orientation, inst);
        r[0] = make_float4(c.x, c.y, c.z, __uint_as_float(face));
        r[1] = make_float4(q.s, q.v.x, q.v.y, q.v.z);
        break;
    }
    default: {  // polygon: 2-D position and the rotation quaternion about z
        Qt q = loadq(in.orientation, p);
        r[0] = make_float4(in.position[2 * size_t(p)], in.position[2 * size_t(p) + 1], 0.0f, 0.0f);
        r[1] = make_float4(q.s, q.v.x, q.v.y, q.v.z);
        break;
    }
    }
}

// Leaf-ordered copies of the primitive data the intersection loop reads.
__global__ void k_gather(BuildInput in, uint32_t n, const uint32_t* sorted_vals, float4* leaf_data,
                         uint32_t* order, uint32_t* /*leaf_geom*/)
{
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n)
        return;
    uint32_t p = sorted_vals[s];
    order[s] = p;
    write_record(in, p, leaf_data + (in.type == FR_GEOM_SPHERE ? s : 2 * size_t(s)));
}

// Combined trees: sorted_vals holds combined indices; order gets the index within the geometry.
__global__ void k_gather(PartsInput in, uint32_t n, const uint32_t* sorted_vals,
                         float4* leaf_data, uint32_t* order, uint32_t* leaf_geom)
{
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n)
        return;
    const uint32_t g = sorted_vals[s];
    const uint32_t p = part_of(in, g);
    const uint32_t local = g - in.first[p];
    order[s] = local;
    leaf_geom[s] = in.geom[p];
    write_record(in.part[p], local, leaf_data + 2 * size_t(s));
}

// Combined trees being refitted: the combined index of each leaf slot, from its geometry and
// its index within it.
__global__ void k_combined_order(PartsInput in, uint32_t n, const uint32_t* order,
                                 const uint32_t* leaf_geom, uint32_t* combined, uint32_t* status)
{
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n)
        return;
    const uint32_t gi = leaf_geom[s];
    uint32_t p = 0;
    while (p < in.n_parts && in.geom[p] != gi)
        ++p;
    if (p == in.n_parts || order[s] >= in.first[p + 1] - in.first[p]) {
        atomicOr(status, ERR_BUILD);
        combined[s] = 0;
        return;
    }
    combined[s] = in.first[p] + order[s];
}

// ---------------------------------------------------------------------------------------------
// 4-wide collapse: every 4-wide node takes the two children of a binary interior node and keeps
// opening its largest-area interior child until it has four children (a leaf of the binary tree
// stays a leaf).  Processed top-down, one level of 4-wide nodes per launch.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ float node2_area(float4 lo, float4 hi)
{
    return half_area(make_float3(lo.x, lo.y, lo.z), make_float3(hi.x, hi.y, hi.z));
}

__global__ void k_collapse4(const float4* nodes2, uint32_t n_nodes2, const uint2* in_q,
                            const uint32_t* in_count, uint2* out_q, uint32_t* out_count,
                            uint32_t* node4_count, uint32_t node4_cap, float4* nodes4,
                            uint32_t* status)
{
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= *in_count)
        return;
    uint2 job = in_q[t];  // (binary node, 4-wide node)
    if (job.x >= n_nodes2 || job.y >= node4_cap) {
        atomicOr(status, ERR_BUILD);
        return;
    }
    uint32_t child[4];
    int nc = 0;
    float4 root_hi = nodes2[2 * size_t(job.x) + 1];
    if (__float_as_uint(root_hi.w) != 0) {  // the binary root is itself a leaf
        child[nc++] = job.x;
    } else {
        uint32_t a = __float_as_uint(nodes2[2 * size_t(job.x)].w);
        if (a + 1u >= n_nodes2) {
            atomicOr(status, ERR_BUILD);
            return;
        }
        child[nc++] = a;
        child[nc++] = a + 1;
        while (nc < 4) {
            int best = -1;
            float best_area = -1.0f;
            for (int k = 0; k < nc; ++k) {
                float4 lo = nodes2[2 * size_t(child[k])], hi = nodes2[2 * size_t(child[k]) + 1];
                if (__float_as_uint(hi.w) == 0) {
                    float ar = node2_area(lo, hi);
                    if (ar > best_area) {
                        best_area = ar;
                        best = k;
                    }
                }
            }
            if (best < 0)
                break;
            uint32_t a2 = __float_as_uint(nodes2[2 * size_t(child[best])].w);
            if (a2 + 1u >= n_nodes2) {
                atomicOr(status, ERR_BUILD);
                return;
            }
            child[best] = a2;
            child[nc++] = a2 + 1;
        }
    }
    float lo[3][4], hi[3][4];
    uint32_t idx[4], cnt[4];
    for (int k = 0; k < 4; ++k) {
        if (k >= nc || child[k] >= n_nodes2) {
            for (int ax = 0; ax < 3; ++ax) {
                lo[ax][k] = 0.0f;
                hi[ax][k] = 0.0f;
            }
            idx[k] = 0;
            cnt[k] = EMPTY_CHILD;
            if (k < nc)
                atomicOr(status, ERR_BUILD);
            continue;
        }
        float4 l = nodes2[2 * size_t(child[k])], h = nodes2[2 * size_t(child[k]) + 1];
        lo[0][k] = l.x;
        lo[1][k] = l.y;
        lo[2][k] = l.z;
        hi[0][k] = h.x;
        hi[1][k] = h.y;
        hi[2][k] = h.z;
        uint32_t b = __float_as_uint(h.w);
        if (b != 0) {  // leaf
            idx[k] = __float_as_uint(l.w);
            cnt[k] = b;
        } else {
            uint32_t q = atomicAdd(node4_count, 1u);
            if (q >= node4_cap) {
                atomicOr(status, ERR_BUILD);
                idx[k] = 0;
                cnt[k] = EMPTY_CHILD;
                continue;
            }
            idx[k] = q;
            cnt[k] = 0;
            uint32_t slot = atomicAdd(out_count, 1u);
            out_q[slot] = make_uint2(child[k], q);
        }
    }
    float4* o = nodes4 + 8 * size_t(job.y);
    o[0] = make_float4(lo[0][0], lo[0][1], lo[0][2], lo[0][3]);
    o[1] = make_float4(hi[0][0], hi[0][1], hi[0][2], hi[0][3]);
    o[2] = make_float4(lo[1][0], lo[1][1], lo[1][2], lo[1][3]);
    o[3] = make_float4(hi[1][0], hi[1][1], hi[1][2], hi[1][3]);
    o[4] = make_float4(lo[2][0], lo[2][1], lo[2][2], lo[2][3]);
    o[5] = make_float4(hi[2][0], hi[2][1], hi[2][2], hi[2][3]);
    o[6] = make_float4(__uint_as_float(idx[0]), __uint_as_float(idx[1]), __uint_as_float(idx[2]),
                       __uint_as_float(idx[3]));
    o[7] = make_float4(__uint_as_float(cnt[0]), __uint_as_float(cnt[1]), __uint_as_float(cnt[2]),
                       __uint_as_float(cnt[3]));
}

// ---------------------------------------------------------------------------------------------
// PLOC: parallel locally-ordered clustering (Meister & Bittner, "Parallel Locally-Ordered
// Clustering for Bounding Volume Hierarchy Construction", IEEE TVCG 2018).  Clusters start as
// the primitives in Morton order; each round every cluster finds, among the PLOC_R clusters on
// either side in the current order, the one whose union box has the smallest surface area;
// mutual nearest neighbours merge into a new node that takes the lower one's place, and the
// array is compacted.  Ties are broken by (area, index distance, parity of the lower index,
// lower index), a total order on pairs, so the globally closest pair is always mutual and every
// round merges; the parity rule pairs (0,1), (2,3), ... when many boxes are equal (coincident
// primitives), so such runs still halve every round.  Because a new node is
// only made from two finished clusters, its surface-area cost and the leaf-collapse decision
// (as in k_refit) are taken when it is created.
// ---------------------------------------------------------------------------------------------
constexpr int PLOC_R = 16;

__global__ void k_ploc_init(uint32_t n, const uint32_t* sorted_vals, const float4* box_lo,
                            const float4* box_hi, float4* nlo, float4* nhi, uint32_t* ncount,
                            uint8_t* ncol, uint32_t* cid, float c_isect)
{
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n)
        return;
    uint32_t p = sorted_vals[s];
    float4 lo = box_lo[p], hi = box_hi[p];
    float a = half_area(make_float3(lo.x, lo.y, lo.z), make_float3(hi.x, hi.y, hi.z));
    nlo[s] = make_float4(lo.x, lo.y, lo.z, c_isect * a);  // w: surface-area cost
    nhi[s] = make_float4(hi.x, hi.y, hi.z, 0.0f);
    ncount[s] = 1u;
    ncol[s] = 1u;
    cid[s] = s;
}

__global__ void __launch_bounds__(256) k_ploc_nn(uint32_t m, const uint32_t* cid,
                                                 const float4* nlo, const float4* nhi,
                                                 uint32_t* nn)
{
    __shared__ float3 slo[256 + 2 * PLOC_R], shi[256 + 2 * PLOC_R];
    const int b0 = int(blockIdx.x * 256u);
    for (int t = int(threadIdx.x); t < 256 + 2 * PLOC_R; t += 256) {
        int g = b0 - PLOC_R + t;
        if (g >= 0 && g < int(m)) {
            uint32_t c = cid[g];
            float4 lo = nlo[c], hi = nhi[c];
            slo[t] = make_float3(lo.x, lo.y, lo.z);
            shi[t] = make_float3(hi.x, hi.y, hi.z);
        }
    }
    __syncthreads();
    const int i = b0 + int(threadIdx.x);
    if (i >= int(m))
        return;
    const int li = int(threadIdx.x) + PLOC_R;
    const float3 lo = slo[li], hi = shi[li];
    float best = __int_as_float(0x7f800000);
    int bj = -1, bd = 0, bmn = 0;
    for (int d = 1; d <= PLOC_R; ++d) {
#pragma unroll
        for (int sgn = -1; sgn <= 1; sgn += 2) {
            const int j = i + sgn * d;
            if (j < 0 || j >= int(m))
                continue;
            const int lj = li + sgn * d;
            float a = half_area(f3min(lo, slo[lj]), f3max(hi, shi[lj]));
            if (!(a == a))
                a = __int_as_float(0x7f800000);
            const int mn = min(i, j);
            bool better = bj < 0 || a < best;
            if (!better && a == best) {
                if (d != bd)
                    better = d < bd;
                else if ((mn & 1) != (bmn & 1))
                    better = (mn & 1) < (bmn & 1);
                else
                    better = mn < bmn;
            }
            if (better) {
                best = a;
                bj = j;
                bd = d;
                bmn = mn;
            }
        }
    }
    nn[i] = bj < 0 ? uint32_t(i) : uint32_t(bj);
}

// flags: high word 1 if the cluster leads a merge (mutual pair, lower index), low word 1 if a
// cluster survives at this index (a leader's new node, or an unmerged cluster)
__global__ void k_ploc_flags(uint32_t m, const uint32_t* nn, unsigned long long* flags)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m)
        return;
    uint32_t j = nn[i];
    bool mutual = j != i && j < m && nn[j] == i;
    bool lead = mutual && i < j;
    bool keep = !mutual || i < j;
    flags[i] = ((unsigned long long)(lead ? 1u : 0u) << 32) | (keep ? 1ull : 0ull);
}

__global__ void k_ploc_merge(uint32_t m, const uint32_t* cid, const uint32_t* nn,
                             const unsigned long long* flags, const unsigned long long* prefix,
                             uint32_t next, uint32_t node_cap, float4* nlo, float4* nhi,
                             uint2* nchild, uint32_t* ncount, uint8_t* ncol, uint32_t* cid_out,
                             int leaf_max, float c_trav, float c_isect, uint32_t* status)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m)
        return;
    const unsigned long long f = flags[i], pre = prefix[i];
    const uint32_t out = uint32_t(pre & 0xffffffffull);
    if (f >> 32) {
        const uint32_t k = next + uint32_t(pre >> 32);
        if (k >= node_cap || out >= m) {
            atomicOr(status, ERR_BUILD);
            return;
        }
        const uint32_t a = cid[i], b = cid[nn[i]];
        const float4 la = nlo[a], ha = nhi[a], lb = nlo[b], hb = nhi[b];
        const float3 lo = f3min(make_float3(la.x, la.y, la.z), make_float3(lb.x, lb.y, lb.z));
        const float3 hi = f3max(make_float3(ha.x, ha.y, ha.z), make_float3(hb.x, hb.y, hb.z));
        const float area = half_area(lo, hi);
        const uint32_t count = ncount[a] + ncount[b];
        const float split_cost = c_trav * area + la.w + lb.w;
        const float leaf_cost = c_isect * area * float(count);
        const bool col = count <= uint32_t(leaf_max) && leaf_cost <= split_cost;
        nlo[k] = make_float4(lo.x, lo.y, lo.z, col ? leaf_cost : split_cost);
        nhi[k] = make_float4(hi.x, hi.y, hi.z, 0.0f);
        nchild[k] = make_uint2(a, b);
        ncount[k] = count;
        ncol[k] = col ? 1u : 0u;
        cid_out[out] = k;
    } else if (f & 1ull) {
        if (out >= m) {
            atomicOr(status, ERR_BUILD);
            return;
        }
        cid_out[out] = cid[i];
    }
}

// Top-down emission into the compacted binary layout (children of an interior node adjacent,
// leaves naming a run of leaf slots), one tree level per launch.  Queue items: (node, output
// slot, first leaf slot).  A leaf of the output tree (a primitive, or a collapsed subtree) lists
// its primitives left to right into leaf_vals.
__global__ void k_ploc_emit(uint32_t n, const uint4* in_q, const uint32_t* in_count, uint4* out_q,
                            uint32_t* out_count, uint32_t* node_counter, uint32_t node_cap,
                            const float4* nlo, const float4* nhi, const uint2* nchild,
                            const uint32_t* ncount, const uint8_t* ncol,
                            const uint32_t* sorted_vals, uint32_t* leaf_vals, float4* nodes,
                            uint32_t* status)
{
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= *in_count)
        return;
    const uint4 q = in_q[t];
    const uint32_t k = q.x, slot = q.y, off = q.z;
    if (k >= 2 * n - 1 || slot >= node_cap) {
        atomicOr(status, ERR_BUILD);
        return;
    }
    const float4 lo = nlo[k], hi = nhi[k];
    const uint32_t cnt = ncount[k];
    if (k < n || ncol[k]) {
        if (off > n || cnt > n - off) {
            atomicOr(status, ERR_BUILD);
            return;
        }
        write_node(nodes, slot, lo, hi, off, cnt);
        uint32_t stack[32];
        int sp = 0;
        stack[sp++] = k;
        uint32_t w = 0;
        while (sp > 0) {
            const uint32_t c = stack[--sp];
            if (c < n) {
                if (w < cnt)
                    leaf_vals[off + w] = sorted_vals[c];
                ++w;
            } else if (c < 2 * n - 1 && sp + 2 <= 32) {
                const uint2 ch = nchild[c];
                stack[sp++] = ch.y;
                stack[sp++] = ch.x;
            } else {
                atomicOr(status, ERR_BUILD);
                return;
            }
        }
        if (w != cnt)
            atomicOr(status, ERR_BUILD);
        return;
    }
    const uint32_t p = atomicAdd(node_counter, 2u);
    if (p + 1u >= node_cap) {
        atomicOr(status, ERR_BUILD);
        return;
    }
    write_node(nodes, slot, lo, hi, p, 0u);
    const uint2 ch = nchild[k];
    const uint32_t o = atomicAdd(out_count, 2u);
    if (o + 1u >= n) {  // a level of a binary tree over n leaves has fewer than n nodes
        atomicOr(status, ERR_BUILD);
        return;
    }
    out_q[o] = make_uint4(ch.x, p, off, 0u);
    out_q[o + 1] = make_uint4(ch.y, p + 1u, off + ncount[ch.x], 0u);
}

// ---------------------------------------------------------------------------------------------
// Refit: new primitive boxes in an unchanged topology (the primitives moved, their number did
// not).  Leaves recompute their box from their primitives; each interior node is written by the
// second of its two children to arrive (one counter per node), as in k_refit.
// ---------------------------------------------------------------------------------------------
__global__ void k_parents(const float4* nodes, uint32_t n_nodes, uint32_t* parent,
                          uint32_t* status)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_nodes)
        return;
    if (__float_as_uint(nodes[2 * size_t(i) + 1].w) != 0u)
        return;  // leaf
    uint32_t a = __float_as_uint(nodes[2 * size_t(i)].w);
    if (a == 0u || a + 1u >= n_nodes) {
        atomicOr(status, ERR_BUILD);
        return;
    }
    parent[a] = i;
    parent[a + 1] = i;
}

__global__ void k_refit_tree(float4* nodes, uint32_t n_nodes, const uint32_t* order, uint32_t n,
                             const float4* box_lo, const float4* box_hi, const uint32_t* parent,
                             uint32_t* arrive, uint32_t* status)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_nodes)
        return;
    const float4 l0 = nodes[2 * size_t(i)], h0 = nodes[2 * size_t(i) + 1];
    const uint32_t count = __float_as_uint(h0.w);
    if (count == 0u)
        return;  // interior: written by its children
    const uint32_t first = __float_as_uint(l0.w);
    if (first > n || count > n - first) {
        atomicOr(status, ERR_BUILD);
        return;
    }
    float3 lo = make_float3(__int_as_float(0x7f800000), __int_as_float(0x7f800000),
                            __int_as_float(0x7f800000));
    float3 hi = make_float3(-lo.x, -lo.y, -lo.z);
    for (uint32_t s = first; s < first + count; ++s) {
        const uint32_t p = order[s];
        if (p >= n) {
            atomicOr(status, ERR_BUILD);
            return;
        }
        const float4 bl = box_lo[p], bh = box_hi[p];
        lo = f3min(lo, make_float3(bl.x, bl.y, bl.z));
        hi = f3max(hi, make_float3(bh.x, bh.y, bh.z));
    }
    __stcg(&nodes[2 * size_t(i)], make_float4(lo.x, lo.y, lo.z, l0.w));
    __stcg(&nodes[2 * size_t(i) + 1], make_float4(hi.x, hi.y, hi.z, h0.w));
    uint32_t node = i == 0u ? 0xFFFFFFFFu : parent[i];
    for (int guard = 0; node != 0xFFFFFFFFu; ++guard) {
        if (node >= n_nodes || guard > 4096) {
            atomicOr(status, ERR_BUILD);
            return;
        }
        __threadfence();
        if (atomicAdd(arrive + node, 1u) == 0u)
            return;
        __threadfence();
        const float4 nl = __ldcg(&nodes[2 * size_t(node)]);
        const float4 nh = __ldcg(&nodes[2 * size_t(node) + 1]);
        const uint32_t a = __float_as_uint(nl.w);
        if (a + 1u >= n_nodes) {
            atomicOr(status, ERR_BUILD);
            return;
        }
        const float4 al = __ldcg(&nodes[2 * size_t(a)]), ah = __ldcg(&nodes[2 * size_t(a) + 1]);
        const float4 bl = __ldcg(&nodes[2 * size_t(a + 1)]),
                     bh = __ldcg(&nodes[2 * size_t(a + 1) + 1]);
        const float3 ulo = f3min(make_float3(al.x, al.y, al.z), make_float3(bl.x, bl.y, bl.z));
        const float3 uhi = f3max(make_float3(ah.x, ah.y, ah.z), make_float3(bh.x, bh.y, bh.z));
        __stcg(&nodes[2 * size_t(node)], make_float4(ulo.x, ulo.y, ulo.z, nl.w));
        __stcg(&nodes[2 * size_t(node) + 1], make_float4(uhi.x, uhi.y, uhi.z, nh.w));
        node = node == 0u ? 0xFFFFFFFFu : parent[node];
    }
}

inline uint32_t blocks_for(size_t n, int threads) { return uint32_t((n + threads - 1) / threads); }

}  // namespace

size_t leaf_record_float4s(int type) { return type == FR_GEOM_SPHERE ? 1 : 2; }

namespace {
size_t record_size(const BuildInput& in) { return leaf_record_float4s(in.type); }
size_t record_size(const PartsInput&) { return 2; }
constexpr bool is_parts(const BuildInput&) { return false; }
constexpr bool is_parts(const PartsInput&) { return true; }
}  // namespace

// Collapse the binary tree in out.nodes into out.nodes4 (top-down, one launch per level).
cudaError_t collapse4(BvhBuffers& out, Scratch& scratch, uint32_t* status, cudaStream_t st)
{
    out.n_nodes4 = 0;
    if (out.n_nodes == 0)
        return cudaSuccess;
    const uint32_t cap = (out.n_nodes + 1) / 2 + 1;  // at most one per binary interior node
    cudaError_t e;
    if ((e = out.nodes4.reserve(size_t(8) * cap)) != cudaSuccess)
        return e;
    ScratchLayout L;
    uint2* qa = L.take<uint2>(cap);
    uint2* qb = L.take<uint2>(cap);
    uint32_t* cnt = L.take<uint32_t>(4);
    if ((e = scratch.reserve(L.bytes)) != cudaSuccess)
        return e;
    L.bind(scratch.ptr);
    qa = L.at(qa);
    qb = L.at(qb);
    cnt = L.at(cnt);
    // cnt[0]: jobs in qa, cnt[1]: jobs in qb, cnt[2]: 4-wide nodes allocated
    uint32_t init[3] = {1u, 0u, 1u};
    uint2 root = make_uint2(0u, 0u);
    if ((e = cudaMemcpyAsync(cnt, init, sizeof(init), cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return e;
    if ((e = cudaMemcpyAsync(qa, &root, sizeof(root), cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return e;
    uint32_t jobs = 1;
    for (int level = 0; jobs > 0 && level < 256; ++level) {
        uint32_t* cin = cnt + (level & 1);
        uint32_t* cout = cnt + ((level + 1) & 1);
        uint2* qin = (level & 1) ? qb : qa;
        uint2* qout = (level & 1) ? qa : qb;
        if ((e = cudaMemsetAsync(cout, 0, sizeof(uint32_t), st)) != cudaSuccess)
            return e;
        k_collapse4<<<blocks_for(jobs, 256), 256, 0, st>>>(out.nodes.ptr, out.n_nodes, qin, cin,
                                                           qout, cout, cnt + 2, cap,
                                                           out.nodes4.ptr, status);
        if ((e = cudaMemcpyAsync(&jobs, cout, sizeof(uint32_t), cudaMemcpyDeviceToHost, st)) !=
            cudaSuccess)
            return e;
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess)
            return e;
    }
    uint32_t n4 = 0;
    if ((e = cudaMemcpyAsync(&n4, cnt + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, st)) !=
        cudaSuccess)
        return e;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess)
        return e;
    out.n_nodes4 = n4 < cap ? n4 : cap;
    return cudaGetLastError();
}

template <class In>
static cudaError_t build_impl(const In& in, uint32_t n, const BuildParams& bp, BvhBuffers& out,
                              Scratch& scratch, uint32_t* status, cudaStream_t st)
{
    out.n_nodes = 0;
    if (n == 0)
        return cudaSuccess;
    const int T = 256;
    const size_t rec = record_size(in);
    // persistent outputs
    cudaError_t e;
    if ((e = out.nodes.reserve(size_t(2) * (2 * size_t(n) - 1))) != cudaSuccess)
        return e;
    if ((e = out.leaf_data.reserve(rec * n)) != cudaSuccess)
        return e;
    if ((e = out.order.reserve(n)) != cudaSuccess)
        return e;
    if (is_parts(in) && (e = out.leaf_geom.reserve(n)) != cudaSuccess)
        return e;

    // scratch carve-up
    size_t sort_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (uint64_t*)nullptr, (uint64_t*)nullptr,
                                    (uint32_t*)nullptr, (uint32_t*)nullptr, int(n), 0, 63, st);
    size_t scan_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                  int(n), st);
    ScratchLayout L;
    float4* box_lo = L.take<float4>(n);
    float4* box_hi = L.take<float4>(n);
    uint64_t* keys = L.take<uint64_t>(n);
    uint64_t* keys_sorted = L.take<uint64_t>(n);
    uint32_t* vals = L.take<uint32_t>(n);
    uint32_t* vals_sorted = L.take<uint32_t>(n);
    int2* range = L.take<int2>(n);
    uint32_t* split = L.take<uint32_t>(n);
    uint32_t* parent_int = L.take<uint32_t>(n);
    uint32_t* parent_leaf = L.take<uint32_t>(n);
    uint32_t* arrive = L.take<uint32_t>(n);
    NodeInfo* info = L.take<NodeInfo>(n);
    uint8_t* collapse = L.take<uint8_t>(n);
    uint32_t* keep = L.take<uint32_t>(n);
    uint32_t* removed = L.take<uint32_t>(n);
    uint32_t* pair_index = L.take<uint32_t>(n);
    uint32_t* cbounds = L.take<uint32_t>(8);
    // PLOC working set (only carved when that builder is selected)
    const bool ploc = bp.builder == 1 && n >= 2;
    const size_t nn2 = ploc ? 2 * size_t(n) : 0, nn1 = ploc ? size_t(n) : 0;
    size_t scan64_bytes = 0;
    if (ploc)
        cub::DeviceScan::ExclusiveSum(nullptr, scan64_bytes, (unsigned long long*)nullptr,
                                      (unsigned long long*)nullptr, int(n), st);
    float4* p_lo = L.take<float4>(nn2);
    float4* p_hi = L.take<float4>(nn2);
    uint2* p_child = L.take<uint2>(nn2);
    uint32_t* p_count = L.take<uint32_t>(nn2);
    uint8_t* p_col = L.take<uint8_t>(nn2);
    uint32_t* p_cid_a = L.take<uint32_t>(nn1);
    uint32_t* p_cid_b = L.take<uint32_t>(nn1);
    uint32_t* p_nn = L.take<uint32_t>(nn1);
    unsigned long long* p_flags = L.take<unsigned long long>(nn1);
    unsigned long long* p_prefix = L.take<unsigned long long>(nn1);
    uint4* p_qa = L.take<uint4>(nn1);
    uint4* p_qb = L.take<uint4>(nn1);
    uint32_t* p_leaf_vals = L.take<uint32_t>(nn1);
    uint32_t* p_cnt = L.take<uint32_t>(ploc ? 4 : 0);
    size_t tmp_need = sort_bytes > scan_bytes ? sort_bytes : scan_bytes;
    if (scan64_bytes > tmp_need)
        tmp_need = scan64_bytes;
    uint8_t* cub_tmp = L.take<uint8_t>(tmp_need);
    if ((e = scratch.reserve(L.bytes)) != cudaSuccess)
        return e;
    L.bind(scratch.ptr);
#define FR_RELOC(p) p = L.at(p)
    FR_RELOC(box_lo);
    FR_RELOC(box_hi);
    FR_RELOC(keys);
    FR_RELOC(keys_sorted);
    FR_RELOC(vals);
    FR_RELOC(vals_sorted);
    FR_RELOC(range);
    FR_RELOC(split);
    FR_RELOC(parent_int);
    FR_RELOC(parent_leaf);
    FR_RELOC(arrive);
    FR_RELOC(info);
    FR_RELOC(collapse);
    FR_RELOC(keep);
    FR_RELOC(removed);
    FR_RELOC(pair_index);
    FR_RELOC(cbounds);
    FR_RELOC(p_lo);
    FR_RELOC(p_hi);
    FR_RELOC(p_child);
    FR_RELOC(p_count);
    FR_RELOC(p_col);
    FR_RELOC(p_cid_a);
    FR_RELOC(p_cid_b);
    FR_RELOC(p_nn);
    FR_RELOC(p_flags);
    FR_RELOC(p_prefix);
    FR_RELOC(p_qa);
    FR_RELOC(p_qb);
    FR_RELOC(p_leaf_vals);
    FR_RELOC(p_cnt);
    FR_RELOC(cub_tmp);
#undef FR_RELOC

    // centroid bounds: min slots start at 0xff.., max slots at 0
    if ((e = cudaMemsetAsync(cbounds, 0xff, 3 * sizeof(uint32_t), st)) != cudaSuccess)
        return e;
    if ((e = cudaMemsetAsync(cbounds + 3, 0, 3 * sizeof(uint32_t), st)) != cudaSuccess)
        return e;
    uint32_t gb = blocks_for(n, T);
    if (gb > 4096)
        gb = 4096;
    k_bounds<<<gb, T, 0, st>>>(in, n, box_lo, box_hi, cbounds);
    k_morton<<<blocks_for(n, T), T, 0, st>>>(n, box_lo, box_hi, cbounds, keys, vals);
    size_t tmp_bytes = sort_bytes;
    if ((e = cub::DeviceRadixSort::SortPairs(cub_tmp, tmp_bytes, keys, keys_sorted, vals,
                                             vals_sorted, int(n), 0, 63, st)) != cudaSuccess)
        return e;
    const uint32_t* leaf_order = vals_sorted;  // leaf slot -> primitive
    if (n == 1) {
        k_single_leaf<<<1, 1, 0, st>>>(box_lo, box_hi, out.nodes.ptr);
        out.n_nodes = 1;
    }
    bool built = n == 1;
    if (!built && ploc) {
        const uint32_t node_cap = 2 * n - 1;
        k_ploc_init<<<blocks_for(n, T), T, 0, st>>>(n, vals_sorted, box_lo, box_hi, p_lo, p_hi,
                                                   p_count, p_col, p_cid_a, bp.c_isect);
        uint32_t m = n, next = n;
        uint32_t* cin = p_cid_a;
        uint32_t* cout = p_cid_b;
        bool converged = true;
        for (int round = 0; m > 1; ++round) {
            if (round > 1024) {
                converged = false;
                break;
            }
            k_ploc_nn<<<blocks_for(m, 256), 256, 0, st>>>(m, cin, p_lo, p_hi, p_nn);
            k_ploc_flags<<<blocks_for(m, T), T, 0, st>>>(m, p_nn, p_flags);
            size_t tb = tmp_need;
            if ((e = cub::DeviceScan::ExclusiveSum(cub_tmp, tb, p_flags, p_prefix, int(m), st)) !=
                cudaSuccess)
                return e;
            k_ploc_merge<<<blocks_for(m, T), T, 0, st>>>(m, cin, p_nn, p_flags, p_prefix, next,
                                                        node_cap, p_lo, p_hi, p_child, p_count,
                                                        p_col, cout, bp.leaf_max, bp.c_trav,
                                                        bp.c_isect, status);
            unsigned long long last[2];
            if ((e = cudaMemcpyAsync(last, p_flags + (m - 1), 8, cudaMemcpyDeviceToHost, st)) !=
                cudaSuccess)
                return e;
            if ((e = cudaMemcpyAsync(last + 1, p_prefix + (m - 1), 8, cudaMemcpyDeviceToHost,
                                     st)) != cudaSuccess)
                return e;
            if ((e = cudaStreamSynchronize(st)) != cudaSuccess)
                return e;
            const uint32_t merges = uint32_t(last[0] >> 32) + uint32_t(last[1] >> 32);
            const uint32_t kept = uint32_t(last[0] & 0xffffffffull) +
                                  uint32_t(last[1] & 0xffffffffull);
            if (merges == 0 || kept >= m || next + merges > node_cap) {
                converged = false;  // no progress: build the LBVH instead
                break;
            }
            next += merges;
            m = kept;
            uint32_t* tmp = cin;
            cin = cout;
            cout = tmp;
        }
        uint32_t root = 0;
        if (converged &&
            (e = cudaMemcpyAsync(&root, cin, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            return e;
        // emission: counters [0], [1] queue lengths, [2] output nodes
        uint32_t init[3] = {1u, 0u, 1u};
        if ((e = cudaMemcpyAsync(p_cnt, init, sizeof(init), cudaMemcpyHostToDevice, st)) !=
            cudaSuccess)
            return e;
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess)
            return e;
        uint4 first = make_uint4(root, 0u, 0u, 0u);
        if ((e = cudaMemcpyAsync(p_qa, &first, sizeof(first), cudaMemcpyHostToDevice, st)) !=
            cudaSuccess)
            return e;
        uint32_t jobs = converged ? 1u : 0u;
        for (int level = 0; jobs > 0; ++level) {
            if (level > 4096)
                return cudaErrorUnknown;
            uint32_t* cq_in = p_cnt + (level & 1);
            uint32_t* cq_out = p_cnt + ((level + 1) & 1);
            uint4* q_in = (level & 1) ? p_qb : p_qa;
            uint4* q_out = (level & 1) ? p_qa : p_qb;
            if ((e = cudaMemsetAsync(cq_out, 0, 4, st)) != cudaSuccess)
                return e;
            k_ploc_emit<<<blocks_for(jobs, T), T, 0, st>>>(n, q_in, cq_in, q_out, cq_out, p_cnt + 2,
                                                          node_cap, p_lo, p_hi, p_child, p_count,
                                                          p_col, vals_sorted, p_leaf_vals,
                                                          out.nodes.ptr, status);
            if ((e = cudaMemcpyAsync(&jobs, cq_out, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
                return e;
            if ((e = cudaStreamSynchronize(st)) != cudaSuccess)
                return e;
        }
        uint32_t n_out = 0;
        if ((e = cudaMemcpyAsync(&n_out, p_cnt + 2, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            return e;
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess)
            return e;
        if (converged) {
            out.n_nodes = n_out < node_cap ? n_out : node_cap;
            leaf_order = p_leaf_vals;
            built = true;
        }
    }
    if (!built) {
        // unset parents read as 0xffffffff (out of range) and are reported, never followed
        if ((e = cudaMemsetAsync(parent_int, 0xff, n * sizeof(uint32_t), st)) != cudaSuccess)
            return e;
        if ((e = cudaMemsetAsync(parent_leaf, 0xff, n * sizeof(uint32_t), st)) != cudaSuccess)
            return e;
        k_karras<<<blocks_for(n - 1, T), T, 0, st>>>(n, keys_sorted, range, split, parent_int,
                                                    parent_leaf);
        if ((e = cudaMemsetAsync(arrive, 0, n * sizeof(uint32_t), st)) != cudaSuccess)
            return e;
        k_refit<<<blocks_for(n, T), T, 0, st>>>(n, vals_sorted, box_lo, box_hi, range, split,
                                                parent_int, parent_leaf, arrive, info, collapse,
                                                bp.leaf_max, bp.c_trav, bp.c_isect, status);
        if ((e = cudaMemsetAsync(keep, 0, n * sizeof(uint32_t), st)) != cudaSuccess)
            return e;
        k_mark<<<blocks_for(n - 1, T), T, 0, st>>>(n, split, parent_int, collapse, keep, removed);
        tmp_bytes = scan_bytes;
        if ((e = cub::DeviceScan::ExclusiveSum(cub_tmp, tmp_bytes, keep, pair_index, int(n),
                                               st)) != cudaSuccess)
            return e;
        k_emit<<<blocks_for(n - 1, T), T, 0, st>>>(n, range, split, collapse, removed, pair_index,
                                                   info, vals_sorted, box_lo, box_hi,
                                                   out.nodes.ptr);
        // node count = 1 + 2 * (number of kept pairs) = 1 + 2 * (pair_index[n-1] + keep[n-1])
        uint32_t tail[2];
        if ((e = cudaMemcpyAsync(tail, pair_index + (n - 1), sizeof(uint32_t),
                                 cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            return e;
        if ((e = cudaMemcpyAsync(tail + 1, keep + (n - 1), sizeof(uint32_t),
                                 cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            return e;
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess)
            return e;
        out.n_nodes = 1u + 2u * (tail[0] + tail[1]);
    }
    k_gather<<<blocks_for(n, T), T, 0, st>>>(in, n, leaf_order, out.leaf_data.ptr, out.order.ptr,
                                             out.leaf_geom.ptr);
    if ((e = cudaGetLastError()) != cudaSuccess)
        return e;
    if (bp.width != 4) {
        out.n_nodes4 = 0;
        return cudaSuccess;
    }
    return collapse4(out, scratch, status, st);
}

static void k_combined_order_for(const BuildInput&, uint32_t, BvhBuffers&, uint32_t*, uint32_t*,
                                 cudaStream_t)
{
}

static void k_combined_order_for(const PartsInput& in, uint32_t n, BvhBuffers& out,
                                 uint32_t* combined, uint32_t* status, cudaStream_t st)
{
    k_combined_order<<<blocks_for(n, 256), 256, 0, st>>>(in, n, out.order.ptr, out.leaf_geom.ptr,
                                                         combined, status);
}

template <class In>
static cudaError_t refit_impl(const In& in, uint32_t n, const BuildParams& bp, BvhBuffers& out,
                              Scratch& scratch, uint32_t* status, cudaStream_t st)
{
    if (n == 0 || out.n_nodes == 0 || out.order.cap < n || out.leaf_data.cap < record_size(in) * n ||
        (is_parts(in) && out.leaf_geom.cap < n))
        return cudaErrorInvalidValue;
    const int T = 256;
    const uint32_t nn = out.n_nodes;
    ScratchLayout L;
    float4* box_lo = L.take<float4>(n);
    float4* box_hi = L.take<float4>(n);
    uint32_t* parent = L.take<uint32_t>(nn);
    uint32_t* arrive = L.take<uint32_t>(nn);
    uint32_t* cbounds = L.take<uint32_t>(8);
    uint32_t* combined = L.take<uint32_t>(is_parts(in) ? n : 0);
    cudaError_t e;
    if ((e = scratch.reserve(L.bytes)) != cudaSuccess)
        return e;
    L.bind(scratch.ptr);
    box_lo = L.at(box_lo);
    box_hi = L.at(box_hi);
    parent = L.at(parent);
    arrive = L.at(arrive);
    cbounds = L.at(cbounds);
    combined = L.at(combined);
    // leaf slot -> index in the build's numbering (the geometry's own, or the combined one)
    const uint32_t* slot_prim = out.order.ptr;
    if (is_parts(in)) {
        k_combined_order_for(in, n, out, combined, status, st);
        slot_prim = combined;
    }
    if ((e = cudaMemsetAsync(cbounds, 0xff, 3 * sizeof(uint32_t), st)) != cudaSuccess)
        return e;
    if ((e = cudaMemsetAsync(cbounds + 3, 0, 3 * sizeof(uint32_t), st)) != cudaSuccess)
        return e;
    uint32_t gb = blocks_for(n, T);
    if (gb > 4096)
        gb = 4096;
    k_bounds<<<gb, T, 0, st>>>(in, n, box_lo, box_hi, cbounds);
    // same leaf order: re-gather the moved primitives' records in place
    k_gather<<<blocks_for(n, T), T, 0, st>>>(in, n, slot_prim, out.leaf_data.ptr, out.order.ptr,
                                             out.leaf_geom.ptr);
    if ((e = cudaMemsetAsync(parent, 0xff, nn * sizeof(uint32_t), st)) != cudaSuccess)
        return e;
    if ((e = cudaMemsetAsync(arrive, 0, nn * sizeof(uint32_t), st)) != cudaSuccess)
        return e;
    k_parents<<<blocks_for(nn, T), T, 0, st>>>(out.nodes.ptr, nn, parent, status);
    k_refit_tree<<<blocks_for(nn, T), T, 0, st>>>(out.nodes.ptr, nn, slot_prim, n, box_lo,
                                                  box_hi, parent, arrive, status);
    if ((e = cudaGetLastError()) != cudaSuccess)
        return e;
    if (bp.width != 4) {
        out.n_nodes4 = 0;
        return cudaSuccess;
    }
    return collapse4(out, scratch, status, st);
}

namespace {
__global__ void k_part_boxes(PartsInput in, uint32_t n, float4* lo, float4* hi)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const Box b = prim_bounds(in, i);
    lo[i] = make_float4(b.lo.x, b.lo.y, b.lo.z, 0.0f);
    hi[i] = make_float4(b.hi.x, b.hi.y, b.hi.z, 0.0f);
}
}  // namespace

cudaError_t parts_boxes(const PartsInput& in, uint32_t n, float4* lo, float4* hi, cudaStream_t st)
{
    if (n == 0)
        return cudaSuccess;
    k_part_boxes<<<(n + 255) / 256, 256, 0, st>>>(in, n, lo, hi);
    return cudaGetLastError();
}

namespace {
// A reference's geometry word of a grid over parts: the geometry index with its type above it.
__global__ void k_tag_types(PartsInput in, uint32_t n, uint32_t* geom)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n)
        return;
    const uint32_t gi = geom[s];
    uint32_t type = 0;
    for (uint32_t p = 0; p < in.n_parts; ++p)
        if (in.geom[p] == gi)
            type = uint32_t(in.part[p].type);
    geom[s] = gi | (type << PART_TYPE_SHIFT);
}
}  // namespace

cudaError_t gather_parts(const PartsInput& in, const uint32_t* prims, uint32_t total,
                         float4* data, uint32_t* order, uint32_t* geom, cudaStream_t st)
{
    if (total == 0)
        return cudaSuccess;
    k_gather<<<(total + 255) / 256, 256, 0, st>>>(in, total, prims, data, order, geom);
    k_tag_types<<<(total + 255) / 256, 256, 0, st>>>(in, total, geom);
    return cudaGetLastError();
}

cudaError_t build_bvh(const BuildInput& in, uint32_t n, const BuildParams& bp, BvhBuffers& out,
                      Scratch& scratch, uint32_t* status, cudaStream_t st)
{
    return build_impl(in, n, bp, out, scratch, status, st);
}

cudaError_t build_bvh(const PartsInput& in, uint32_t n, const BuildParams& bp, BvhBuffers& out,
                      Scratch& scratch, uint32_t* status, cudaStream_t st)
{
    return build_impl(in, n, bp, out, scratch, status, st);
}

cudaError_t refit_bvh(const BuildInput& in, uint32_t n, const BuildParams& bp, BvhBuffers& out,
                      Scratch& scratch, uint32_t* status, cudaStream_t st)
{
    return refit_impl(in, n, bp, out, scratch, status, st);
}

cudaError_t refit_bvh(const PartsInput& in, uint32_t n, const BuildParams& bp, BvhBuffers& out,
                      Scratch& scratch, uint32_t* status, cudaStream_t st)
{
    return refit_impl(in, n, bp, out, scratch, status, st);
}

}  // namespace fr
