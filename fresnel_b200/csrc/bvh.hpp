// bvh.hpp -- device buffers and the LBVH builder's host interface.
#ifndef FR_BVH_HPP
#define FR_BVH_HPP

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

namespace fr {

// A growable device allocation: reserve() only reallocates when the request exceeds capacity.
template <class T> struct DevArray {
    T* ptr = nullptr;
    size_t cap = 0;  // elements
    cudaError_t reserve(size_t n)
    {
        if (n <= cap)
            return cudaSuccess;
        release();
        if (n == 0)
            return cudaSuccess;
        cudaError_t e = cudaMalloc((void**)&ptr, n * sizeof(T));
        if (e != cudaSuccess) {
            ptr = nullptr;
            cap = 0;
            return e;
        }
        cap = n;
        return cudaSuccess;
    }
    void release()
    {
        if (ptr)
            cudaFree(ptr);
        ptr = nullptr;
        cap = 0;
    }
    DevArray() = default;
    DevArray(const DevArray&) = delete;
    DevArray& operator=(const DevArray&) = delete;
    ~DevArray() { release(); }
};

// Byte scratch shared by the builds of one device.
struct Scratch {
    DevArray<unsigned char> buf;
    void* ptr = nullptr;
    cudaError_t reserve(size_t bytes)
    {
        cudaError_t e = buf.reserve(bytes);
        ptr = buf.ptr;
        return e;
    }
};

// Carves typed, 256-byte aligned sub-arrays out of one scratch block: take() records offsets
// (returned as pointers relative to address 0), bind() sets the base, at() relocates.
struct ScratchLayout {
    size_t bytes = 0;
    char* base = nullptr;
    template <class T> T* take(size_t n)
    {
        bytes = (bytes + 255) & ~size_t(255);
        T* off = reinterpret_cast<T*>(bytes);
        bytes += n * sizeof(T);
        return off;
    }
    void bind(void* b) { base = static_cast<char*>(b); }
    template <class T> T* at(T* off) const
    {
        return reinterpret_cast<T*>(base + reinterpret_cast<size_t>(off));
    }
};

struct BuildInput {
    int type;  // FR_GEOM_*
    const float* position;
    const float* radius;
    const float* points;
    const float* orientation;
    const float* vertices;
    uint32_t n_faces;
    float poly_radius;  // polyhedron / polygon: bounding radius about the position
    int instances;      // mesh: one primitive per instance (grids over parts) instead of one
                        // per triangle (trees)
};

// Several geometries' primitives in one tree (a scene's combined BVH): primitive i of the
// combined numbering is primitive i - first[p] of part p, where first[p] <= i < first[p + 1].
constexpr int MAX_PARTS = 8;
struct PartsInput {
    BuildInput part[MAX_PARTS];
    uint32_t first[MAX_PARTS + 1];
    uint32_t geom[MAX_PARTS];  // scene geometry index of each part
    uint32_t n_parts;
};

struct BuildParams {
    int builder = 0;       // 0: LBVH (Karras hierarchy); 1: PLOC (locally-ordered clustering)
    int width = 4;         // 2: binary tree only; 4: also collapse to the 4-wide tree
    int leaf_max = 2;      // largest leaf the SAH collapse may form
    float c_trav = 1.0f;   // cost of one child-pair visit, in units of one primitive test
    float c_isect = 1.0f;
};

struct BvhBuffers {
    DevArray<float4> nodes;      // binary tree, 2 float4 per node
    DevArray<float4> nodes4;     // 4-wide tree traversed by the renderers, 8 float4 per node
    uint32_t n_nodes4 = 0;
    DevArray<float4> leaf_data;  // leaf_record_float4s(type) per primitive
    DevArray<uint32_t> order;    // leaf slot -> primitive index (within its geometry)
    DevArray<uint32_t> leaf_geom;  // combined trees: leaf slot -> scene geometry index
    uint32_t n_nodes = 0;
};

size_t leaf_record_float4s(int type);

// Collapse the binary tree of `out` into its 4-wide tree (called by build_bvh).
cudaError_t collapse4(BvhBuffers& out, Scratch& scratch, uint32_t* status, cudaStream_t st);

// New boxes for a tree built by build_bvh over the same n primitives (they moved; their number
// and the build parameters did not): primitive boxes, leaf records and every node's box are
// recomputed bottom-up in the existing topology, then the 4-wide tree is collapsed again.
// Returns cudaErrorInvalidValue if `out` holds no tree for n primitives.
cudaError_t refit_bvh(const BuildInput& in, uint32_t n, const BuildParams& bp, BvhBuffers& out,
                      Scratch& scratch, uint32_t* status, cudaStream_t st);

// The same for a combined tree over the parts of `in` (n = in.first[in.n_parts] primitives):
// every leaf slot holds 2 float4 (a sphere uses the first) and its geometry in leaf_geom.
cudaError_t refit_bvh(const PartsInput& in, uint32_t n, const BuildParams& bp, BvhBuffers& out,
                      Scratch& scratch, uint32_t* status, cudaStream_t st);
cudaError_t build_bvh(const PartsInput& in, uint32_t n, const BuildParams& bp, BvhBuffers& out,
                      Scratch& scratch, uint32_t* status, cudaStream_t st);

// The padded box of each of the n primitives of the parts of `in` (one thread per primitive, as
// the tree builds compute them; an empty box, lower > upper, for a primitive left out).
cudaError_t parts_boxes(const PartsInput& in, uint32_t n, float4* lo, float4* hi, cudaStream_t st);

// Geometry word of a grid-over-parts reference: the scene geometry index (below 2^24), with the
// geometry's FR_GEOM_* type from bit PART_TYPE_SHIFT on, so that a walk learns a reference's type
// without reading the geometry table.
constexpr uint32_t PART_TYPE_SHIFT = 24;

// For each of `total` references to primitives of `in` (combined numbering, prims[r]): its
// leaf-slot record (2 float4 at data + 2 r), its index within its geometry and its geometry word.
cudaError_t gather_parts(const PartsInput& in, const uint32_t* prims, uint32_t total,
                         float4* data, uint32_t* order, uint32_t* geom, cudaStream_t st);

// Build the BVH of n primitives (n == 0 leaves an empty tree).  Synchronises the stream once
// to read back the node count.
// Construction errors (an inconsistent hierarchy) are reported by or-ing ERR_BUILD into
// *status; no kernel follows an out-of-range index.
cudaError_t build_bvh(const BuildInput& in, uint32_t n, const BuildParams& bp, BvhBuffers& out,
                      Scratch& scratch, uint32_t* status, cudaStream_t st);

}  // namespace fr

#endif
