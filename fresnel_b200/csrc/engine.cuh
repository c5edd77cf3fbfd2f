// engine.cuh -- device-side scene layout and closest-hit traversal.
//
// Layout in HBM, per geometry:
//   nodes4     4-wide BVH nodes of 128 bytes (one cache line), eight float4: lo.x, hi.x, lo.y,
//              hi.y, lo.z, hi.z of the four children (one child per float4 lane), then the
//              child references and counts (count 0: interior child, its node index; count
//              n > 0: leaf of n primitives starting at that slot; EMPTY_CHILD: unused slot).
//              Node 0 is the root.  The renderers traverse this tree.
//   nodes      the binary LBVH it is collapsed from, 32-byte nodes of two float4:
//              (lo.xyz, a) and (hi.xyz, b); interior b == 0 with children at a and a+1, leaves
//              b == primitive count and a == first slot.
//   leaf_data  primitives in BVH leaf order, packed for the intersection loop
//              (sphere: 1 float4 (x,y,z,r); cylinder: (A,r),(B,-); polyhedron: (p,-),(quat);
//              mesh: (p, face bits),(quat)).
//   order      leaf slot -> primitive index of the user's arrays.
//   position/radius/color/... the user's arrays (read only when shading a hit).
// A scene is an array of GeomDev records; every ray traverses the BVH of each enabled
// geometry in turn, carrying its closest t so far (the reference puts all geometries in one
// Embree/OptiX acceleration structure; the closest hit is the same).
#ifndef FR_ENGINE_CUH
#define FR_ENGINE_CUH

#include <cstdint>

#include "bvh.hpp"
#include "fresnel_b200.h"
#include "frmath.cuh"

namespace fr {

constexpr int TRAVERSAL_STACK = 64;
constexpr uint32_t MISS = 0xFFFFFFFFu;
constexpr uint32_t EMPTY_CHILD = 0xFFFFFFFFu;  // count of an unused 4-wide child slot

// error bits reported through the device status word
constexpr uint32_t ERR_STACK_OVERFLOW = 1u;
constexpr uint32_t ERR_ITERATION_CAP = 2u;
constexpr uint32_t ERR_BAD_NODE = 4u;    // a BVH index out of range (never followed)
constexpr uint32_t ERR_BUILD = 8u;       // BVH construction found an inconsistent hierarchy
constexpr uint32_t ERR_KERNEL = 16u;     // a kernel met an acceleration structure it lacks

struct GeomDev {
    int32_t type;
    int32_t enabled;
    uint32_t n_prims;  // BVH primitives (mesh: instances * faces)
    uint32_t n_nodes;
    uint32_t n_nodes4;
    const float4* nodes;
    const float4* nodes4;
    const float4* leaf_data;
    const uint32_t* order;
    const float* position;
    const float* radius;
    const float* color;
    const float* points;
    const float* orientation;
    const float* vertices;
    const float* planes;  // [n_planes][9]: origin, unit normal, colour
    uint32_t n_faces;
    uint32_t n_planes;
    uint32_t n_vertices;    // polygon: vertices [n_vertices][2]
    float rounding_radius;  // polygon
    float bound_radius;     // polyhedron, polygon: bounding radius about the position; mesh: the
                            // largest vertex distance from the instance origin
    const float4* face_box;  // mesh: per face its padded box in the instance frame (lo, hi)
    float color_by_face;
    float outline_width;
    Mat material;
    Mat outline;
};

// Uniform grid of a scene (n_cells == 0: the scene has none), over the spheres of its one
// geometry or over the primitives of its parts (parts = 1).  Cell (ix, iy, iz) spans
// lo + (i, i + 1) * h per axis and is numbered (iz * ny + iy) * nx + ix; its references are
// [cell_start[c], cell_start[c + 1]): for spheres a copy of the sphere (x, y, z, r) and its index,
// for parts a leaf-slot record (SceneDev::leaf_data, leaf_geom, order).  A primitive is referenced
// by every cell its padded bounding box touches (a mesh by instance: the box of the instance).
struct GridDev {
    uint32_t n_cells;
    uint32_t nx, ny, nz;
    float lox, loy, loz;
    float hix, hiy, hiz;  // far corner (lo + n * h)
    float hx, hy, hz;     // cell size
    float ihx, ihy, ihz;  // 1 / cell size
    uint32_t geom;        // scene index of the sphere geometry
    const uint32_t* cell_start;
    const float4* ref_sphere;
    const uint32_t* ref_prim;
    // 1: a grid over the primitives of several geometries (or one non-sphere geometry); its
    // references are records laid out as a combined tree's leaf slots (SceneDev::leaf_data,
    // leaf_geom, order), and ref_sphere / ref_prim / geom are unused
    uint32_t parts;
};

struct SceneDev {
    const GeomDev* geoms;
    uint32_t n_geoms;
    uint32_t* status;  // error bits (device)
    GridDev grid;      // scenes traced through a uniform grid instead of a BVH
    // Combined 4-wide tree over the primitives of several geometries (n_nodes4 == 0: none, each
    // enabled geometry's own tree is traversed in turn): leaf slot s holds 2 float4 of its
    // primitive's record, its geometry (leaf_geom) and its index within the geometry (order).
    uint32_t n_nodes4;
    uint32_t n_prims;
    const float4* nodes4;
    const float4* leaf_data;
    const uint32_t* leaf_geom;
    const uint32_t* order;
};

// --------------------------------------------------------------------------------------------
// loads
// --------------------------------------------------------------------------------------------
__device__ __forceinline__ float4 ldg4(const float4* p) { return __ldg(p); }

__device__ __forceinline__ V3 load3(const float* a, uint32_t i)
{
    return v3(__ldg(a + 3 * i), __ldg(a + 3 * i + 1), __ldg(a + 3 * i + 2));
}

__device__ __forceinline__ C3 loadc3(const float* a, uint32_t i)
{
    return c3(__ldg(a + 3 * i), __ldg(a + 3 * i + 1), __ldg(a + 3 * i + 2));
}

__device__ __forceinline__ Qt loadq(const float* a, uint32_t i)
{
    return Qt{__ldg(a + 4 * i), v3(__ldg(a + 4 * i + 1), __ldg(a + 4 * i + 2), __ldg(a + 4 * i + 3))};
}

// --------------------------------------------------------------------------------------------
// ray/box slab test with precomputed reciprocal direction (boxes are inflated at build time,
// so the single rounding of each fused multiply-add cannot cull a primitive that the exact
// intersector accepts)
// --------------------------------------------------------------------------------------------
struct RayK {
    V3 o, d;
    V3 inv, oinv;  // 1/d and -o/d
};

__device__ __forceinline__ RayK make_rayk(V3 o, V3 d)
{
    RayK r;
    r.o = o;
    r.d = d;
    auto safe_inv = [](float x) {
        float ax = fabsf(x);
        return 1.0f / (ax < 1e-30f ? copysignf(1e-30f, x) : x);
    };
    r.inv = v3(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
    r.oinv = v3(-o.x * r.inv.x, -o.y * r.inv.y, -o.z * r.inv.z);
    return r;
}

__device__ __forceinline__ bool slab(const RayK& r, float4 lo, float4 hi, float tmax, float& tentry)
{
    float tx0 = fmaf(lo.x, r.inv.x, r.oinv.x), tx1 = fmaf(hi.x, r.inv.x, r.oinv.x);
    float ty0 = fmaf(lo.y, r.inv.y, r.oinv.y), ty1 = fmaf(hi.y, r.inv.y, r.oinv.y);
    float tz0 = fmaf(lo.z, r.inv.z, r.oinv.z), tz1 = fmaf(hi.z, r.inv.z, r.oinv.z);
    float t0 = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), 0.0f));
    float t1 = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), tmax));
    tentry = t0;
    return t0 <= t1;
}

// --------------------------------------------------------------------------------------------
// per-type leaf tests: update (tmax, hit) when a primitive is accepted with tnear < t < tmax
// (the acceptance rule of fresnel/cpu/Geometry*.cc).  Only t is computed here; the shading
// quantities are recomputed for the one closest hit (hit_surface below).
// --------------------------------------------------------------------------------------------
struct PolyHit {
    bool hit;
    float t;
    int plane;
    V3 n, p;  // local-frame normal and origin of the hit plane
    V3 ol, dl;
};

// Exact ties.  A primitive hit at exactly the distance of the closest hit so far (coincident
// surfaces: duplicated primitives, shared end caps, rounding-level crossings) wins when its
// (geometry, primitive) index is the lower one, so that the closest hit does not depend on the
// order in which a structure (either BVH builder, the sphere grid, the oracle's tree) offers
// the candidates; fresnel's CPU path keeps whichever its Embree traversal offered first.  A ray
// without a hit yet never ties.  `cand_prim` is read only when the geometries are equal.
template <class CandPrim, class BestPrim>
__device__ __forceinline__ bool tie_wins(uint32_t cand_geom, uint32_t best_geom,
                                         const CandPrim& cand_prim, const BestPrim& best_prim)
{
    return best_geom != MISS &&
           (cand_geom < best_geom || (cand_geom == best_geom && cand_prim() < best_prim()));
}

struct NoTie {
    __device__ __forceinline__ bool operator()() const { return false; }
};

// slab test over the face planes (fresnel/cpu/GeometryConvexPolyhedron.cc:146-224); the entry
// (else the exit) distance is accepted when it lies in (tnear, tfar), or equals tfar and
// `tie()` says the primitive wins the tie.
template <class Tie = NoTie>
__device__ __forceinline__ PolyHit poly_planes(const GeomDev& g, V3 o, V3 d, V3 pos, Qt q,
                                               float tnear, float tfar, const Tie& tie = Tie())
{
    PolyHit r;
    r.hit = false;
    r.t = 0.0f;
    r.plane = 0;
    r.n = v3(0, 0, 1);
    r.p = v3(0, 0, 0);
    float t0 = -3.402823466e+38f, t1 = 3.402823466e+38f;
    V3 dl = rotate(conj(q), d);
    V3 ol = rotate(conj(q), o - pos);
    r.ol = ol;
    r.dl = dl;
    V3 t0n = v3(0, 0, 0), t0p = v3(0, 0, 0), t1n = v3(0, 0, 0), t1p = v3(0, 0, 0);
    int t0_plane = 0, t1_plane = 0;
    for (uint32_t i = 0; i < g.n_planes && t0 < t1; ++i) {
        const float* pl = g.planes + 9 * i;
        V3 p = v3(__ldg(pl), __ldg(pl + 1), __ldg(pl + 2));
        V3 n = v3(__ldg(pl + 3), __ldg(pl + 4), __ldg(pl + 5));
        float dd = -dot(n, p);
        float denom = dot(n, dl);
        float t = -(dd + dot(n, ol)) / denom;
        if (double(fabsf(denom)) < 1e-5) {
            if (dot(ol - p, n) > 0)
                return r;
        } else if (denom < 0) {
            if (t > t0) {
                t0 = t;
                t0n = n;
                t0p = p;
                t0_plane = int(i);
            }
        } else {
            if (t < t1) {
                t1 = t;
                t1n = n;
                t1p = p;
                t1_plane = int(i);
            }
        }
    }
    if (t0 > t1)
        return r;
    if ((tnear < t0) & ((t0 < tfar) || (t0 == tfar && tie()))) {
        r.hit = true;
        r.t = tfar = t0;
        r.n = t0n;
        r.p = t0p;
        r.plane = t0_plane;
        return r;  // the exit (t1 >= t0) cannot be closer
    }
    if ((tnear < t1) & ((t1 < tfar) || (t1 == tfar && tie()))) {
        r.hit = true;
        r.t = tfar = t1;
        r.n = t1n;
        r.p = t1p;
        r.plane = t1_plane;
    }
    return r;
}

// double-sided instanced triangle (fresnel/cpu/GeometryMesh.cc:115-166)
struct TriHit {
    bool hit;
    float u, v, w, t, d;
    V3 n;
};

__device__ __forceinline__ TriHit mesh_triangle(const GeomDev& g, uint32_t face, V3 o, V3 d, V3 pos,
                                                Qt q)
{
    TriHit r;
    V3 dl = rotate(conj(q), d);
    V3 ol = rotate(conj(q), o - pos);
    V3 v0 = load3(g.vertices, 3 * face), v1 = load3(g.vertices, 3 * face + 1),
       v2 = load3(g.vertices, 3 * face + 2);
    r.u = r.v = r.w = r.t = r.d = 0.0f;
    r.n = v3(0, 0, 0);
    V3 q2 = ol + dl;
    r.hit = isect_triangle(r.u, r.v, r.w, r.t, r.d, r.n, ol, q2, v0, v1, v2)
            || isect_triangle(r.v, r.u, r.w, r.t, r.d, r.n, ol, q2, v1, v0, v2);
    return r;
}

// Rounded polygon in the z = 0 plane (fresnel/cpu/GeometryPolygon.cc:146-230): the ray, taken
// into the polygon's frame, meets the plane at t; the hit point counts if its signed distance to
// the outline (negative inside, by the crossing-number test of :113-140 and the point-segment
// distance of fresnel/common/GeometryMath.h:28-39) is at most the rounding radius.  d is the
// outline distance (rounding radius minus the signed distance), n the plane normal facing the
// ray (double sided), both in the polygon's frame.
struct PgHit {
    bool hit;
    float t, d;
    V3 n;
};

__device__ __forceinline__ float pg_min(float a, float b) { return (b < a) ? b : a; }  // std::min
__device__ __forceinline__ float pg_max(float a, float b) { return (a < b) ? b : a; }  // std::max

__device__ __forceinline__ PgHit polygon_hit(const GeomDev& g, V3 o, V3 d, float px, float py,
                                             Qt q)
{
    PgHit r;
    r.hit = false;
    r.t = r.d = 0.0f;
    r.n = v3(0, 0, 1);
    const V3 dl = rotate(conj(q), d);
    const V3 ol = rotate(conj(q), o - v3(px, py, 0.0f));
    const V3 n = v3(0, 0, 1);
    const V3 p = v3(0, 0, 0);
    const float dd = -dot(n, p);
    const float denom = dot(n, dl);
    const float t = -(dd + dot(n, ol)) / denom;
    if (double(fabsf(denom)) < 1e-5)
        return r;
    const V3 rh = ol + t * dl;
    // crossing number and the distance to the nearest edge
    const float2* vt = reinterpret_cast<const float2*>(g.vertices);
    const uint32_t nv = g.n_vertices;
    float min_d = 3.402823466e+38f;
    bool odd = false;
    float2 vj = nv ? __ldg(vt + (nv - 1u)) : make_float2(0.0f, 0.0f);
    for (uint32_t i = 0; i < nv; ++i) {
        const float2 vi = __ldg(vt + i);
        const float abx = vj.x - vi.x, aby = vj.y - vi.y;
        const float L = abx * abx + aby * aby;
        const float s = pg_max(0.0f, pg_min(1.0f, ((rh.x - vi.x) * abx + (rh.y - vi.y) * aby) / L));
        const float wx = rh.x - (vi.x + s * abx), wy = rh.y - (vi.y + s * aby);
        min_d = pg_min(min_d, sqrtf(wx * wx + wy * wy));
        if ((vi.y < rh.y && vj.y >= rh.y) || (vj.y < rh.y && vi.y >= rh.y)) {
            if (vi.x + (rh.y - vi.y) / (vj.y - vi.y) * (vj.x - vi.x) < rh.x)
                odd = !odd;
        }
        vj = vi;
    }
    const float d_edge = odd ? -min_d : min_d;
    if (d_edge > g.rounding_radius)
        return r;
    r.d = g.rounding_radius - d_edge;
    r.t = t;
    r.n = (dot(n, dl) < 0.0f) ? n : -n;
    r.hit = true;
    return r;
}

// box and primitive tests of one thread (summed into the tracer's counters per warp)
struct TraceCount {
    uint32_t box = 0;
    uint32_t prim = 0;
};

template <int TYPE>
__device__ __forceinline__ void leaf_test(const GeomDev& g, uint32_t gi, const RayK& ray,
                                          uint32_t first, uint32_t count, float tnear,
                                          float& tmax, uint32_t& hit_geom, uint32_t& hit_slot,
                                          TraceCount& tc)
{
    tc.prim += count;
    for (uint32_t s = first; s < first + count; ++s) {
        // exact tie with the closest hit so far: the lower (geometry, primitive) index wins
        const auto tie = [&]() {
            return tie_wins(
                gi, hit_geom, [&]() { return __ldg(g.order + s); },
                [&]() { return __ldg(g.order + hit_slot); });
        };
        float t = 0.0f;
        bool ok;
        if (TYPE == FR_GEOM_SPHERE) {
            float4 q = ldg4(g.leaf_data + s);
            ok = sphere_t(ray.o, ray.d, v3(q.x, q.y, q.z), q.w, t);
        } else if (TYPE == FR_GEOM_CYLINDER) {
            float4 a = ldg4(g.leaf_data + 2 * s), b = ldg4(g.leaf_data + 2 * s + 1);
            float de;
            V3 N;
            uint32_t ci;
            ok = isect_spherocylinder(t, de, N, ci, ray.o, ray.d, v3(a.x, a.y, a.z),
                                      v3(b.x, b.y, b.z), a.w);
        } else if (TYPE == FR_GEOM_POLYHEDRON) {
            float4 a = ldg4(g.leaf_data + 2 * s), b = ldg4(g.leaf_data + 2 * s + 1);
            PolyHit ph = poly_planes(g, ray.o, ray.d, v3(a.x, a.y, a.z), Qt{b.x, v3(b.y, b.z, b.w)},
                                     tnear, tmax, tie);
            ok = ph.hit;
            t = ph.t;
        } else if (TYPE == FR_GEOM_MESH) {
            float4 a = ldg4(g.leaf_data + 2 * s), b = ldg4(g.leaf_data + 2 * s + 1);
            TriHit th = mesh_triangle(g, __float_as_uint(a.w), ray.o, ray.d, v3(a.x, a.y, a.z),
                                      Qt{b.x, v3(b.y, b.z, b.w)});
            ok = th.hit;
            t = th.t;
        } else {
            float4 a = ldg4(g.leaf_data + 2 * s), b = ldg4(g.leaf_data + 2 * s + 1);
            PgHit ph = polygon_hit(g, ray.o, ray.d, a.x, a.y, Qt{b.x, v3(b.y, b.z, b.w)});
            ok = ph.hit;
            t = ph.t;
        }
        if (ok && (tnear < t) && ((t < tmax) || (t == tmax && tie()))) {
            tmax = t;
            hit_geom = gi;
            hit_slot = s;
        }
    }
}

// Closest hit in one geometry's BVH (stack-light: a 64-entry per-thread stack of child pairs
// with their entry distances, near child first, leaves tested as soon as their box is hit).
template <int TYPE>
__device__ __forceinline__ void traverse(const GeomDev& g, uint32_t gi, const RayK& ray, float tnear,
                                         float& tmax, uint32_t& hit_geom, uint32_t& hit_slot,
                                         uint32_t* status, TraceCount& tc)
{
    if (g.n_nodes == 0)
        return;
    float te;
    tc.box += 1;
    float4 rlo = ldg4(g.nodes), rhi = ldg4(g.nodes + 1);
    if (!slab(ray, rlo, rhi, tmax, te))
        return;
    uint32_t rb = __float_as_uint(rhi.w);
    if (rb != 0) {
        uint32_t first = __float_as_uint(rlo.w);
        if (first > g.n_prims || rb > g.n_prims - first) {
            atomicOr(status, ERR_BAD_NODE);
            return;
        }
        leaf_test<TYPE>(g, gi, ray, first, rb, tnear, tmax, hit_geom, hit_slot, tc);
        return;
    }
    uint32_t stack_node[TRAVERSAL_STACK];
    float stack_t[TRAVERSAL_STACK];
    int sp = 0;
    uint32_t cur = __float_as_uint(rlo.w);
    uint32_t guard = 2u * g.n_nodes + 8u;
    while (true) {
        if (--guard == 0u) {
            atomicOr(status, ERR_ITERATION_CAP);
            return;
        }
        if (cur + 1u >= g.n_nodes) {  // the child pair must lie inside the node array
            atomicOr(status, ERR_BAD_NODE);
            return;
        }
        const float4* np = g.nodes + 2 * size_t(cur);
        float4 alo = ldg4(np), ahi = ldg4(np + 1), blo = ldg4(np + 2), bhi = ldg4(np + 3);
        float ta, tb;
        tc.box += 2;
        bool ha = slab(ray, alo, ahi, tmax, ta);
        bool hb = slab(ray, blo, bhi, tmax, tb);
        uint32_t ca = __float_as_uint(ahi.w), cb = __float_as_uint(bhi.w);
        if ((ca != 0 && (__float_as_uint(alo.w) > g.n_prims ||
                         ca > g.n_prims - __float_as_uint(alo.w))) ||
            (cb != 0 && (__float_as_uint(blo.w) > g.n_prims ||
                         cb > g.n_prims - __float_as_uint(blo.w)))) {
            atomicOr(status, ERR_BAD_NODE);
            return;
        }
        if (ha && ca != 0) {
            leaf_test<TYPE>(g, gi, ray, __float_as_uint(alo.w), ca, tnear, tmax, hit_geom, hit_slot,
                            tc);
            ha = false;
        }
        if (hb && cb != 0) {
            if (tb <= tmax)
                leaf_test<TYPE>(g, gi, ray, __float_as_uint(blo.w), cb, tnear, tmax, hit_geom,
                                hit_slot, tc);
            hb = false;
        }
        if (ha && hb) {
            uint32_t near_n = __float_as_uint(alo.w), far_n = __float_as_uint(blo.w);
            float far_t = tb;
            if (tb < ta) {
                near_n = __float_as_uint(blo.w);
                far_n = __float_as_uint(alo.w);
                far_t = ta;
            }
            if (sp < TRAVERSAL_STACK) {
                stack_node[sp] = far_n;
                stack_t[sp] = far_t;
                ++sp;
            } else {
                atomicOr(status, ERR_STACK_OVERFLOW);
            }
            cur = near_n;
            continue;
        }
        if (ha) {
            cur = __float_as_uint(alo.w);
            continue;
        }
        if (hb) {
            cur = __float_as_uint(blo.w);
            continue;
        }
        bool found = false;
        while (sp > 0) {
            --sp;
            if (stack_t[sp] <= tmax) {
                cur = stack_node[sp];
                found = true;
                break;
            }
        }
        if (!found)
            return;
    }
}

__device__ __forceinline__ uint32_t pick4(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t k)
{
    return k == 0 ? a : (k == 1 ? b : (k == 2 ? c : d));
}

__device__ __forceinline__ void cswap(uint32_t& a, uint32_t& b)
{
    uint32_t lo = min(a, b), hi = max(a, b);
    a = lo;
    b = hi;
}

// Closest hit in one geometry's 4-wide BVH: per step one 128-byte node and four slab tests;
// hit leaves are tested at once; hit interior children are ordered by entry distance with a
// five-comparator sorting network on keys (distance bits | child slot), the nearest is visited
// next and the others are pushed far to near on a 64-entry per-thread stack.  Everything stays
// in registers (no dynamically indexed arrays besides the stack).
// Node float4 holding each axis's near planes for this ray (the far planes are the other one of
// the pair): a 4-wide node stores lo.x, hi.x, lo.y, hi.y, lo.z, hi.z, and a ray whose direction
// component is negative enters through the hi plane.
struct NearFar {
    int x, y, z;
};

__device__ __forceinline__ NearFar near_far(const RayK& r)
{
    return NearFar{r.inv.x < 0.0f ? 1 : 0, r.inv.y < 0.0f ? 3 : 2, r.inv.z < 0.0f ? 5 : 4};
}

// Slab test of one child against its near (n) and far (f) planes: the same entry and exit
// distances as min/max over the lo/hi planes for every non-empty box (a fused multiply-add is
// monotonic in the plane), with half the min/max operations.  Empty boxes (lo > hi) are missed.
__device__ __forceinline__ bool slab4_child(const RayK& ray, float nx, float fx, float ny, float fy,
                                            float nz, float fz, float tmax, float& te)
{
    const float tnx = fmaf(nx, ray.inv.x, ray.oinv.x), tfx = fmaf(fx, ray.inv.x, ray.oinv.x);
    const float tny = fmaf(ny, ray.inv.y, ray.oinv.y), tfy = fmaf(fy, ray.inv.y, ray.oinv.y);
    const float tnz = fmaf(nz, ray.inv.z, ray.oinv.z), tfz = fmaf(fz, ray.inv.z, ray.oinv.z);
    const float t0 = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, 0.0f));
    const float t1 = fminf(fminf(tfx, tfy), fminf(tfz, tmax));
    te = t0;
    return t0 <= t1;
}

// One visit of a 4-wide node: test its four children, test the leaves the ray hits (through
// `leaf(first, count)`, which lowers tmax on a closer hit), descend into the nearest interior
// child hit and push the others far to near, or pop the next stacked node still in reach.
// Returns false once nothing is left to visit (or a bad index was met and reported).
template <class Leaf>
__device__ __forceinline__ bool visit4(const float4* nodes4, uint32_t n_nodes4, uint32_t n_prims,
                                       const RayK& ray, const NearFar& nf, float& tmax,
                                       uint32_t& cur, int& sp, uint32_t* stack_node,
                                       float* stack_t, uint32_t* status, TraceCount& tc,
                                       Leaf&& leaf)
{
    const float4* np = nodes4 + 8 * size_t(cur);
    const float4 nx = ldg4(np + nf.x), fx = ldg4(np + (nf.x ^ 1)), ny = ldg4(np + nf.y),
                 fy = ldg4(np + (nf.y ^ 1)), nz = ldg4(np + nf.z), fz = ldg4(np + (nf.z ^ 1));
    const uint4 ci = __ldg(reinterpret_cast<const uint4*>(np + 6));
    const uint4 cc = __ldg(reinterpret_cast<const uint4*>(np + 7));
    tc.box += 4;
    float te0, te1, te2, te3;
    auto test = [&](float nxk, float fxk, float nyk, float fyk, float nzk, float fzk,
                    uint32_t cck, float& te) {
        return slab4_child(ray, nxk, fxk, nyk, fyk, nzk, fzk, tmax, te) && cck != EMPTY_CHILD;
    };
    const bool h0 = test(nx.x, fx.x, ny.x, fy.x, nz.x, fz.x, cc.x, te0);
    const bool h1 = test(nx.y, fx.y, ny.y, fy.y, nz.y, fz.y, cc.y, te1);
    const bool h2 = test(nx.z, fx.z, ny.z, fy.z, nz.z, fz.z, cc.z, te2);
    const bool h3 = test(nx.w, fx.w, ny.w, fy.w, nz.w, fz.w, cc.w, te3);
    // leaves: one shared copy of the primitive loop, iterated over a bit mask
    uint32_t leaves = (h0 && cc.x != 0u ? 1u : 0u) | (h1 && cc.y != 0u ? 2u : 0u) |
                      (h2 && cc.z != 0u ? 4u : 0u) | (h3 && cc.w != 0u ? 8u : 0u);
    while (leaves) {
        const uint32_t k = uint32_t(__ffs(leaves) - 1);
        leaves &= leaves - 1u;
        const uint32_t first = pick4(ci.x, ci.y, ci.z, ci.w, k);
        const uint32_t count = pick4(cc.x, cc.y, cc.z, cc.w, k);
        if (first > n_prims || count > n_prims - first) {
            atomicOr(status, ERR_BAD_NODE);
            return false;
        }
        leaf(first, count);
    }
    // interior children: key = entry distance bits (non-negative float) | child slot
    auto key = [&](bool h, uint32_t cck, float te, uint32_t k) {
        return (h && cck == 0u && te <= tmax) ? ((__float_as_uint(te) & ~3u) | k) : 0xFFFFFFFFu;
    };
    uint32_t k0 = key(h0, cc.x, te0, 0), k1 = key(h1, cc.y, te1, 1);
    uint32_t k2 = key(h2, cc.z, te2, 2), k3 = key(h3, cc.w, te3, 3);
    cswap(k0, k1);
    cswap(k2, k3);
    cswap(k0, k2);
    cswap(k1, k3);
    cswap(k1, k2);
    if (k0 != 0xFFFFFFFFu) {
        // push the farther ones (far to near), descend into the nearest
        const uint32_t ks[3] = {k3, k2, k1};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (ks[a] != 0xFFFFFFFFu) {
                const uint32_t node = pick4(ci.x, ci.y, ci.z, ci.w, ks[a] & 3u);
                if (sp < TRAVERSAL_STACK) {
                    stack_node[sp] = node;
                    stack_t[sp] = __uint_as_float(ks[a] & ~3u);
                    ++sp;
                } else {
                    atomicOr(status, ERR_STACK_OVERFLOW);
                }
            }
        }
        cur = pick4(ci.x, ci.y, ci.z, ci.w, k0 & 3u);
        if (cur >= n_nodes4) {
            atomicOr(status, ERR_BAD_NODE);
            return false;
        }
        return true;
    }
    while (sp > 0) {
        --sp;
        if (stack_t[sp] <= tmax) {
            cur = stack_node[sp];
            return cur < n_nodes4;
        }
    }
    return false;
}

template <class Leaf>
__device__ __forceinline__ void traverse4_core(const float4* nodes4, uint32_t n_nodes4,
                                               uint32_t n_prims, const RayK& ray, float& tmax,
                                               uint32_t* status, TraceCount& tc, Leaf&& leaf)
{
    if (n_nodes4 == 0)
        return;
    uint32_t stack_node[TRAVERSAL_STACK];
    float stack_t[TRAVERSAL_STACK];
    int sp = 0;
    uint32_t cur = 0;
    uint32_t guard = n_nodes4 + 8u;
    const NearFar nf = near_far(ray);
    while (true) {
        if (--guard == 0u) {
            atomicOr(status, ERR_ITERATION_CAP);
            return;
        }
        if (!visit4(nodes4, n_nodes4, n_prims, ray, nf, tmax, cur, sp, stack_node, stack_t,
                    status, tc, leaf))
            return;
    }
}

// Warp-cooperative form of traverse4_core for coherent rays (neighbouring samples of the same
// pixels): the warp walks one node sequence; each lane tests its own ray against a node's four
// children and its own leaves; the warp descends into every interior child that some lane hits,
// nearest first by the smallest entry distance over the lanes, and drops a stacked subtree once
// its entry distance is beyond every lane's closest hit.  Each lane therefore tests exactly the
// leaves its own ray reaches with its own closest distance, as in traverse4_core, and gets the
// same closest hit (the visiting order only matters between primitives at exactly equal t).
// The stack is the warp's own (shared memory, TRAVERSAL_STACK entries).  All 32 lanes must call
// together; lanes without a ray pass active = false.
template <class Leaf>
__device__ __forceinline__ void traverse4_packet_core(const float4* nodes4, uint32_t n_nodes4,
                                                      uint32_t n_prims, const RayK& ray,
                                                      bool active, float& tmax, uint32_t* status,
                                                      TraceCount& tc, uint32_t* stk_node,
                                                      float* stk_t, Leaf&& leaf)
{
    constexpr uint32_t FULL = 0xffffffffu, NONE = 0xFFFFFFFFu;
    if (n_nodes4 == 0)
        return;
    const bool lead = (threadIdx.x & 31u) == 0u;
    int sp = 0;
    uint32_t cur = 0;
    uint32_t guard = n_nodes4 + 8u;
    const NearFar nf = near_far(ray);
    while (true) {
        if (--guard == 0u) {
            if (lead)
                atomicOr(status, ERR_ITERATION_CAP);
            return;
        }
        const float4* np = nodes4 + 8 * size_t(cur);
        const float4 nx = ldg4(np + nf.x), fx = ldg4(np + (nf.x ^ 1)), ny = ldg4(np + nf.y),
                     fy = ldg4(np + (nf.y ^ 1)), nz = ldg4(np + nf.z), fz = ldg4(np + (nf.z ^ 1));
        const uint4 ci = __ldg(reinterpret_cast<const uint4*>(np + 6));
        const uint4 cc = __ldg(reinterpret_cast<const uint4*>(np + 7));
        if (active)
            tc.box += 4;
        float te0, te1, te2, te3;
        auto test = [&](float nxk, float fxk, float nyk, float fyk, float nzk, float fzk,
                        uint32_t cck, float& te) {
            return active && slab4_child(ray, nxk, fxk, nyk, fyk, nzk, fzk, tmax, te) &&
                   cck != EMPTY_CHILD;
        };
        const bool h0 = test(nx.x, fx.x, ny.x, fy.x, nz.x, fz.x, cc.x, te0);
        const bool h1 = test(nx.y, fx.y, ny.y, fy.y, nz.y, fz.y, cc.y, te1);
        const bool h2 = test(nx.z, fx.z, ny.z, fy.z, nz.z, fz.z, cc.z, te2);
        const bool h3 = test(nx.w, fx.w, ny.w, fy.w, nz.w, fz.w, cc.w, te3);
        // leaves: the warp goes through every leaf some lane hits; each lane tests its own
        const uint32_t leaves = (h0 && cc.x != 0u ? 1u : 0u) | (h1 && cc.y != 0u ? 2u : 0u) |
                                (h2 && cc.z != 0u ? 4u : 0u) | (h3 && cc.w != 0u ? 8u : 0u);
        uint32_t any_leaves = __reduce_or_sync(FULL, leaves);
        while (any_leaves) {
            const uint32_t k = uint32_t(__ffs(any_leaves) - 1);
            any_leaves &= any_leaves - 1u;
            const uint32_t first = pick4(ci.x, ci.y, ci.z, ci.w, k);
            const uint32_t count = pick4(cc.x, cc.y, cc.z, cc.w, k);
            if (first > n_prims || count > n_prims - first) {
                if (lead)
                    atomicOr(status, ERR_BAD_NODE);
                return;
            }
            if (leaves & (1u << k))
                leaf(first, count);
        }
        // interior children, keyed by the nearest entry over the lanes that reach them
        auto key = [&](bool h, uint32_t cck, float te, uint32_t k) {
            const uint32_t own = (h && cck == 0u && te <= tmax) ? __float_as_uint(te) : NONE;
            const uint32_t m = __reduce_min_sync(FULL, own);
            return m == NONE ? NONE : ((m & ~3u) | k);
        };
        uint32_t k0 = key(h0, cc.x, te0, 0), k1 = key(h1, cc.y, te1, 1);
        uint32_t k2 = key(h2, cc.z, te2, 2), k3 = key(h3, cc.w, te3, 3);
        cswap(k0, k1);
        cswap(k2, k3);
        cswap(k0, k2);
        cswap(k1, k3);
        cswap(k1, k2);
        if (k0 != NONE) {
            const uint32_t ks[3] = {k3, k2, k1};
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                if (ks[a] != NONE) {
                    if (sp < TRAVERSAL_STACK) {
                        if (lead) {
                            stk_node[sp] = pick4(ci.x, ci.y, ci.z, ci.w, ks[a] & 3u);
                            stk_t[sp] = __uint_as_float(ks[a] & ~3u);
                        }
                        ++sp;
                    } else if (lead) {
                        atomicOr(status, ERR_STACK_OVERFLOW);
                    }
                }
            }
            __syncwarp();
            cur = pick4(ci.x, ci.y, ci.z, ci.w, k0 & 3u);
            if (cur >= n_nodes4) {
                if (lead)
                    atomicOr(status, ERR_BAD_NODE);
                return;
            }
            continue;
        }
        // the farthest any lane still needs to look (closest hits are non-negative)
        const float reach =
            __uint_as_float(__reduce_max_sync(FULL, active ? __float_as_uint(tmax) : 0u));
        bool found = false;
        while (sp > 0) {
            --sp;
            if (stk_t[sp] <= reach) {
                cur = stk_node[sp];
                found = cur < n_nodes4;
                break;
            }
        }
        __syncwarp();
        if (!found)
            return;
    }
}

template <int TYPE>
__device__ __forceinline__ void traverse4(const GeomDev& g, uint32_t gi, const RayK& ray,
                                          float tnear, float& tmax, uint32_t& hit_geom,
                                          uint32_t& hit_slot, uint32_t* status, TraceCount& tc)
{
    traverse4_core(g.nodes4, g.n_nodes4, g.n_prims, ray, tmax, status, tc,
                   [&](uint32_t first, uint32_t count) {
                       leaf_test<TYPE>(g, gi, ray, first, count, tnear, tmax, hit_geom, hit_slot,
                                       tc);
                   });
}

// Test of leaf slot s of a combined tree (or reference s of a grid over parts) of geometry g,
// its record's first float4 in a: whether the ray meets the primitive, and where (t).  tmax and
// tie serve the polyhedron slab test's acceptance of an exit at exactly tmax.
template <uint32_t MASK, class Tie>
__device__ __forceinline__ bool mixed_prim_t(const SceneDev& sc, const GeomDev& g, int type,
                                             float4 a, uint32_t s, const RayK& ray, float tnear,
                                             float tmax, const Tie& tie, float& t)
{
    t = 0.0f;
    if ((MASK & (1u << FR_GEOM_SPHERE)) && type == FR_GEOM_SPHERE)
        return sphere_t(ray.o, ray.d, v3(a.x, a.y, a.z), a.w, t);
    if ((MASK & (1u << FR_GEOM_CYLINDER)) && type == FR_GEOM_CYLINDER) {
        const float4 b = ldg4(sc.leaf_data + 2 * size_t(s) + 1);
        float de;
        V3 N;
        uint32_t ci;
        return isect_spherocylinder(t, de, N, ci, ray.o, ray.d, v3(a.x, a.y, a.z),
                                    v3(b.x, b.y, b.z), a.w);
    }
    if ((MASK & (1u << FR_GEOM_POLYHEDRON)) && type == FR_GEOM_POLYHEDRON) {
        const float4 b = ldg4(sc.leaf_data + 2 * size_t(s) + 1);
        PolyHit ph = poly_planes(g, ray.o, ray.d, v3(a.x, a.y, a.z), Qt{b.x, v3(b.y, b.z, b.w)},
                                 tnear, tmax, tie);
        t = ph.t;
        return ph.hit;
    }
    if ((MASK & (1u << FR_GEOM_MESH)) && type == FR_GEOM_MESH) {
        const float4 b = ldg4(sc.leaf_data + 2 * size_t(s) + 1);
        TriHit th = mesh_triangle(g, __float_as_uint(a.w), ray.o, ray.d, v3(a.x, a.y, a.z),
                                  Qt{b.x, v3(b.y, b.z, b.w)});
        t = th.t;
        return th.hit;
    }
    if ((MASK & (1u << FR_GEOM_POLYGON)) && type == FR_GEOM_POLYGON) {
        const float4 b = ldg4(sc.leaf_data + 2 * size_t(s) + 1);
        PgHit ph = polygon_hit(g, ray.o, ray.d, a.x, a.y, Qt{b.x, v3(b.y, b.z, b.w)});
        t = ph.t;
        return ph.hit;
    }
    return false;
}

// Leaf of a combined tree: each slot names its geometry; the primitive test is that geometry
// type's (only the types in MASK are compiled in).
template <uint32_t MASK>
__device__ __forceinline__ void leaf_test_mixed(const SceneDev& sc, const RayK& ray,
                                                uint32_t first, uint32_t count, float tnear,
                                                float& tmax, uint32_t& hit_geom,
                                                uint32_t& hit_slot, TraceCount& tc)
{
    tc.prim += count;
    for (uint32_t s = first; s < first + count; ++s) {
        const uint32_t gi = __ldg(sc.leaf_geom + s);
        if (gi >= sc.n_geoms)
            continue;
        const GeomDev& g = sc.geoms[gi];
        const float4 a = ldg4(sc.leaf_data + 2 * size_t(s));
        // exact tie with the closest hit so far: the lower (geometry, primitive) index wins
        const auto tie = [&]() {
            return tie_wins(
                gi, hit_geom, [&]() { return __ldg(sc.order + s); },
                [&]() { return __ldg(sc.order + hit_slot); });
        };
        float t;
        const bool ok = mixed_prim_t<MASK>(sc, g, g.type, a, s, ray, tnear, tmax, tie, t);
        if (ok && (tnear < t) && ((t < tmax) || (t == tmax && tie()))) {
            tmax = t;
            hit_geom = gi;
            hit_slot = s;
        }
    }
}

// The references of one cell of a grid over parts: the test and acceptance rule of every type
// (mixed_prim_t, as the combined tree's leaves), with hit_prim (the primitive's index within its
// geometry) kept instead of a leaf slot.  A cylinder, polyhedron or polygon is tested only when
// the ray segment (0, tmax) enters its bounding box (the cylinder's, or the box about the
// position of the bounding radius; padded beyond the tree builds' padding) as a tree's box test
// would allow.  A mesh is referenced by instance: once the ray meets the instance's bounding
// sphere (the mesh's largest vertex distance times the squared norm of the quaternion, as
// rotate() scales, with a margin), the ray is taken into the instance frame once, exactly as
// mesh_triangle takes it for each triangle, and each face whose padded local box the segment
// enters gets mesh_triangle's two-sided test, face by face (primitive = instance * faces + face).
// No primitive or instance is tested again right after itself (last_geom, last_prim: one
// spanning several cells along the ray; its test and the acceptance are exact, so a repeat
// could not change the hit).
template <uint32_t MASK>
__device__ __forceinline__ void parts_cell_test(const SceneDev& sc, const RayK& ray,
                                                uint32_t first, uint32_t last, float tnear,
                                                float& tmax, uint32_t& hit_geom,
                                                uint32_t& hit_prim, uint32_t& last_geom,
                                                uint32_t& last_prim, TraceCount& tc)
{
    tc.prim += last - first;
    for (uint32_t s = first; s < last; ++s) {
        // geometry index and type in one word (gather_parts): a sphere needs nothing from the
        // geometry table
        const uint32_t gw = __ldg(sc.leaf_geom + s);
        const uint32_t gi = gw & ((1u << PART_TYPE_SHIFT) - 1u);
        if (gi >= sc.n_geoms)
            continue;
        const GeomDev& g = sc.geoms[gi];
        const int type = int(gw >> PART_TYPE_SHIFT);
        const float4 a = ldg4(sc.leaf_data + 2 * size_t(s));
        if ((MASK & (1u << FR_GEOM_MESH)) && type == FR_GEOM_MESH) {
            // the instance's bounding sphere (the distance of its centre from the ray's line
            // from a cross product, which keeps its precision far from the ray's origin)
            const float4 b = ldg4(sc.leaf_data + 2 * size_t(s) + 1);
            const float r = g.bound_radius * (b.x * b.x + b.y * b.y + b.z * b.z + b.w * b.w);
            const V3 pos = v3(a.x, a.y, a.z);
            const V3 oc = pos - ray.o;
            const float scale = fmaxf(fmaxf(fabsf(oc.x), fabsf(oc.y)), fabsf(oc.z)) + r;
            const float rp = r + 1e-4f * scale + 1e-5f;
            const float dd = dot(ray.d, ray.d), bb = dot(oc, ray.d);
            const V3 cr = cross(oc, ray.d);
            if (!(dot(cr, cr) <= rp * rp * dd))
                continue;  // the line misses the sphere
            const float reach = rp * sqrtf(dd);
            if (bb + reach < 0.0f || bb - reach > tmax * dd)
                continue;  // the sphere lies behind the origin or beyond the closest hit
            const uint32_t inst = __ldg(sc.order + s);
            if (gi == last_geom && inst == last_prim)
                continue;
            last_geom = gi;
            last_prim = inst;
            const Qt q = Qt{b.x, v3(b.y, b.z, b.w)};
            const V3 dl = rotate(conj(q), ray.d);
            const V3 ol = rotate(conj(q), ray.o - pos);
            const V3 q2 = ol + dl;
            const RayK lr = make_rayk(ol, dl);  // t along it is t along the ray
            const float lpad = 1e-4f * (fmaxf(fmaxf(fabsf(ol.x), fabsf(ol.y)), fabsf(ol.z)) +
                                        g.bound_radius) + 1e-5f;
            for (uint32_t f = 0; f < g.n_faces; ++f) {
                float4 lo = ldg4(g.face_box + 2 * size_t(f)), hi = ldg4(g.face_box + 2 * size_t(f) + 1);
                lo = make_float4(lo.x - lpad, lo.y - lpad, lo.z - lpad, 0.0f);
                hi = make_float4(hi.x + lpad, hi.y + lpad, hi.z + lpad, 0.0f);
                float tentry;
                if (!slab(lr, lo, hi, tmax, tentry))
                    continue;
                const V3 v0 = load3(g.vertices, 3 * f), v1 = load3(g.vertices, 3 * f + 1),
                         v2 = load3(g.vertices, 3 * f + 2);
                float u, v, w, t, de;
                V3 n;
                const bool hit = isect_triangle(u, v, w, t, de, n, ol, q2, v0, v1, v2) ||
                                 isect_triangle(v, u, w, t, de, n, ol, q2, v1, v0, v2);
                const uint32_t prim = inst * g.n_faces + f;
                if (hit && (tnear < t) &&
                    ((t < tmax) || (t == tmax && tie_wins(
                                                     gi, hit_geom, [&]() { return prim; },
                                                     [&]() { return hit_prim; })))) {
                    tmax = t;
                    hit_geom = gi;
                    hit_prim = prim;
                }
            }
            continue;
        }
        if (type != FR_GEOM_SPHERE) {
            float4 lo, hi;
            if (type == FR_GEOM_CYLINDER) {
                const float4 b = ldg4(sc.leaf_data + 2 * size_t(s) + 1);
                lo = make_float4(fminf(a.x, b.x) - a.w, fminf(a.y, b.y) - a.w,
                                 fminf(a.z, b.z) - a.w, 0.0f);
                hi = make_float4(fmaxf(a.x, b.x) + a.w, fmaxf(a.y, b.y) + a.w,
                                 fmaxf(a.z, b.z) + a.w, 0.0f);
            } else {
                const float r = g.bound_radius;
                const float rz = type == FR_GEOM_POLYGON ? 0.0f : r;
                lo = make_float4(a.x - r, a.y - r, a.z - rz, 0.0f);
                hi = make_float4(a.x + r, a.y + r, a.z + rz, 0.0f);
            }
            const float scale = fmaxf(fmaxf(fmaxf(fabsf(lo.x), fabsf(hi.x)),
                                            fmaxf(fabsf(lo.y), fabsf(hi.y))),
                                      fmaxf(fabsf(lo.z), fabsf(hi.z)));
            const float pad = 1e-4f * scale + 1e-5f;
            lo = make_float4(lo.x - pad, lo.y - pad, lo.z - pad, 0.0f);
            hi = make_float4(hi.x + pad, hi.y + pad, hi.z + pad, 0.0f);
            float tentry;
            if (!slab(ray, lo, hi, tmax, tentry))
                continue;
            const uint32_t prim = __ldg(sc.order + s);
            if (gi == last_geom && prim == last_prim)
                continue;
            last_geom = gi;
            last_prim = prim;
        }
        const auto tie = [&]() {
            return tie_wins(
                gi, hit_geom, [&]() { return __ldg(sc.order + s); }, [&]() { return hit_prim; });
        };
        float t;
        const bool ok = mixed_prim_t<MASK>(sc, g, type, a, s, ray, tnear, tmax, tie, t);
        if (ok && (tnear < t) && ((t < tmax) || (t == tmax && tie()))) {
            tmax = t;
            hit_geom = gi;
            hit_prim = __ldg(sc.order + s);
        }
    }
}

struct Hit {
    uint32_t geom;  // MISS if none
    uint32_t prim;  // index into the geometry's user arrays
};

// Closest sphere hit through a uniform grid: a 3-D DDA walk over the cells the ray crosses
// (Amanatides & Woo, "A fast voxel traversal algorithm for ray tracing", Eurographics 1987),
// testing every sphere a cell references with the same sphere test and acceptance rule as the
// BVH leaves.  The walk stops once the closest hit so far lies before the exit from the current
// cell: a sphere the ray meets earlier touches a cell already walked (boxes are padded well
// beyond the rounding of the cell boundaries), so it has been tested.  Cell exits are
// recomputed from the plane positions at every step, so rounding does not accumulate.  The next
// cell's reference range is loaded before this cell's spheres are tested, and spheres are
// loaded two at a time, to shorten the chain of dependent loads (extension pass 5% faster).
//
// The walk is split into grid_walk_begin (entry cell) and grid_walk_step (one cell), so that a
// kernel can interleave the cells of different rays in one lane (per-lane refill).
struct GridWalk {
    int ix, iy, iz;         // current cell
    float tnx, tny, tnz;    // distances to the planes the ray leaves it through, per axis
    float t_out;            // distance at which the ray leaves the grid
    uint32_t first, last;   // the current cell's reference range
    uint32_t guard;         // cells left before the walk is cut (a bound, never reached)
};

__device__ __forceinline__ float grid_exit_t(int i, float inv, float lo, float h, float oinv)
{
    return fmaf(fmaf(float(i + (inv >= 0.0f ? 1 : 0)), h, lo), inv, oinv);
}

__device__ __forceinline__ uint32_t grid_cell_id(const GridDev& G, int x, int y, int z)
{
    return (uint32_t(z) * G.ny + uint32_t(y)) * G.nx + uint32_t(x);
}

// Sets up the walk of `ray`; false when the ray misses the grid (nothing to walk).
__device__ __forceinline__ bool grid_walk_begin(const GridDev& G, const RayK& ray, GridWalk& W)
{
    float tx0 = fmaf(G.lox, ray.inv.x, ray.oinv.x), tx1 = fmaf(G.hix, ray.inv.x, ray.oinv.x);
    float ty0 = fmaf(G.loy, ray.inv.y, ray.oinv.y), ty1 = fmaf(G.hiy, ray.inv.y, ray.oinv.y);
    float tz0 = fmaf(G.loz, ray.inv.z, ray.oinv.z), tz1 = fmaf(G.hiz, ray.inv.z, ray.oinv.z);
    const float t_in = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), 0.0f));
    W.t_out = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fmaxf(tz0, tz1));
    if (!(t_in <= W.t_out))
        return false;  // misses the grid (or NaN)
    // the cell holding the entry point (clamped: the entry lies on the grid's surface)
    auto cell_of = [](float p, float lo, float ih, uint32_t n) {
        const float u = (p - lo) * ih;
        return u >= 0.0f ? int(fminf(u, float(n - 1u))) : 0;  // NaN compares false: cell 0
    };
    W.ix = cell_of(ray.o.x + t_in * ray.d.x, G.lox, G.ihx, G.nx);
    W.iy = cell_of(ray.o.y + t_in * ray.d.y, G.loy, G.ihy, G.ny);
    W.iz = cell_of(ray.o.z + t_in * ray.d.z, G.loz, G.ihz, G.nz);
    W.tnx = grid_exit_t(W.ix, ray.inv.x, G.lox, G.hx, ray.oinv.x);
    W.tny = grid_exit_t(W.iy, ray.inv.y, G.loy, G.hy, ray.oinv.y);
    W.tnz = grid_exit_t(W.iz, ray.inv.z, G.loz, G.hz, ray.oinv.z);
    W.guard = G.nx + G.ny + G.nz + 3u;
    const uint32_t c = grid_cell_id(G, W.ix, W.iy, W.iz);
    W.first = __ldg(G.cell_start + c);
    W.last = __ldg(G.cell_start + c + 1);
    return true;
}

// Tests the primitives of the walk's current cell (test(first, last) over its reference range)
// and moves to the next cell; false when the walk is over (the closest hit so far, tmax, lies
// before the cell's exit, or the ray leaves the grid).
template <class CellTest>
__device__ __forceinline__ bool grid_walk_visit(const GridDev& G, const RayK& ray,
                                                const float& tmax, GridWalk& W, TraceCount& tc,
                                                const CellTest& test)
{
    // the next cell along the ray, and its reference range loaded now so that the load
    // overlaps the primitive tests of this cell
    const int sx = ray.inv.x >= 0.0f ? 1 : -1;
    const int sy = ray.inv.y >= 0.0f ? 1 : -1;
    const int sz = ray.inv.z >= 0.0f ? 1 : -1;
    const float t_cell = fminf(W.tnx, fminf(W.tny, W.tnz));
    const int axis = (W.tnx <= W.tny && W.tnx <= W.tnz) ? 0 : (W.tny <= W.tnz ? 1 : 2);
    const int nx = W.ix + (axis == 0 ? sx : 0), ny = W.iy + (axis == 1 ? sy : 0),
              nz = W.iz + (axis == 2 ? sz : 0);
    const bool more = t_cell < W.t_out && nx >= 0 && nx < int(G.nx) && ny >= 0 &&
                      ny < int(G.ny) && nz >= 0 && nz < int(G.nz);
    uint32_t next_first = 0, next_last = 0;
    if (more) {
        const uint32_t nc = grid_cell_id(G, nx, ny, nz);
        next_first = __ldg(G.cell_start + nc);
        next_last = __ldg(G.cell_start + nc + 1);
    }
    tc.box += 1;
    test(W.first, W.last);
    if (tmax <= t_cell || !more || --W.guard == 0u)
        return false;
    W.ix = nx;
    W.iy = ny;
    W.iz = nz;
    if (axis == 0)
        W.tnx = grid_exit_t(W.ix, ray.inv.x, G.lox, G.hx, ray.oinv.x);
    else if (axis == 1)
        W.tny = grid_exit_t(W.iy, ray.inv.y, G.loy, G.hy, ray.oinv.y);
    else
        W.tnz = grid_exit_t(W.iz, ray.inv.z, G.loz, G.hz, ray.oinv.z);
    W.first = next_first;
    W.last = next_last;
    return true;
}

// One cell of a sphere grid's walk (grid_walk_visit with the sphere tests); slot receives the
// reference index of a closer hit.
__device__ __forceinline__ bool grid_walk_step(const GridDev& G, const RayK& ray, float tnear,
                                               float& tmax, uint32_t& slot, GridWalk& W,
                                               TraceCount& tc)
{
    return grid_walk_visit(G, ray, tmax, W, tc, [&](uint32_t first, uint32_t last) {
        tc.prim += last - first;
        // exact tie with the closest hit so far: the lower sphere index wins (one geometry)
        const auto tie = [&](uint32_t r) {
            return slot != MISS && __ldg(G.ref_prim + r) < __ldg(G.ref_prim + slot);
        };
        uint32_t k = first;
        for (; k + 1 < last; k += 2) {  // two spheres in flight
            const float4 q0 = ldg4(G.ref_sphere + k), q1 = ldg4(G.ref_sphere + k + 1);
            float t0, t1;
            if (sphere_t(ray.o, ray.d, v3(q0.x, q0.y, q0.z), q0.w, t0) && (tnear < t0) &&
                ((t0 < tmax) || (t0 == tmax && tie(k)))) {
                tmax = t0;
                slot = k;
            }
            if (sphere_t(ray.o, ray.d, v3(q1.x, q1.y, q1.z), q1.w, t1) && (tnear < t1) &&
                ((t1 < tmax) || (t1 == tmax && tie(k + 1)))) {
                tmax = t1;
                slot = k + 1;
            }
        }
        if (k < last) {
            const float4 q = ldg4(G.ref_sphere + k);
            float t;
            if (sphere_t(ray.o, ray.d, v3(q.x, q.y, q.z), q.w, t) && (tnear < t) &&
                ((t < tmax) || (t == tmax && tie(k)))) {
                tmax = t;
                slot = k;
            }
        }
    });
}

// The whole walk of one ray.
__device__ __forceinline__ void trace_grid(const GridDev& G, const RayK& ray, float tnear,
                                           float& tmax, uint32_t& slot, TraceCount& tc)
{
    GridWalk W;
    if (!grid_walk_begin(G, ray, W))
        return;
    while (grid_walk_step(G, ray, tnear, tmax, slot, W, tc)) {
    }
}

__device__ __forceinline__ Hit trace_grid_hit(const GridDev& G, const RayK& ray, float tnear,
                                              float tmax, TraceCount& tc)
{
    uint32_t slot = MISS;
    trace_grid(G, ray, tnear, tmax, slot, tc);
    Hit h;
    h.geom = slot == MISS ? MISS : G.geom;
    h.prim = slot == MISS ? 0u : __ldg(G.ref_prim + slot);
    return h;
}

// Closest hit through a grid over the primitives of several geometries (GridDev::parts): the
// same walk, with each cell's references tested as the leaf slots of a combined tree (the test
// and acceptance rule of every geometry type, ties to the lower (geometry, primitive) index) by
// parts_cell_test.
template <uint32_t TYPES>
__device__ __forceinline__ Hit trace_grid_parts(const SceneDev& sc, const RayK& ray, float tnear,
                                                float tmax, TraceCount& tc)
{
    const GridDev& G = sc.grid;
    uint32_t hg = MISS, hp = 0, last_g = MISS, last_p = 0;
    GridWalk W;
    if (grid_walk_begin(G, ray, W)) {
        while (grid_walk_visit(G, ray, tmax, W, tc, [&](uint32_t first, uint32_t last) {
            parts_cell_test<TYPES>(sc, ray, first, last, tnear, tmax, hg, hp, last_g, last_p, tc);
        })) {
        }
    }
    Hit h;
    h.geom = hg;
    h.prim = hg == MISS ? 0u : hp;
    return h;
}

// Geometry-type masks a kernel is specialised for (bit FR_GEOM_* set = type handled).
constexpr uint32_t MASK_SPHERES = 1u << FR_GEOM_SPHERE;
constexpr uint32_t MASK_ALL = 0x1Fu;  // every FR_GEOM_* type
// Kernels specialised for a scene of spheres traced through its uniform grid (SceneDev::grid),
// with no BVH code compiled in.
constexpr uint32_t MASK_GRID = 1u << 31;
// Kernels specialised for a scene traced through a grid over its parts (GridDev::parts = 1),
// every geometry type compiled in, no BVH code.
constexpr uint32_t MASK_GRID_PARTS = MASK_GRID | MASK_ALL;
// The same without the mesh code (scenes of parts none of which is a mesh: fewer registers).
constexpr uint32_t MASK_GRID_PARTS_NO_MESH = MASK_GRID | (MASK_ALL & ~(1u << FR_GEOM_MESH));
// Added to a tree kernel's mask: it may also meet grids over parts (the kernels of batches whose
// renders trace different kinds of structure).  The single-render tree kernels go without: the
// grid-over-parts walk would raise their register count (k_path_extend: 80 -> 98, one block per
// SM less), and those renders run the MASK_GRID_PARTS kernels.
constexpr uint32_t MASK_MAY_PARTS = 1u << 29;

// Blocks of 256 threads per SM the fused trace-and-shade kernels are compiled for.  The grid walk
// fits 64 registers with few spills, and the fourth block hides its memory latency better (1080p
// frame of 1M spheres: 82.8 against 85.3 ms; spheres and bonds over parts, 2M primitives: 4.87
// against 5.42 ms); the BVH traversals spill heavily at 64 and keep 3, and so do the grid-over-
// parts kernels with the mesh code (mixed scene: 69.9 against 70.5 ms at 4, 79.7 at 2).
__host__ __device__ constexpr int fused_blocks(uint32_t mask)
{
    return (mask == MASK_GRID || mask == MASK_GRID_PARTS_NO_MESH) ? 4 : 3;
}

// Closest hit through the scene's BVHs: its combined tree, or each enabled geometry's tree.
template <int WIDTH, uint32_t MASK>
__device__ __forceinline__ Hit trace_closest_bvh(const SceneDev& sc, const RayK& ray, float tnear,
                                                 TraceCount& tc)
{
    float tmax = __int_as_float(0x7f800000);  // +inf
    uint32_t hg = MISS, hs = 0;
    if (WIDTH == 4 && sc.n_nodes4 != 0) {
        traverse4_core(sc.nodes4, sc.n_nodes4, sc.n_prims, ray, tmax, sc.status, tc,
                       [&](uint32_t first, uint32_t count) {
                           leaf_test_mixed<MASK>(sc, ray, first, count, tnear, tmax, hg, hs, tc);
                       });
        Hit h;
        h.geom = hg;
        h.prim = (hg == MISS) ? 0u : __ldg(sc.order + hs);
        return h;
    }
    for (uint32_t gi = 0; gi < sc.n_geoms; ++gi) {
        const GeomDev& g = sc.geoms[gi];
        if (!g.enabled)
            continue;
#define FR_TRAVERSE(T)                                                            \
    if ((MASK & (1u << T)) && g.type == T) {                                      \
        if (WIDTH == 4)                                                           \
            traverse4<T>(g, gi, ray, tnear, tmax, hg, hs, sc.status, tc);        \
        else                                                                      \
            traverse<T>(g, gi, ray, tnear, tmax, hg, hs, sc.status, tc);         \
        continue;                                                                 \
    }
        FR_TRAVERSE(FR_GEOM_SPHERE)
        FR_TRAVERSE(FR_GEOM_CYLINDER)
        FR_TRAVERSE(FR_GEOM_POLYHEDRON)
        FR_TRAVERSE(FR_GEOM_MESH)
        FR_TRAVERSE(FR_GEOM_POLYGON)
#undef FR_TRAVERSE
    }
    Hit h;
    h.geom = hg;
    h.prim = (hg == MISS) ? 0u : __ldg(sc.geoms[hg].order + hs);
    return h;
}

// Closest hit over all enabled geometries of the scene.  WIDTH selects the binary (2) or
// 4-wide (4) tree; MASK the geometry types compiled in (the host only launches a MASK that
// covers every enabled geometry of the scene), MASK_GRID for the sphere grid alone, or
// MASK_GRID_PARTS for a grid over the scene's parts.
template <int WIDTH, uint32_t MASK>
__device__ __forceinline__ Hit trace_closest(const SceneDev& sc, V3 o, V3 d, float tnear,
                                             TraceCount& tc)
{
    const RayK ray = make_rayk(o, d);
    const float tmax = __int_as_float(0x7f800000);  // +inf
    if constexpr (MASK == MASK_GRID) {
        return trace_grid_hit(sc.grid, ray, tnear, tmax, tc);
    } else if constexpr ((MASK & MASK_GRID) != 0u) {
        return trace_grid_parts<MASK & MASK_ALL>(sc, ray, tnear, tmax, tc);
    } else {
        // kernels for BVH scenes also serve sphere grids (a batch may mix both), and grids over
        // parts when MASK has MASK_MAY_PARTS
        if (sc.grid.n_cells != 0) {
            if (sc.grid.parts) {
                if constexpr ((MASK & MASK_MAY_PARTS) != 0u) {
                    return trace_grid_parts<MASK & MASK_ALL>(sc, ray, tnear, tmax, tc);
                } else {
                    atomicOr(sc.status, ERR_KERNEL);  // not launched so: reported, no hit
                    Hit h;
                    h.geom = MISS;
                    h.prim = 0;
                    return h;
                }
            }
            if (MASK & MASK_SPHERES)
                return trace_grid_hit(sc.grid, ray, tnear, tmax, tc);
        }
        return trace_closest_bvh<WIDTH, MASK & MASK_ALL>(sc, ray, tnear, tc);
    }
}

// Closest hit for coherent rays with the warp-cooperative traversal (4-wide trees only).  All
// 32 lanes of the warp call together; `active` marks the lanes that have a ray.
template <uint32_t MASK>
__device__ __forceinline__ Hit trace_closest_packet(const SceneDev& sc, V3 o, V3 d, bool active,
                                                    float tnear, TraceCount& tc,
                                                    uint32_t* stk_node, float* stk_t)
{
    RayK ray = make_rayk(o, d);
    float tmax = __int_as_float(0x7f800000);  // +inf
    uint32_t hg = MISS, hs = 0;
    if (sc.n_nodes4 != 0) {
        traverse4_packet_core(sc.nodes4, sc.n_nodes4, sc.n_prims, ray, active, tmax, sc.status,
                              tc, stk_node, stk_t, [&](uint32_t first, uint32_t count) {
                                  leaf_test_mixed<MASK>(sc, ray, first, count, tnear, tmax, hg,
                                                        hs, tc);
                              });
        Hit h;
        h.geom = hg;
        h.prim = (hg == MISS) ? 0u : __ldg(sc.order + hs);
        return h;
    }
    for (uint32_t gi = 0; gi < sc.n_geoms; ++gi) {
        const GeomDev& g = sc.geoms[gi];
        if (!g.enabled)
            continue;
#define FR_TRAVERSE(T)                                                                     \
    if ((MASK & (1u << T)) && g.type == T) {                                               \
        traverse4_packet_core(g.nodes4, g.n_nodes4, g.n_prims, ray, active, tmax, sc.status, \
                              tc, stk_node, stk_t, [&](uint32_t first, uint32_t count) {   \
                                  leaf_test<T>(g, gi, ray, first, count, tnear, tmax, hg, hs, \
                                               tc);                                        \
                              });                                                          \
        continue;                                                                          \
    }
        FR_TRAVERSE(FR_GEOM_SPHERE)
        FR_TRAVERSE(FR_GEOM_CYLINDER)
        FR_TRAVERSE(FR_GEOM_POLYHEDRON)
        FR_TRAVERSE(FR_GEOM_MESH)
        FR_TRAVERSE(FR_GEOM_POLYGON)
#undef FR_TRAVERSE
    }
    Hit h;
    h.geom = hg;
    h.prim = (hg == MISS) ? 0u : __ldg(sc.geoms[hg].order + hs);
    return h;
}

// --------------------------------------------------------------------------------------------
// Step-wise 4-wide traversal for persistent warps (Aila & Laine, "Understanding the efficiency
// of ray traversal on GPUs", HPG 2009): each call visits one node of the current geometry's
// tree; a lane whose ray is finished fetches a new one, so lanes stay busy although rays need
// very different numbers of steps.
// --------------------------------------------------------------------------------------------
constexpr uint32_t NEED_GEOM = 0xFFFFFFFFu;  // cur: start the next geometry's tree

struct LaneRay {
    RayK ray;
    float tnear, tmax;
    uint32_t hit_geom, hit_slot;
    uint32_t gi;   // geometry being traversed
    uint32_t cur;  // node to visit, or NEED_GEOM
    int sp;
    uint32_t guard;
};

__device__ __forceinline__ void lane_begin(LaneRay& L, V3 o, V3 d, float tnear)
{
    L.ray = make_rayk(o, d);
    L.tnear = tnear;
    L.tmax = __int_as_float(0x7f800000);
    L.hit_geom = MISS;
    L.hit_slot = 0;
    L.gi = 0;
    L.cur = NEED_GEOM;
    L.sp = 0;
    L.guard = 0;
}

template <uint32_t MASK>
__device__ __forceinline__ void leaf_dispatch(const GeomDev& g, LaneRay& L, uint32_t first,
                                              uint32_t count, TraceCount& tc)
{
    if ((MASK & MASK_SPHERES) && (MASK == MASK_SPHERES || g.type == FR_GEOM_SPHERE))
        leaf_test<FR_GEOM_SPHERE>(g, L.gi, L.ray, first, count, L.tnear, L.tmax, L.hit_geom,
                                  L.hit_slot, tc);
    else if ((MASK & (1u << FR_GEOM_CYLINDER)) && g.type == FR_GEOM_CYLINDER)
        leaf_test<FR_GEOM_CYLINDER>(g, L.gi, L.ray, first, count, L.tnear, L.tmax, L.hit_geom,
                                    L.hit_slot, tc);
    else if ((MASK & (1u << FR_GEOM_POLYHEDRON)) && g.type == FR_GEOM_POLYHEDRON)
        leaf_test<FR_GEOM_POLYHEDRON>(g, L.gi, L.ray, first, count, L.tnear, L.tmax, L.hit_geom,
                                      L.hit_slot, tc);
    else if ((MASK & (1u << FR_GEOM_MESH)) && g.type == FR_GEOM_MESH)
        leaf_test<FR_GEOM_MESH>(g, L.gi, L.ray, first, count, L.tnear, L.tmax, L.hit_geom,
                                L.hit_slot, tc);
    else if ((MASK & (1u << FR_GEOM_POLYGON)) && g.type == FR_GEOM_POLYGON)
        leaf_test<FR_GEOM_POLYGON>(g, L.gi, L.ray, first, count, L.tnear, L.tmax, L.hit_geom,
                                   L.hit_slot, tc);
}

// One step of the lane's traversal; returns false once the ray is finished (every enabled
// geometry's tree traversed).  Indices are checked before use; a bad one ends the ray and sets
// an error bit.
template <uint32_t MASK>
__device__ __forceinline__ bool step4(const SceneDev& sc, LaneRay& L, uint32_t* stack_node,
                                      float* stack_t, TraceCount& tc)
{
    if (L.cur == NEED_GEOM) {
        while (L.gi < sc.n_geoms) {
            const GeomDev& gg = sc.geoms[L.gi];
            if (gg.enabled && gg.n_nodes4 && (MASK & (1u << gg.type)))
                break;
            ++L.gi;
        }
        if (L.gi >= sc.n_geoms)
            return false;
        L.cur = 0;
        L.sp = 0;
        L.guard = sc.geoms[L.gi].n_nodes4 + 8u;
    }
    const GeomDev& g = sc.geoms[L.gi];
    if (L.guard-- == 0u || L.cur >= g.n_nodes4) {
        atomicOr(sc.status, L.cur >= g.n_nodes4 ? ERR_BAD_NODE : ERR_ITERATION_CAP);
        return false;
    }
    const float4* np = g.nodes4 + 8 * size_t(L.cur);
    const float4 lx = ldg4(np), hx = ldg4(np + 1), ly = ldg4(np + 2), hy = ldg4(np + 3),
                 lz = ldg4(np + 4), hz = ldg4(np + 5);
    const uint4 ci = __ldg(reinterpret_cast<const uint4*>(np + 6));
    const uint4 cc = __ldg(reinterpret_cast<const uint4*>(np + 7));
    tc.box += 4;
    const RayK& ray = L.ray;
    const float tmax0 = L.tmax;
    auto test = [&](float lxk, float hxk, float lyk, float hyk, float lzk, float hzk,
                    uint32_t cck, float& te) {
        float tx0 = fmaf(lxk, ray.inv.x, ray.oinv.x), tx1 = fmaf(hxk, ray.inv.x, ray.oinv.x);
        float ty0 = fmaf(lyk, ray.inv.y, ray.oinv.y), ty1 = fmaf(hyk, ray.inv.y, ray.oinv.y);
        float tz0 = fmaf(lzk, ray.inv.z, ray.oinv.z), tz1 = fmaf(hzk, ray.inv.z, ray.oinv.z);
        float t0 = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), 0.0f));
        float t1 = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), tmax0));
        te = t0;
        return t0 <= t1 && cck != EMPTY_CHILD;
    };
    float te0, te1, te2, te3;
    bool h0 = test(lx.x, hx.x, ly.x, hy.x, lz.x, hz.x, cc.x, te0);
    bool h1 = test(lx.y, hx.y, ly.y, hy.y, lz.y, hz.y, cc.y, te1);
    bool h2 = test(lx.z, hx.z, ly.z, hy.z, lz.z, hz.z, cc.z, te2);
    bool h3 = test(lx.w, hx.w, ly.w, hy.w, lz.w, hz.w, cc.w, te3);
    uint32_t leaves = (h0 && cc.x != 0u ? 1u : 0u) | (h1 && cc.y != 0u ? 2u : 0u) |
                      (h2 && cc.z != 0u ? 4u : 0u) | (h3 && cc.w != 0u ? 8u : 0u);
    while (leaves) {
        uint32_t k = uint32_t(__ffs(leaves) - 1);
        leaves &= leaves - 1u;
        uint32_t first = pick4(ci.x, ci.y, ci.z, ci.w, k);
        uint32_t count = pick4(cc.x, cc.y, cc.z, cc.w, k);
        if (first > g.n_prims || count > g.n_prims - first) {
            atomicOr(sc.status, ERR_BAD_NODE);
            return false;
        }
        leaf_dispatch<MASK>(g, L, first, count, tc);
    }
    const float tmax = L.tmax;
    auto key = [&](bool h, uint32_t cck, float te, uint32_t k) {
        return (h && cck == 0u && te <= tmax) ? ((__float_as_uint(te) & ~3u) | k) : 0xFFFFFFFFu;
    };
    uint32_t k0 = key(h0, cc.x, te0, 0), k1 = key(h1, cc.y, te1, 1);
    uint32_t k2 = key(h2, cc.z, te2, 2), k3 = key(h3, cc.w, te3, 3);
    cswap(k0, k1);
    cswap(k2, k3);
    cswap(k0, k2);
    cswap(k1, k3);
    cswap(k1, k2);
    if (k0 != 0xFFFFFFFFu) {
        uint32_t ks[3] = {k3, k2, k1};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (ks[a] != 0xFFFFFFFFu) {
                if (L.sp < TRAVERSAL_STACK) {
                    stack_node[L.sp] = pick4(ci.x, ci.y, ci.z, ci.w, ks[a] & 3u);
                    stack_t[L.sp] = __uint_as_float(ks[a] & ~3u);
                    ++L.sp;
                } else {
                    atomicOr(sc.status, ERR_STACK_OVERFLOW);
                }
            }
        }
        L.cur = pick4(ci.x, ci.y, ci.z, ci.w, k0 & 3u);
        return true;
    }
    while (L.sp > 0) {
        --L.sp;
        if (stack_t[L.sp] <= tmax) {
            L.cur = stack_node[L.sp];
            return true;
        }
    }
    // this geometry's tree is done: continue with the next geometry
    ++L.gi;
    L.cur = NEED_GEOM;
    return true;
}

// Lane index within the warp (independent of the block's shape).
__device__ __forceinline__ uint32_t lane_id()
{
    uint32_t l;
    asm volatile("mov.u32 %0, %%laneid;" : "=r"(l));
    return l;
}

// Add the warp's traversal counts to counters[0] (box tests) and counters[1] (primitive tests).
__device__ __forceinline__ void flush_counts(const TraceCount& tc, unsigned long long* counters)
{
    unsigned long long b = tc.box, p = tc.prim;
    for (int off = 16; off > 0; off >>= 1) {
        b += __shfl_xor_sync(0xffffffffu, b, off);
        p += __shfl_xor_sync(0xffffffffu, p, off);
    }
    if (lane_id() == 0u && (b | p)) {
        atomicAdd(counters, b);
        atomicAdd(counters + 1, p);
    }
}

// --------------------------------------------------------------------------------------------
// shading quantities of the closest hit (what the reference's intersect callbacks leave in
// RTCHit::Ng, FresnelRTCIntersectContext::shading_color and ::d)
// --------------------------------------------------------------------------------------------
struct Surface {
    float t;
    V3 Ng;
    C3 color;
    float d_edge;
};

__device__ __forceinline__ Surface hit_surface(const GeomDev& g, uint32_t prim, V3 o, V3 d,
                                               float tnear)
{
    Surface s;
    s.t = 0.0f;
    s.Ng = v3(0, 0, 1);
    s.color = c3(0, 0, 0);
    s.d_edge = 0.0f;
    switch (g.type) {
    case FR_GEOM_SPHERE: {  // fresnel/cpu/GeometrySphere.cc:81-118
        V3 p = load3(g.position, prim);
        float r = __ldg(g.radius + prim);
        V3 N;
        isect_sphere(s.t, s.d_edge, N, o, d, p, r);
        s.Ng = v3(o.x + s.t * d.x - p.x, o.y + s.t * d.y - p.y, o.z + s.t * d.z - p.z);
        s.color = loadc3(g.color, prim);
        break;
    }
    case FR_GEOM_CYLINDER: {  // fresnel/cpu/GeometryCylinder.cc:76-120
        V3 A = load3(g.points, 2 * prim), B = load3(g.points, 2 * prim + 1);
        float r = __ldg(g.radius + prim);
        uint32_t ci = 0;
        float t = HUGE_VALF, de = HUGE_VALF;
        V3 N = v3(0, 0, 0);
        isect_spherocylinder(t, de, N, ci, o, d, A, B, r);
        s.t = t;
        s.d_edge = de;
        s.Ng = N;
        s.color = loadc3(g.color, 2 * prim + ci);
        break;
    }
    case FR_GEOM_POLYHEDRON: {  // fresnel/cpu/GeometryConvexPolyhedron.cc:226-335
        V3 pos = load3(g.position, prim);
        Qt q = loadq(g.orientation, prim);
        PolyHit ph = poly_planes(g, o, d, pos, q, tnear, __int_as_float(0x7f800000));
        s.t = ph.t;
        s.Ng = rotate(q, ph.n);
        const float* pl = g.planes + 9 * ph.plane;
        s.color = lerp(g.color_by_face, loadc3(g.color, prim),
                       c3(__ldg(pl + 6), __ldg(pl + 7), __ldg(pl + 8)));
        float min_d = 3.402823466e+38f;
        V3 r_hit = ph.ol + ph.t * ph.dl;
        for (uint32_t i = 0; i < g.n_planes; ++i) {
            const float* pi = g.planes + 9 * i;
            V3 p = v3(__ldg(pi), __ldg(pi + 1), __ldg(pi + 2));
            V3 n = v3(__ldg(pi + 3), __ldg(pi + 4), __ldg(pi + 5));
            V3 u = cross(n, ph.n);
            if (double(fabsf(dot(u, u))) >= 1e-5) {
                int maxc;
                if (fabsf(u.x) > fabsf(u.y))
                    maxc = (fabsf(u.x) > fabsf(u.z)) ? 1 : 3;
                else
                    maxc = (fabsf(u.y) > fabsf(u.z)) ? 2 : 3;
                V3 x0 = v3(0, 0, 0);
                float d1 = -dot(n, p);
                float d2 = -dot(ph.n, ph.p);
                if (maxc == 1) {
                    x0.y = (d2 * n.z - d1 * ph.n.z) / u.x;
                    x0.z = (d1 * ph.n.y - d2 * n.y) / u.x;
                } else if (maxc == 2) {
                    x0.x = (d1 * ph.n.z - d2 * n.z) / u.y;
                    x0.z = (d2 * n.x - d1 * ph.n.x) / u.y;
                } else {
                    x0.x = (d2 * n.y - d1 * ph.n.y) / u.z;
                    x0.y = (d1 * ph.n.x - d2 * n.x) / u.z;
                }
                V3 view = div_recip(-ph.dl, sqrtf(dot(ph.dl, ph.dl)));
                u = u - dot(u, view) * view;
                V3 w = x0 - r_hit;
                V3 w_perp = w - dot(w, view) * view;
                x0 = r_hit + w_perp;
                V3 vv = cross(u, x0 - r_hit);
                float dist = sqrtf(dot(vv, vv) / dot(u, u));
                if (dist < min_d)
                    min_d = dist;
            }
        }
        s.d_edge = min_d;
        break;
    }
    case FR_GEOM_POLYGON: {  // fresnel/cpu/GeometryPolygon.cc:146-230
        Qt q = loadq(g.orientation, prim);
        PgHit ph = polygon_hit(g, o, d, __ldg(g.position + 2 * size_t(prim)),
                               __ldg(g.position + 2 * size_t(prim) + 1), q);
        s.t = ph.t;
        s.d_edge = ph.d;
        s.Ng = rotate(q, ph.n);
        s.color = loadc3(g.color, prim);
        break;
    }
    default: {  // mesh, fresnel/cpu/GeometryMesh.cc:115-193
        uint32_t inst = prim / g.n_faces, face = prim - inst * g.n_faces;
        V3 pos = load3(g.position, inst);
        Qt q = loadq(g.orientation, inst);
        TriHit th = mesh_triangle(g, face, o, d, pos, q);
        s.t = th.t;
        s.d_edge = th.d;
        s.Ng = rotate(q, th.n);
        s.color = loadc3(g.color, 3 * face + 0) * th.u + loadc3(g.color, 3 * face + 1) * th.v
                  + loadc3(g.color, 3 * face + 2) * th.w;
        break;
    }
    }
    return s;
}

}  // namespace fr

#endif
