// oracle_core.cpp -- TEST INFRASTRUCTURE (CPU oracle), not part of the product.
//
// A CPU restatement of fresnel's Embree backend: per-geometry closest-hit glue restated from
// fresnel/cpu/Geometry{Sphere,Cylinder,ConvexPolyhedron,Mesh,Polygon}.cc, the tile loops of
// fresnel/cpu/TracerPath.cc and fresnel/cpu/TracerDirect.cc, and a binned-SAH BVH2 standing in
// for Embree's scene BVH.  Closest-hit results do not depend on the BVH: Embree keeps whichever
// of two primitives hit at exactly the same t its traversal offers first, and the oracle, like
// the engine, instead gives such exact ties to the lower (geometry, primitive) index
// (accept_hit below).  The shading/intersection arithmetic comes from namespace M, which is either the
// restatement (restated_math.hpp) or the reference's own headers (ref_math_adapter.hpp,
// selected with -DFR_ORACLE_REFERENCE_MATH).
//
// Build: oracle/build_oracle.py (g++ -O3 -ffp-contract=off, so no FMA contraction changes a
// rounding the reference does not make).

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <new>
#include <thread>
#include <vector>

#include "oracle.h"
#include "restated_math.hpp"

#ifdef FR_ORACLE_REFERENCE_MATH
#include "ref_math_adapter.hpp"
namespace M = frref;
static const char* k_math_kind = "reference-headers";
#else
namespace M = frm;
static const char* k_math_kind = "restated";
#endif

using frm::F3;
using frm::Mat;
using frm::PathState;
using frm::Quat;
using frm::RGB3;

namespace {

// ---------------------------------------------------------------------------------------------
// scene
// ---------------------------------------------------------------------------------------------
struct Geom {
    int type = 0;
    uint32_t n = 0;        // user primitives (mesh: instances)
    uint32_t n_faces = 0;  // mesh only
    std::vector<F3> position;
    std::vector<float> radius;
    std::vector<RGB3> color;
    std::vector<F3> points;  // cylinder: 2 per primitive
    std::vector<Quat> orientation;
    std::vector<F3> vertices;
    std::vector<F3> plane_origin, plane_normal;
    std::vector<RGB3> plane_color;
    float poly_radius = 0, color_by_face = 0;
    // polygon: 2-D positions, rotation quaternions (from the angles), 2-D outline vertices
    std::vector<float> pos2, verts2;
    std::vector<Quat> pq;
    float rounding_radius = 0, pg_radius = 0;
    Mat material{}, outline{};
    float outline_width = 0;
    bool enabled = true;
    uint32_t prim_count() const { return type == FR_GEOM_MESH ? n * n_faces : n; }
};

struct Box {
    float lo[3], hi[3];
};

struct Node {  // 32 bytes
    float lo[3];
    uint32_t a;  // interior: right child; leaf: first reference
    float hi[3];
    uint32_t count;  // 0 = interior (left child is this index + 1)
};

struct PrimRef {
    uint32_t geom, prim;
};

}  // namespace

struct or_scene {
    std::vector<Geom> geoms;  // indexed like the caller's array (disabled ones kept, unused)
    std::vector<Node> nodes;
    std::vector<PrimRef> refs;
};

namespace {

Mat to_mat(const fr_material& m)
{
    Mat r;
    r.solid = m.solid;
    r.color = RGB3{m.color[0], m.color[1], m.color[2]};
    r.primitive_color_mix = m.primitive_color_mix;
    r.roughness = m.roughness;
    r.specular = m.specular;
    r.metal = m.metal;
    r.spec_trans = m.spec_trans;
    return r;
}

inline void box_grow(Box& b, float x, float y, float z)
{
    b.lo[0] = std::min(b.lo[0], x);
    b.lo[1] = std::min(b.lo[1], y);
    b.lo[2] = std::min(b.lo[2], z);
    b.hi[0] = std::max(b.hi[0], x);
    b.hi[1] = std::max(b.hi[1], y);
    b.hi[2] = std::max(b.hi[2], z);
}

inline Box box_empty()
{
    const float inf = std::numeric_limits<float>::infinity();
    return Box{{inf, inf, inf}, {-inf, -inf, -inf}};
}

inline void box_union(Box& a, const Box& b)
{
    for (int k = 0; k < 3; ++k) {
        a.lo[k] = std::min(a.lo[k], b.lo[k]);
        a.hi[k] = std::max(a.hi[k], b.hi[k]);
    }
}

inline float box_area(const Box& b)
{
    float dx = b.hi[0] - b.lo[0], dy = b.hi[1] - b.lo[1], dz = b.hi[2] - b.lo[2];
    if (!(dx >= 0) || !(dy >= 0) || !(dz >= 0))
        return 0.0f;
    return 2.0f * (dx * dy + dy * dz + dz * dx);
}

inline Box box_of(float lx, float ly, float lz, float ux, float uy, float uz)
{
    return Box{{lx, ly, lz}, {ux, uy, uz}};
}

// Primitive bounds with the reference's formulas (fresnel/cpu/GeometrySphere.cc:60-73,
// GeometryCylinder.cc:55-70, GeometryConvexPolyhedron.cc:119-132, GeometryMesh.cc:81-113,
// GeometryPolygon.cc:89-104): a box with lower > upper (a negative radius) or a non-finite
// bound is left out of the tree, as Embree leaves out invalid user-geometry boxes.  Valid boxes
// are inflated by a small relative margin so that rounding in the box test can never cull a
// primitive the intersector accepts.
Box prim_box(const Geom& g, uint32_t prim)
{
    Box b = box_empty();
    switch (g.type) {
    case FR_GEOM_SPHERE: {
        F3 p = g.position[prim];
        float r = g.radius[prim];
        b = box_of(p.x - r, p.y - r, p.z - r, p.x + r, p.y + r, p.z + r);
        break;
    }
    case FR_GEOM_CYLINDER: {
        F3 A = g.points[2 * prim], B = g.points[2 * prim + 1];
        float r = g.radius[prim];
        b = box_of(std::min(A.x - r, B.x - r), std::min(A.y - r, B.y - r),
                   std::min(A.z - r, B.z - r), std::max(A.x + r, B.x + r),
                   std::max(A.y + r, B.y + r), std::max(A.z + r, B.z + r));
        break;
    }
    case FR_GEOM_POLYHEDRON: {
        F3 p = g.position[prim];
        float r = g.poly_radius;
        b = box_of(p.x - r, p.y - r, p.z - r, p.x + r, p.y + r, p.z + r);
        break;
    }
    case FR_GEOM_MESH: {
        uint32_t inst = prim / g.n_faces, face = prim % g.n_faces;
        F3 p = g.position[inst];
        Quat q = g.orientation[inst];
        for (int k = 0; k < 3; ++k) {
            F3 v = M::rotate(q, g.vertices[3 * face + k]) + p;
            box_grow(b, v.x, v.y, v.z);
        }
        break;
    }
    case FR_GEOM_POLYGON: {
        const float x = g.pos2[2 * prim], y = g.pos2[2 * prim + 1], r = g.pg_radius;
        b = box_of(x - r, y - r, float(0.0 - 1e-5), x + r, y + r, float(0.0 + 1e-5));
        break;
    }
    }
    for (int k = 0; k < 3; ++k)
        if (!(std::isfinite(b.lo[k]) && std::isfinite(b.hi[k]) && b.lo[k] <= b.hi[k]))
            return box_empty();
    float scale = 0;
    for (int k = 0; k < 3; ++k)
        scale = std::max(scale, std::max(std::fabs(b.lo[k]), std::fabs(b.hi[k])));
    float pad = 1e-5f * scale + 1e-6f * (b.hi[0] - b.lo[0] + b.hi[1] - b.lo[1] + b.hi[2] - b.lo[2])
                + 1e-30f;
    for (int k = 0; k < 3; ++k) {
        b.lo[k] -= pad;
        b.hi[k] += pad;
    }
    return b;
}

// ---------------------------------------------------------------------------------------------
// binned SAH BVH2
// ---------------------------------------------------------------------------------------------
struct Builder {
    std::vector<Box> boxes;
    std::vector<F3> cent;
    std::vector<uint32_t> idx;
    std::vector<Node>& nodes;
    int leaf_max;
    explicit Builder(std::vector<Node>& n, int lm) : nodes(n), leaf_max(lm) {}

    uint32_t build(uint32_t begin, uint32_t end)
    {
        Box bb = box_empty(), cb = box_empty();
        for (uint32_t i = begin; i < end; ++i) {
            box_union(bb, boxes[idx[i]]);
            box_grow(cb, cent[idx[i]].x, cent[idx[i]].y, cent[idx[i]].z);
        }
        uint32_t me = uint32_t(nodes.size());
        nodes.push_back(Node{});
        Node nd{};
        for (int k = 0; k < 3; ++k) {
            nd.lo[k] = bb.lo[k];
            nd.hi[k] = bb.hi[k];
        }
        uint32_t n = end - begin;
        auto make_leaf = [&]() {
            nd.a = begin;
            nd.count = n;
            nodes[me] = nd;
            return me;
        };
        if (n <= 1)
            return make_leaf();
        // best split over 32 bins per axis
        const int NB = 32;
        float best_cost = std::numeric_limits<float>::infinity();
        int best_axis = -1, best_bin = -1;
        for (int axis = 0; axis < 3; ++axis) {
            float lo = (&cb.lo[0])[axis], hi = (&cb.hi[0])[axis];
            if (!(hi > lo))
                continue;
            Box bin_box[NB];
            uint32_t bin_cnt[NB];
            for (int b = 0; b < NB; ++b) {
                bin_box[b] = box_empty();
                bin_cnt[b] = 0;
            }
            float scale = NB / (hi - lo);
            for (uint32_t i = begin; i < end; ++i) {
                float c = (&cent[idx[i]].x)[axis];
                int b = std::min(NB - 1, std::max(0, int((c - lo) * scale)));
                bin_cnt[b]++;
                box_union(bin_box[b], boxes[idx[i]]);
            }
            float right_area[NB];
            uint32_t right_cnt[NB];
            Box acc = box_empty();
            uint32_t cnt = 0;
            for (int b = NB - 1; b > 0; --b) {
                box_union(acc, bin_box[b]);
                cnt += bin_cnt[b];
                right_area[b] = box_area(acc);
                right_cnt[b] = cnt;
            }
            acc = box_empty();
            cnt = 0;
            for (int b = 0; b < NB - 1; ++b) {
                box_union(acc, bin_box[b]);
                cnt += bin_cnt[b];
                if (cnt == 0 || right_cnt[b + 1] == 0)
                    continue;
                float cost = box_area(acc) * cnt + right_area[b + 1] * right_cnt[b + 1];
                if (cost < best_cost) {
                    best_cost = cost;
                    best_axis = axis;
                    best_bin = b;
                }
            }
        }
        if (best_axis < 0) {
            // all centroids coincide
            if (int(n) <= leaf_max)
                return make_leaf();
            uint32_t mid = begin + n / 2;
            build(begin, mid);
            nd.a = build(mid, end);
            nd.count = 0;
            nodes[me] = nd;
            return me;
        }
        // SAH with unit traversal and intersection costs
        float leaf_cost = box_area(bb) * float(n);
        float split_cost = box_area(bb) + best_cost;
        if (int(n) <= leaf_max && leaf_cost <= split_cost)
            return make_leaf();
        float lo = (&cb.lo[0])[best_axis], hi = (&cb.hi[0])[best_axis];
        float scale = NB / (hi - lo);
        uint32_t* first = idx.data() + begin;
        uint32_t* last = idx.data() + end;
        uint32_t* mid = std::partition(first, last, [&](uint32_t p) {
            float c = (&cent[p].x)[best_axis];
            int b = std::min(NB - 1, std::max(0, int((c - lo) * scale)));
            return b <= best_bin;
        });
        uint32_t m = uint32_t(mid - idx.data());
        if (m == begin || m == end)
            m = begin + n / 2;
        build(begin, m);
        uint32_t r = build(m, end);
        nd.a = r;
        nd.count = 0;
        nodes[me] = nd;
        return me;
    }
};

// ---------------------------------------------------------------------------------------------
// closest-hit glue (Embree user-geometry intersect callbacks)
// ---------------------------------------------------------------------------------------------
struct Hit {
    float t;       // ray.tfar
    uint32_t geom;  // UINT32_MAX = miss
    uint32_t prim;
    F3 Ng;
    RGB3 color;
    float d;
};

// Acceptance of a candidate hit at t (fresnel/cpu/GeometrySphere.cc:101: tnear < t < tfar), with
// exact ties at tfar broken toward the lower (geometry, primitive) index; a ray with no hit yet
// never ties.
inline bool accept_hit(float t, float tnear, const Hit& h, uint32_t gi, uint32_t prim)
{
    if (!(tnear < t))
        return false;
    if (t < h.t)
        return true;
    return t == h.t && h.geom != UINT32_MAX && (gi < h.geom || (gi == h.geom && prim < h.prim));
}

// fresnel/cpu/GeometrySphere.cc:81-118
inline void glue_sphere(const Geom& g, uint32_t gi, uint32_t prim, F3 o, F3 dir, float tnear,
                        Hit& h)
{
    const F3 p = g.position[prim];
    const float r = g.radius[prim];
    float t = 0, d = 0;
    F3 N;
    bool hit = M::isect_sphere(t, d, N, o, dir, p, r);
    if (hit && accept_hit(t, tnear, h, gi, prim)) {
        h.t = t;
        h.geom = gi;
        h.prim = prim;
        h.Ng = F3{o.x + t * dir.x - p.x, o.y + t * dir.y - p.y, o.z + t * dir.z - p.z};
        h.color = g.color[prim];
        h.d = d;
    }
}

// fresnel/cpu/GeometryCylinder.cc:76-120
inline void glue_cylinder(const Geom& g, uint32_t gi, uint32_t prim, F3 o, F3 dir, float tnear,
                          Hit& h)
{
    const F3 A = g.points[2 * prim], B = g.points[2 * prim + 1];
    const float r = g.radius[prim];
    float t = HUGE_VALF, d = HUGE_VALF;
    F3 N{0, 0, 0};
    unsigned ci = 0;
    bool hit = M::isect_spherocylinder(t, d, N, ci, o, dir, A, B, r);
    if (hit && accept_hit(t, tnear, h, gi, prim)) {
        h.t = t;
        h.geom = gi;
        h.prim = prim;
        h.Ng = N;
        h.color = g.color[2 * prim + ci];
        h.d = d;
    }
}

// fresnel/cpu/GeometryConvexPolyhedron.cc:140-335
inline void glue_polyhedron(const Geom& g, uint32_t gi, uint32_t prim, F3 o, F3 dir, float tnear,
                            Hit& h)
{
    using frm::cross;
    using frm::dot;
    const int n_planes = int(g.plane_normal.size());
    float t0 = -std::numeric_limits<float>::max();
    float t1 = std::numeric_limits<float>::max();
    const F3 pos = g.position[prim];
    const Quat q = g.orientation[prim];
    F3 dl = M::rotate(M::conj(q), dir);
    F3 ol = M::rotate(M::conj(q), o - pos);
    F3 t0n{0, 0, 0}, t0p{0, 0, 0}, t1n{0, 0, 0}, t1p{0, 0, 0};
    int t0_plane = 0, t1_plane = 0;
    for (int i = 0; i < n_planes && t0 < t1; ++i) {
        F3 n = g.plane_normal[i];
        F3 p = g.plane_origin[i];
        float dd = -dot(n, p);
        float denom = dot(n, dl);
        float t = -(dd + dot(n, ol)) / denom;
        if (double(std::fabs(denom)) < 1e-5) {
            if (dot(ol - p, n) > 0)
                return;
        } else if (denom < 0) {
            if (t > t0) {
                t0 = t;
                t0n = n;
                t0p = p;
                t0_plane = i;
            }
        } else {
            if (t < t1) {
                t1 = t;
                t1n = n;
                t1p = p;
                t1_plane = i;
            }
        }
    }
    if (t0 > t1)
        return;
    float t_hit = 0;
    bool hit = false;
    F3 n_hit{0, 0, 0}, p_hit{0, 0, 0};
    Hit cand = h;
    if (accept_hit(t0, tnear, h, gi, prim)) {
        t_hit = t0;
        cand.Ng = M::rotate(q, t0n);
        n_hit = t0n;
        p_hit = t0p;
        cand.color = frm::lerp(g.color_by_face, g.color[prim], g.plane_color[t0_plane]);
        hit = true;
    } else if (accept_hit(t1, tnear, h, gi, prim)) {  // the exit (t1 >= t0)
        t_hit = t1;
        cand.Ng = M::rotate(q, t1n);
        n_hit = t1n;
        p_hit = t1p;
        cand.color = frm::lerp(g.color_by_face, g.color[prim], g.plane_color[t1_plane]);
        hit = true;
    }
    if (!hit)
        return;
    float min_d = std::numeric_limits<float>::max();
    F3 r_hit = ol + t_hit * dl;
    for (int i = 0; i < n_planes; ++i) {
        F3 n = g.plane_normal[i];
        F3 p = g.plane_origin[i];
        F3 u = cross(n, n_hit);
        if (double(std::fabs(dot(u, u))) >= 1e-5) {
            int maxc;
            if (std::fabs(u.x) > std::fabs(u.y))
                maxc = (std::fabs(u.x) > std::fabs(u.z)) ? 1 : 3;
            else
                maxc = (std::fabs(u.y) > std::fabs(u.z)) ? 2 : 3;
            F3 x0{0, 0, 0};
            float d1 = -dot(n, p);
            float d2 = -dot(n_hit, p_hit);
            switch (maxc) {
            case 1:
                x0.x = 0;
                x0.y = (d2 * n.z - d1 * n_hit.z) / u.x;
                x0.z = (d1 * n_hit.y - d2 * n.y) / u.x;
                break;
            case 2:
                x0.x = (d1 * n_hit.z - d2 * n.z) / u.y;
                x0.y = 0;
                x0.z = (d2 * n.x - d1 * n_hit.x) / u.y;
                break;
            default:
                x0.x = (d2 * n.y - d1 * n_hit.y) / u.z;
                x0.y = (d1 * n_hit.x - d2 * n.x) / u.z;
                x0.z = 0;
            }
            F3 view = frm::div_recip(-dl, sqrtf(dot(dl, dl)));
            u = u - dot(u, view) * view;
            F3 w = x0 - r_hit;
            F3 w_perp = w - dot(w, view) * view;
            x0 = r_hit + w_perp;
            F3 v = cross(u, x0 - r_hit);
            float dsq = dot(v, v) / dot(u, u);
            float dist = sqrtf(dsq);
            if (dist < min_d)
                min_d = dist;
        }
    }
    cand.t = t_hit;
    cand.geom = gi;
    cand.prim = prim;
    cand.d = min_d;
    h = cand;
}

// fresnel/cpu/GeometryMesh.cc:115-193 (double-sided: second test with v0/v1 swapped)
inline void glue_mesh(const Geom& g, uint32_t gi, uint32_t item, F3 o, F3 dir, float tnear, Hit& h)
{
    uint32_t inst = item / g.n_faces, face = item % g.n_faces;
    const F3 p3 = g.position[inst];
    const Quat q = g.orientation[inst];
    F3 dl = M::rotate(M::conj(q), dir);
    F3 ol = M::rotate(M::conj(q), o - p3);
    F3 v0 = g.vertices[3 * face], v1 = g.vertices[3 * face + 1], v2 = g.vertices[3 * face + 2];
    float u = 0, v = 0, w = 0, t = 0, d = 0;
    F3 n{0, 0, 0};
    if (!M::isect_triangle(u, v, w, t, d, n, ol, ol + dl, v0, v1, v2)
        && !M::isect_triangle(v, u, w, t, d, n, ol, ol + dl, v1, v0, v2))
        return;
    if (accept_hit(t, tnear, h, gi, item)) {
        h.t = t;
        h.geom = gi;
        h.prim = item;
        h.Ng = M::rotate(q, n);
        h.color = g.color[3 * face + 0] * u + g.color[3 * face + 1] * v + g.color[3 * face + 2] * w;
        h.d = d;
    }
}

// fresnel/cpu/GeometryPolygon.cc:146-230: the ray in the polygon's frame meets the z = 0 plane;
// the hit point's distance to the outline (is_inside, :113-140, with the point-segment distance
// of fresnel/common/GeometryMath.h:28-39), signed negative inside, must not exceed the rounding
// radius.  Double sided: the normal faces the ray.
inline void glue_polygon(const Geom& g, uint32_t gi, uint32_t prim, F3 o, F3 dir, float tnear,
                         Hit& h)
{
    using frm::dot;
    const F3 pos_world{g.pos2[2 * prim], g.pos2[2 * prim + 1], 0.0f};
    const Quat q = g.pq[prim];
    const F3 dl = M::rotate(M::conj(q), dir);
    const F3 ol = M::rotate(M::conj(q), o - pos_world);
    const F3 n{0, 0, 1};
    const F3 p{0, 0, 0};
    const float d = -dot(n, p);
    const float denom = dot(n, dl);
    const float t_hit = -(d + dot(n, ol)) / denom;
    if (double(std::fabs(denom)) < 1e-5)
        return;
    const F3 r_hit = ol + t_hit * dl;
    // is_inside: crossing number (odd = inside) and the distance to the nearest edge
    const uint32_t nvert = uint32_t(g.verts2.size() / 2);
    float min_d = FLT_MAX;
    bool odd = false;
    uint32_t j = nvert - 1;
    for (uint32_t i = 0; i < nvert; ++i) {
        const float xi = g.verts2[2 * i], yi = g.verts2[2 * i + 1];
        const float xj = g.verts2[2 * j], yj = g.verts2[2 * j + 1];
        const float dist = M::point_segment_distance(r_hit.x, r_hit.y, xi, yi, xj, yj);
        min_d = (dist < min_d) ? dist : min_d;  // std::min(min_d, dist)
        if ((yi < r_hit.y && yj >= r_hit.y) || (yj < r_hit.y && yi >= r_hit.y)) {
            if (xi + (r_hit.y - yi) / (yj - yi) * (xj - xi) < r_hit.x)
                odd = !odd;
        }
        j = i;
    }
    float d_edge = min_d;
    if (odd)
        d_edge = -d_edge;
    if (d_edge > g.rounding_radius)
        return;
    const float shade_d = g.rounding_radius - d_edge;
    if (accept_hit(t_hit, tnear, h, gi, prim)) {
        h.t = t_hit;
        h.geom = gi;
        h.prim = prim;
        const F3 n_flip = (dot(n, dl) < 0.0f) ? n : -n;
        h.Ng = M::rotate(q, n_flip);
        h.color = g.color[prim];
        h.d = shade_d;
    }
}

struct Counters {
    uint64_t rays = 0, box = 0, prim = 0, paths = 0, nonfinite = 0;
};

inline bool slab(const Node& nd, const float o[3], const float inv[3], float tmax, float& tentry)
{
    float t0 = 0.0f, t1 = tmax;
    for (int k = 0; k < 3; ++k) {
        float a = (nd.lo[k] - o[k]) * inv[k];
        float b = (nd.hi[k] - o[k]) * inv[k];
        if (a > b)
            std::swap(a, b);
        t0 = a > t0 ? a : t0;
        t1 = b < t1 ? b : t1;
    }
    tentry = t0;
    return t0 <= t1;
}

// Optional log of the rays trace() answers (or_set_ray_log): 7 floats per ray (origin,
// direction, tnear), appended by every thread; rays past the capacity are counted, not stored.
float* g_ray_log = nullptr;
uint64_t g_ray_log_cap = 0;
std::atomic<uint64_t> g_ray_log_n{0};

inline void log_ray(F3 o, F3 d, float tnear)
{
    const uint64_t i = g_ray_log_n.fetch_add(1, std::memory_order_relaxed);
    if (i < g_ray_log_cap) {
        float* r = g_ray_log + 7 * i;
        r[0] = o.x;
        r[1] = o.y;
        r[2] = o.z;
        r[3] = d.x;
        r[4] = d.y;
        r[5] = d.z;
        r[6] = tnear;
    }
}

// Closest hit in (tnear, inf): Embree's rtcIntersect1 with fresnel's user geometries.
Hit trace(const or_scene& s, F3 o, F3 d, float tnear, Counters& c)
{
    Hit h;
    h.t = std::numeric_limits<float>::infinity();
    h.geom = UINT32_MAX;
    h.prim = 0;
    c.rays++;
    if (g_ray_log)
        log_ray(o, d, tnear);
    if (s.nodes.empty())
        return h;
    float of[3] = {o.x, o.y, o.z};
    float df[3] = {d.x, d.y, d.z};
    float inv[3];
    for (int k = 0; k < 3; ++k) {
        float dk = df[k];
        if (std::fabs(dk) < 1e-30f)
            dk = std::copysign(1e-30f, dk);
        inv[k] = 1.0f / dk;
    }
    uint32_t stack[128];
    int sp = 0;
    uint32_t cur = 0;
    float te;
    c.box++;
    if (!slab(s.nodes[0], of, inv, h.t, te))
        return h;
    while (true) {
        const Node& nd = s.nodes[cur];
        if (nd.count > 0) {
            for (uint32_t k = 0; k < nd.count; ++k) {
                const PrimRef& r = s.refs[nd.a + k];
                const Geom& g = s.geoms[r.geom];
                c.prim++;
                switch (g.type) {
                case FR_GEOM_SPHERE:
                    glue_sphere(g, r.geom, r.prim, o, d, tnear, h);
                    break;
                case FR_GEOM_CYLINDER:
                    glue_cylinder(g, r.geom, r.prim, o, d, tnear, h);
                    break;
                case FR_GEOM_POLYHEDRON:
                    glue_polyhedron(g, r.geom, r.prim, o, d, tnear, h);
                    break;
                case FR_GEOM_MESH:
                    glue_mesh(g, r.geom, r.prim, o, d, tnear, h);
                    break;
                case FR_GEOM_POLYGON:
                    glue_polygon(g, r.geom, r.prim, o, d, tnear, h);
                    break;
                }
            }
        } else {
            uint32_t l = cur + 1, r = nd.a;
            float tl, tr;
            c.box += 2;
            bool hl = slab(s.nodes[l], of, inv, h.t, tl);
            bool hr = slab(s.nodes[r], of, inv, h.t, tr);
            if (hl && hr) {
                if (tr < tl)
                    std::swap(l, r);
                if (sp < 128)
                    stack[sp++] = r;
                cur = l;
                continue;
            }
            if (hl) {
                cur = l;
                continue;
            }
            if (hr) {
                cur = r;
                continue;
            }
        }
        // pop (re-test against the shrunken tmax)
        bool found = false;
        while (sp > 0) {
            uint32_t nxt = stack[--sp];
            c.box++;
            if (slab(s.nodes[nxt], of, inv, h.t, te)) {
                cur = nxt;
                found = true;
                break;
            }
        }
        if (!found)
            break;
    }
    return h;
}

// ---------------------------------------------------------------------------------------------
// The engine's uniform sphere grid, restated on the CPU to measure what walking it costs per ray
// (cells visited, spheres tested) on rays the oracle's own renders trace.  Definition: every
// sphere's box (centre -+ r; left out when not finite or inverted), padded by 1e-5 * max|coord| +
// 1e-6 * (sum of extents); the grid spans the union of the padded boxes; cell size
// h = cbrt(volume / (cells_per_sphere * valid spheres)), dims = ceil(extent / h) clamped to
// [1, 1024] per axis (h grown by 1.25 until at most 2^26 cells); each cell lists the spheres whose
// padded box overlaps it, in sphere order.  Walk: a 3-D DDA (Amanatides & Woo 1987) from the cell
// of the ray's entry point; each visited cell's spheres are tested (tnear < t < tmax); the walk
// stops once the closest hit so far lies before the cell's exit.
// ---------------------------------------------------------------------------------------------
struct SphereGrid {
    float lo[3], hi[3], cell[3], ih[3];
    int n[3];
    std::vector<uint32_t> start;  // per cell: first reference; start[cells] = total
    std::vector<uint32_t> refs;   // sphere indices
    const float* pos = nullptr;
    const float* rad = nullptr;
};

inline bool sphere_box_padded(const float* pos, const float* rad, uint32_t i, float blo[3],
                              float bhi[3])
{
    const float r = rad[i];
    bool ok = true;
    for (int k = 0; k < 3; ++k) {
        const float c = pos[3 * size_t(i) + k];
        blo[k] = c - r;
        bhi[k] = c + r;
        ok = ok && std::isfinite(blo[k]) && std::isfinite(bhi[k]) && blo[k] <= bhi[k];
    }
    if (!ok)
        return false;
    float scale = 0.0f, ext = 0.0f;
    for (int k = 0; k < 3; ++k) {
        scale = std::max(scale, std::max(std::fabs(blo[k]), std::fabs(bhi[k])));
        ext += bhi[k] - blo[k];
    }
    const float pad = 1e-5f * scale + 1e-6f * ext + 1e-30f;
    for (int k = 0; k < 3; ++k) {
        blo[k] -= pad;
        bhi[k] += pad;
    }
    return true;
}

inline int grid_cell_index(float x, float lo, float ih, int n)
{
    const float u = std::floor((x - lo) * ih);
    return int(std::min(std::max(u, 0.0f), float(n - 1)));
}

bool build_sphere_grid(const float* pos, const float* rad, uint32_t n, float cells_per_sphere,
                       SphereGrid& G)
{
    G.pos = pos;
    G.rad = rad;
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    uint32_t valid = 0;
    float blo[3], bhi[3];
    for (uint32_t i = 0; i < n; ++i) {
        if (!sphere_box_padded(pos, rad, i, blo, bhi))
            continue;
        for (int k = 0; k < 3; ++k) {
            mn[k] = std::min(mn[k], blo[k]);
            mx[k] = std::max(mx[k], bhi[k]);
        }
        ++valid;
    }
    if (valid == 0)
        return false;
    double lo[3], ext[3], scale = 1.0;
    for (int k = 0; k < 3; ++k) {
        lo[k] = mn[k];
        ext[k] = double(mx[k]) - lo[k];
        scale = std::max(scale, std::max(std::fabs(lo[k]), std::fabs(lo[k] + ext[k])));
    }
    for (int k = 0; k < 3; ++k)
        ext[k] = std::max(ext[k], 1e-6 * scale);
    const double volume = ext[0] * ext[1] * ext[2];
    double h = std::cbrt(volume / (double(cells_per_sphere) * valid));
    for (int pass = 0; pass < 64; ++pass) {
        double cells = 1.0;
        for (int k = 0; k < 3; ++k) {
            G.n[k] = int(std::min(1024.0, std::max(1.0, std::ceil(ext[k] / h))));
            cells *= G.n[k];
        }
        if (cells <= double(1u << 26))
            break;
        h *= 1.25;
    }
    for (int k = 0; k < 3; ++k) {
        G.lo[k] = float(lo[k]);
        G.cell[k] = float(ext[k] / G.n[k]) * (1.0f + 4e-7f);
        G.ih[k] = 1.0f / G.cell[k];
        G.hi[k] = G.lo[k] + float(G.n[k]) * G.cell[k];
    }
    const size_t cells = size_t(G.n[0]) * G.n[1] * G.n[2];
    std::vector<uint32_t> count(cells + 1, 0);
    auto for_cells = [&](uint32_t i, auto&& f) {
        if (!sphere_box_padded(pos, rad, i, blo, bhi))
            return;
        int a[3], b[3];
        for (int k = 0; k < 3; ++k) {
            a[k] = grid_cell_index(blo[k], G.lo[k], G.ih[k], G.n[k]);
            b[k] = grid_cell_index(bhi[k], G.lo[k], G.ih[k], G.n[k]);
        }
        for (int z = a[2]; z <= b[2]; ++z)
            for (int y = a[1]; y <= b[1]; ++y)
                for (int x = a[0]; x <= b[0]; ++x)
                    f((size_t(z) * G.n[1] + y) * G.n[0] + x);
    };
    for (uint32_t i = 0; i < n; ++i)
        for_cells(i, [&](size_t c) { count[c + 1]++; });
    for (size_t c = 0; c < cells; ++c)
        count[c + 1] += count[c];
    G.start = count;
    G.refs.assign(count[cells], 0);
    std::vector<uint32_t> fill(count.begin(), count.end() - 1);
    for (uint32_t i = 0; i < n; ++i)
        for_cells(i, [&](size_t c) { G.refs[fill[c]++] = i; });
    return true;
}

// Walks one ray; returns the closest sphere (UINT32_MAX: none) and counts cells and spheres.
uint32_t walk_sphere_grid(const SphereGrid& G, F3 o, F3 d, float tnear, uint64_t& cells,
                          uint64_t& tests)
{
    float inv[3], oinv[3];
    const float of[3] = {o.x, o.y, o.z}, df[3] = {d.x, d.y, d.z};
    for (int k = 0; k < 3; ++k) {
        const float a = std::fabs(df[k]);
        inv[k] = 1.0f / (a < 1e-30f ? std::copysign(1e-30f, df[k]) : df[k]);
        oinv[k] = -of[k] * inv[k];
    }
    float t0[3], t1[3];
    for (int k = 0; k < 3; ++k) {
        t0[k] = std::fma(G.lo[k], inv[k], oinv[k]);
        t1[k] = std::fma(G.hi[k], inv[k], oinv[k]);
    }
    const float t_in = std::max(std::max(std::min(t0[0], t1[0]), std::min(t0[1], t1[1])),
                                std::max(std::min(t0[2], t1[2]), 0.0f));
    const float t_out = std::min(std::min(std::max(t0[0], t1[0]), std::max(t0[1], t1[1])),
                                 std::max(t0[2], t1[2]));
    if (!(t_in <= t_out))
        return UINT32_MAX;
    int c[3], s[3];
    float tn[3];
    for (int k = 0; k < 3; ++k) {
        const float u = (of[k] + t_in * df[k] - G.lo[k]) * G.ih[k];
        c[k] = u >= 0.0f ? int(std::min(u, float(G.n[k] - 1))) : 0;
        s[k] = inv[k] >= 0.0f ? 1 : -1;
        tn[k] = std::fma(std::fma(float(c[k] + (inv[k] >= 0.0f ? 1 : 0)), G.cell[k], G.lo[k]), inv[k],
                         oinv[k]);
    }
    float tmax = INFINITY;
    uint32_t best = UINT32_MAX;
    for (int guard = G.n[0] + G.n[1] + G.n[2] + 3; guard > 0; --guard) {
        const size_t cell = (size_t(c[2]) * G.n[1] + c[1]) * G.n[0] + c[0];
        ++cells;
        for (uint32_t r = G.start[cell]; r < G.start[cell + 1]; ++r) {
            const uint32_t i = G.refs[r];
            ++tests;
            float t = 0, de = 0;
            F3 N;
            const F3 p{G.pos[3 * size_t(i)], G.pos[3 * size_t(i) + 1], G.pos[3 * size_t(i) + 2]};
            if (M::isect_sphere(t, de, N, o, d, p, G.rad[i]) && tnear < t &&
                (t < tmax || (t == tmax && i < best))) {
                tmax = t;
                best = i;
            }
        }
        const float t_cell = std::min(tn[0], std::min(tn[1], tn[2]));
        const int axis = (tn[0] <= tn[1] && tn[0] <= tn[2]) ? 0 : (tn[1] <= tn[2] ? 1 : 2);
        c[axis] += s[axis];
        if (tmax <= t_cell || !(t_cell < t_out) || c[axis] < 0 || c[axis] >= G.n[axis])
            break;
        tn[axis] = std::fma(std::fma(float(c[axis] + (inv[axis] >= 0.0f ? 1 : 0)), G.cell[axis],
                                     G.lo[axis]),
                            inv[axis], oinv[axis]);
    }
    return best;
}

// ---------------------------------------------------------------------------------------------
// The engine's grid over a scene's parts, restated to measure what walking it costs per ray
// (cells visited, references listed in them) on rays the oracle's own renders trace.
// Definition: one reference per primitive of every enabled geometry (its padded prim_box), but
// one per mesh instance (the box of all its rotated vertices, padded by the same rule); boxes
// that are not finite or are inverted are left out; the grid's shape follows the sphere grid's
// rule over these boxes.  Walk: the sphere grid's DDA, ending at the first cell whose exit lies
// at or beyond the closest hit (the oracle's own trace) or at the grid's exit.  The engine's walk
// ends there too: the closest primitive is referenced by the cell that holds the hit point, so
// once that cell is tested the closest hit so far is the closest hit, and no earlier cell's exit
// reaches it.
// ---------------------------------------------------------------------------------------------
struct CountGrid {
    float lo[3], cell[3], ih[3];
    int n[3];
    std::vector<uint32_t> count;  // references per cell
    uint64_t refs = 0;
};

Box pad_box(Box b)
{
    for (int k = 0; k < 3; ++k)
        if (!(std::isfinite(b.lo[k]) && std::isfinite(b.hi[k]) && b.lo[k] <= b.hi[k]))
            return box_empty();
    float scale = 0;
    for (int k = 0; k < 3; ++k)
        scale = std::max(scale, std::max(std::fabs(b.lo[k]), std::fabs(b.hi[k])));
    float pad = 1e-5f * scale + 1e-6f * (b.hi[0] - b.lo[0] + b.hi[1] - b.lo[1] + b.hi[2] - b.lo[2])
                + 1e-30f;
    for (int k = 0; k < 3; ++k) {
        b.lo[k] -= pad;
        b.hi[k] += pad;
    }
    return b;
}

Box instance_box(const Geom& g, uint32_t inst)
{
    Box b = box_empty();
    const F3 p = g.position[inst];
    const Quat q = g.orientation[inst];
    for (size_t k = 0; k < g.vertices.size(); ++k) {
        F3 v = M::rotate(q, g.vertices[k]) + p;
        box_grow(b, v.x, v.y, v.z);
    }
    return pad_box(b);
}

bool valid_box(const Box& b)
{
    return b.lo[0] <= b.hi[0] && b.lo[1] <= b.hi[1] && b.lo[2] <= b.hi[2];
}

bool build_count_grid(const std::vector<Box>& boxes, float cells_per_prim, CountGrid& G)
{
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    uint32_t valid = 0;
    for (const Box& b : boxes) {
        if (!valid_box(b))
            continue;
        for (int k = 0; k < 3; ++k) {
            mn[k] = std::min(mn[k], b.lo[k]);
            mx[k] = std::max(mx[k], b.hi[k]);
        }
        ++valid;
    }
    if (valid == 0)
        return false;
    double lo[3], ext[3], scale = 1.0;
    for (int k = 0; k < 3; ++k) {
        lo[k] = mn[k];
        ext[k] = double(mx[k]) - lo[k];
        scale = std::max(scale, std::max(std::fabs(lo[k]), std::fabs(lo[k] + ext[k])));
    }
    for (int k = 0; k < 3; ++k)
        ext[k] = std::max(ext[k], 1e-6 * scale);
    const double volume = ext[0] * ext[1] * ext[2];
    double h = std::cbrt(volume / (double(cells_per_prim) * valid));
    for (int pass = 0; pass < 64; ++pass) {
        double cells = 1.0;
        for (int k = 0; k < 3; ++k) {
            G.n[k] = int(std::min(1024.0, std::max(1.0, std::ceil(ext[k] / h))));
            cells *= G.n[k];
        }
        if (cells <= double(1u << 26))
            break;
        h *= 1.25;
    }
    for (int k = 0; k < 3; ++k) {
        G.lo[k] = float(lo[k]);
        G.cell[k] = float(ext[k] / G.n[k]) * (1.0f + 4e-7f);
        G.ih[k] = 1.0f / G.cell[k];
    }
    G.count.assign(size_t(G.n[0]) * G.n[1] * G.n[2], 0);
    G.refs = 0;
    for (const Box& b : boxes) {
        if (!valid_box(b))
            continue;
        int a[3], c[3];
        for (int k = 0; k < 3; ++k) {
            a[k] = grid_cell_index(b.lo[k], G.lo[k], G.ih[k], G.n[k]);
            c[k] = grid_cell_index(b.hi[k], G.lo[k], G.ih[k], G.n[k]);
        }
        for (int z = a[2]; z <= c[2]; ++z)
            for (int y = a[1]; y <= c[1]; ++y)
                for (int x = a[0]; x <= c[0]; ++x) {
                    G.count[(size_t(z) * G.n[1] + y) * G.n[0] + x]++;
                    G.refs++;
                }
    }
    return true;
}

// Cells and references of one ray's walk up to the closest hit at t_hit (inf: none).
void walk_count_grid(const CountGrid& G, F3 o, F3 d, float t_hit, uint64_t& cells, uint64_t& refs)
{
    float inv[3], oinv[3], hi[3];
    const float of[3] = {o.x, o.y, o.z}, df[3] = {d.x, d.y, d.z};
    for (int k = 0; k < 3; ++k) {
        const float a = std::fabs(df[k]);
        inv[k] = 1.0f / (a < 1e-30f ? std::copysign(1e-30f, df[k]) : df[k]);
        oinv[k] = -of[k] * inv[k];
        hi[k] = G.lo[k] + float(G.n[k]) * G.cell[k];
    }
    float t0[3], t1[3];
    for (int k = 0; k < 3; ++k) {
        t0[k] = std::fma(G.lo[k], inv[k], oinv[k]);
        t1[k] = std::fma(hi[k], inv[k], oinv[k]);
    }
    const float t_in = std::max(std::max(std::min(t0[0], t1[0]), std::min(t0[1], t1[1])),
                                std::max(std::min(t0[2], t1[2]), 0.0f));
    const float t_out = std::min(std::min(std::max(t0[0], t1[0]), std::max(t0[1], t1[1])),
                                 std::max(t0[2], t1[2]));
    if (!(t_in <= t_out))
        return;
    int c[3], s[3];
    float tn[3];
    for (int k = 0; k < 3; ++k) {
        const float u = (of[k] + t_in * df[k] - G.lo[k]) * G.ih[k];
        c[k] = u >= 0.0f ? int(std::min(u, float(G.n[k] - 1))) : 0;
        s[k] = inv[k] >= 0.0f ? 1 : -1;
        tn[k] = std::fma(std::fma(float(c[k] + (inv[k] >= 0.0f ? 1 : 0)), G.cell[k], G.lo[k]), inv[k],
                         oinv[k]);
    }
    for (int guard = G.n[0] + G.n[1] + G.n[2] + 3; guard > 0; --guard) {
        ++cells;
        refs += G.count[(size_t(c[2]) * G.n[1] + c[1]) * G.n[0] + c[0]];
        const float t_cell = std::min(tn[0], std::min(tn[1], tn[2]));
        const int axis = (tn[0] <= tn[1] && tn[0] <= tn[2]) ? 0 : (tn[1] <= tn[2] ? 1 : 2);
        c[axis] += s[axis];
        if (t_hit <= t_cell || !(t_cell < t_out) || c[axis] < 0 || c[axis] >= G.n[axis])
            break;
        tn[axis] = std::fma(std::fma(float(c[axis] + (inv[axis] >= 0.0f ? 1 : 0)), G.cell[axis],
                                     G.lo[axis]),
                            inv[axis], oinv[axis]);
    }
}

// ---------------------------------------------------------------------------------------------
// tile loops
// ---------------------------------------------------------------------------------------------
template <class F> void parallel_tiles(uint32_t n_items, int nthreads, F&& body)
{
    if (nthreads <= 0)
        nthreads = int(std::max(1u, std::thread::hardware_concurrency()));
    nthreads = std::max(1, std::min<int>(nthreads, int(n_items)));
    std::atomic<uint32_t> next(0);
    auto worker = [&](int tid) {
        while (true) {
            uint32_t it = next.fetch_add(1);
            if (it >= n_items)
                break;
            body(it, tid);
        }
    };
    if (nthreads == 1) {
        worker(0);
        return;
    }
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; ++t)
        th.emplace_back(worker, t);
    for (auto& t : th)
        t.join();
}

frm::CameraIn to_camera(const fr_user_camera& c)
{
    frm::CameraIn k;
    k.position = F3{c.position[0], c.position[1], c.position[2]};
    k.look_at = F3{c.look_at[0], c.look_at[1], c.look_at[2]};
    k.up = F3{c.up[0], c.up[1], c.up[2]};
    k.h = c.h;
    k.f = c.f;
    k.f_stop = c.f_stop;
    k.focus_distance = c.focus_distance;
    k.model = c.model;
    return k;
}

frm::LightsW world_lights(const fr_lights& in, const M::Cam& cam)
{
    F3 dir[4];
    RGB3 col[4];
    float th[4];
    unsigned n = std::min<unsigned>(in.n, 4);
    for (unsigned i = 0; i < n; ++i) {
        dir[i] = F3{in.direction[i][0], in.direction[i][1], in.direction[i][2]};
        col[i] = RGB3{in.color[i][0], in.color[i][1], in.color[i][2]};
        th[i] = in.theta[i];
    }
    return M::lights_to_world(dir, col, th, n, cam);
}

void write_srgb(const fr_render_params& p, const float px[4], uint8_t* out)
{
    if (!p.highlight_warning || (px[0] <= 1.0f && px[1] <= 1.0f && px[2] <= 1.0f)) {
        M::srgb_encode(px, out);
    } else {
        float c[4] = {p.highlight_color[0], p.highlight_color[1], p.highlight_color[2], px[3]};
        M::srgb_encode(c, out);
    }
}

inline bool finite3(RGB3 c) { return std::isfinite(c.r) && std::isfinite(c.g) && std::isfinite(c.b); }

}  // namespace

// =============================================================================================
// C interface
// =============================================================================================
extern "C" {

const char* or_math_kind(void) { return k_math_kind; }

or_scene* or_scene_create(const or_geometry_desc* gd, uint32_t n_geoms, int leaf_max)
{
    or_scene* s = new (std::nothrow) or_scene();
    if (!s)
        return nullptr;
    if (leaf_max < 1)
        leaf_max = 4;
    s->geoms.resize(n_geoms);
    Builder b(s->nodes, leaf_max);
    for (uint32_t gi = 0; gi < n_geoms; ++gi) {
        const or_geometry_desc& d = gd[gi];
        Geom& g = s->geoms[gi];
        g.type = d.type;
        g.n = d.n;
        g.material = to_mat(d.material);
        g.outline = to_mat(d.outline_material);
        g.outline_width = d.outline_width;
        g.poly_radius = d.poly_radius;
        g.color_by_face = d.color_by_face;
        auto f3 = [](const float* a, size_t n) {
            std::vector<F3> v(n);
            for (size_t i = 0; i < n; ++i)
                v[i] = F3{a[3 * i], a[3 * i + 1], a[3 * i + 2]};
            return v;
        };
        auto c3 = [](const float* a, size_t n) {
            std::vector<RGB3> v(n);
            for (size_t i = 0; i < n; ++i)
                v[i] = RGB3{a[3 * i], a[3 * i + 1], a[3 * i + 2]};
            return v;
        };
        auto q4 = [](const float* a, size_t n) {
            std::vector<Quat> v(n);
            for (size_t i = 0; i < n; ++i)
                v[i] = Quat{a[4 * i], F3{a[4 * i + 1], a[4 * i + 2], a[4 * i + 3]}};
            return v;
        };
        switch (d.type) {
        case FR_GEOM_SPHERE:
            g.position = f3(d.position, d.n);
            g.radius.assign(d.radius, d.radius + d.n);
            g.color = c3(d.color, d.n);
            break;
        case FR_GEOM_CYLINDER:
            g.points = f3(d.points, size_t(d.n) * 2);
            g.radius.assign(d.radius, d.radius + d.n);
            g.color = c3(d.color, size_t(d.n) * 2);
            break;
        case FR_GEOM_POLYHEDRON:
            g.position = f3(d.position, d.n);
            g.orientation = q4(d.orientation, d.n);
            g.color = c3(d.color, d.n);
            g.plane_origin = f3(d.plane_origin, d.n_planes);
            g.plane_normal = f3(d.plane_normal, d.n_planes);
            g.plane_color = c3(d.plane_color, d.n_planes);
            break;
        case FR_GEOM_MESH:
            if (d.n_vertices % 3 != 0) {
                delete s;
                return nullptr;
            }
            g.n_faces = d.n_vertices / 3;
            g.position = f3(d.position, d.n);
            g.orientation = q4(d.orientation, d.n);
            g.vertices = f3(d.vertices, d.n_vertices);
            g.color = c3(d.color, d.n_vertices);
            break;
        case FR_GEOM_POLYGON: {  // fresnel/cpu/GeometryPolygon.cc:20-82
            g.pos2.assign(d.position, d.position + 2 * size_t(d.n));
            g.color = c3(d.color, d.n);
            g.verts2.assign(d.vertices, d.vertices + 2 * size_t(d.n_vertices));
            g.rounding_radius = d.rounding_radius;
            float r = 0;
            for (uint32_t i = 0; i < d.n_vertices; ++i) {
                const float x = d.vertices[2 * i], y = d.vertices[2 * i + 1];
                r = std::max(r, sqrtf(x * x + y * y));
            }
            g.pg_radius = r + d.rounding_radius;
            g.pq.resize(d.n);
            for (uint32_t i = 0; i < d.n; ++i)
                g.pq[i] = M::from_axis_angle(F3{0, 0, 1}, d.angle[i]);
            break;
        }
        default:
            delete s;
            return nullptr;
        }
        g.enabled = d.enabled != 0;
        if (!d.enabled)
            continue;
        uint32_t np = g.prim_count();
        for (uint32_t p = 0; p < np; ++p) {
            Box bx = prim_box(g, p);
            bool ok = true;
            for (int k = 0; k < 3; ++k)
                ok = ok && std::isfinite(bx.lo[k]) && std::isfinite(bx.hi[k]) && bx.lo[k] <= bx.hi[k];
            if (!ok)
                continue;  // invalid primitive (e.g. infinite radius) is never hit
            s->refs.push_back(PrimRef{gi, p});
            b.boxes.push_back(bx);
        }
    }
    size_t n = s->refs.size();
    if (n > 0) {
        b.cent.resize(n);
        b.idx.resize(n);
        for (size_t i = 0; i < n; ++i) {
            const Box& bx = b.boxes[i];
            b.cent[i] = F3{0.5f * (bx.lo[0] + bx.hi[0]), 0.5f * (bx.lo[1] + bx.hi[1]),
                           0.5f * (bx.lo[2] + bx.hi[2])};
            b.idx[i] = uint32_t(i);
        }
        s->nodes.reserve(2 * n);
        b.build(0, uint32_t(n));
        std::vector<PrimRef> sorted(n);
        for (size_t i = 0; i < n; ++i)
            sorted[i] = s->refs[b.idx[i]];
        s->refs.swap(sorted);
    }
    return s;
}

void or_scene_destroy(or_scene* s) { delete s; }

void or_scene_info(const or_scene* s, uint64_t* nodes, uint64_t* prims)
{
    if (nodes)
        *nodes = s->nodes.size();
    if (prims)
        *prims = s->refs.size();
}

int or_trace(const or_scene* s, const float o[3], const float d[3], float tnear, float* t,
             uint32_t* geom, uint32_t* prim)
{
    Counters c;
    Hit h = trace(*s, F3{o[0], o[1], o[2]}, F3{d[0], d[1], d[2]}, tnear, c);
    if (h.geom == UINT32_MAX)
        return 0;
    *t = h.t;
    *geom = h.geom;
    *prim = h.prim;
    return 1;
}

int or_render_path(const or_scene* s, const fr_render_params* p, uint32_t w, uint32_t h,
                   uint32_t first_sample, uint32_t n_render, uint32_t light_samples, float* linear,
                   uint8_t* srgb, float* m2, const uint32_t* pixels, uint32_t n_pixels,
                   int nan_guard, int nthreads, or_stats* stats)
{
    if (!s || !p || w == 0 || h == 0 || light_samples == 0 || !linear || !srgb)
        return 1;
    const uint32_t seed = p->seed;
    const M::Cam cam = M::make_camera(to_camera(p->camera), w, h, seed, true);
    const frm::LightsW lights = world_lights(p->lights, cam);
    const RGB3 bg{p->background_color[0], p->background_color[1], p->background_color[2]};
    const float bg_alpha = p->background_alpha;

    const uint32_t TS = 4;  // 4x4 tiles (fresnel/cpu/TracerPath.cc:78-83)
    const uint32_t ntx = (w + TS - 1) / TS, nty = (h + TS - 1) / TS;
    const uint32_t n_items = pixels ? (n_pixels + 15) / 16 : ntx * nty;
    int nt = nthreads <= 0 ? int(std::max(1u, std::thread::hardware_concurrency())) : nthreads;
    std::vector<Counters> cnt(size_t(std::max(1, nt)));

    auto shade_pixel = [&](uint32_t i, uint32_t j, uint32_t slot, Counters& c) {
        const uint32_t key0 = j * w + i;
        for (uint32_t k = 0; k < n_render; ++k) {
            const uint32_t n_samples = first_sample + k;
            PathState st;
            st.result = RGB3{0, 0, 0};
            st.a = 1.0f;
            st.origin = F3{0, 0, 0};
            st.dir = F3{0, 0, 0};
            F3 o0, d0;
            M::camera_ray(cam, i, j, n_samples, o0, d0);
            Hit h0 = trace(*s, o0, d0, 1e-3f, c);
            for (st.light_sample = 0; st.light_sample < light_samples; st.light_sample++) {
                st.att = RGB3{1.0f, 1.0f, 1.0f};
                st.done = false;
                c.paths++;
                for (st.depth = 0;; st.depth++) {
                    Hit hh;
                    F3 ro, rd;
                    if (st.depth == 0) {
                        hh = h0;
                        ro = o0;
                        rd = d0;
                    } else {
                        ro = st.origin;
                        rd = st.dir;
                        hh = trace(*s, ro, rd, 1e-3f, c);
                    }
                    if (hh.geom != UINT32_MAX) {
                        const Geom& g = s->geoms[hh.geom];
                        M::path_hit(st, g.material, g.outline, hh.d, g.outline_width, hh.color,
                                    hh.Ng, ro, rd, hh.t, key0, seed, n_samples, light_samples);
                    } else {
                        M::path_miss(st, bg, bg_alpha, light_samples, lights, rd);
                    }
                    if (st.done)
                        break;
                }
            }
            // Welford running mean (fresnel/cpu/TracerPath.cc:228-239)
            RGB3 out = frm::rgb_div_recip(st.result, float(light_samples));
            float* px = linear + size_t(slot) * 4;
            float q = 1.0f / float(n_samples);
            float nm[4] = {px[0] + (out.r - px[0]) * q, px[1] + (out.g - px[1]) * q,
                           px[2] + (out.b - px[2]) * q, px[3] + (st.a - px[3]) * q};
            bool fin = std::isfinite(nm[0]) && std::isfinite(nm[1]) && std::isfinite(nm[2]);
            if (!fin)
                c.nonfinite++;
            if (!fin && nan_guard) {
                // keep the previous mean (fresnel/gpu/path.cu:111-113)
            } else {
                if (m2) {
                    float* mm = m2 + size_t(slot) * 3;
                    float xs[3] = {out.r, out.g, out.b};
                    for (int kk = 0; kk < 3; ++kk)
                        mm[kk] += (xs[kk] - px[kk]) * (xs[kk] - nm[kk]);
                }
                px[0] = nm[0];
                px[1] = nm[1];
                px[2] = nm[2];
                px[3] = nm[3];
            }
            write_srgb(*p, px, srgb + size_t(slot) * 4);
        }
    };

    parallel_tiles(n_items, nt, [&](uint32_t item, int tid) {
        Counters& c = cnt[size_t(tid)];
        if (pixels) {
            uint32_t b0 = item * 16, b1 = std::min(n_pixels, b0 + 16);
            for (uint32_t k = b0; k < b1; ++k) {
                uint32_t pix = pixels[k];
                shade_pixel(pix % w, pix / w, k, c);
            }
            return;
        }
        uint32_t ty = item / ntx, tx = item - ty * ntx;
        uint32_t x0 = tx * TS, x1 = std::min(x0 + TS, w);
        uint32_t y0 = ty * TS, y1 = std::min(y0 + TS, h);
        for (uint32_t j = y0; j < y1; ++j)
            for (uint32_t i = x0; i < x1; ++i)
                shade_pixel(i, j, j * w + i, c);
    });
    if (stats) {
        for (auto& c : cnt) {
            stats->rays += c.rays;
            stats->box_tests += c.box;
            stats->prim_tests += c.prim;
            stats->paths += c.paths;
            stats->nonfinite += c.nonfinite;
        }
    }
    return 0;
}

int or_render_preview(const or_scene* s, const fr_render_params* p, uint32_t w, uint32_t h,
                      uint32_t aa_n, float* linear, uint8_t* srgb, uint32_t* hit_ids,
                      int nthreads, or_stats* stats)
{
    if (!s || !p || w == 0 || h == 0 || aa_n == 0 || !linear || !srgb)
        return 1;
    fr_user_camera uc = p->camera;
    uc.f_stop = std::numeric_limits<float>::infinity();  // no depth of field in preview
    const bool sample_aa = (aa_n != 1);
    const M::Cam cam = M::make_camera(to_camera(uc), w, h, p->seed, sample_aa);
    const frm::LightsW lights = world_lights(p->lights, cam);
    const RGB3 bg{p->background_color[0], p->background_color[1], p->background_color[2]};
    const float bg_alpha = p->background_alpha;
    const uint32_t TS = 4;
    const uint32_t ntx = (w + TS - 1) / TS, nty = (h + TS - 1) / TS;
    int nt = nthreads <= 0 ? int(std::max(1u, std::thread::hardware_concurrency())) : nthreads;
    std::vector<Counters> cnt(size_t(std::max(1, nt)));
    const uint32_t ns = aa_n * aa_n;

    parallel_tiles(ntx * nty, nt, [&](uint32_t item, int tid) {
        Counters& c = cnt[size_t(tid)];
        uint32_t ty = item / ntx, tx = item - ty * ntx;
        uint32_t x0 = tx * TS, x1 = std::min(x0 + TS, w);
        uint32_t y0 = ty * TS, y1 = std::min(y0 + TS, h);
        for (uint32_t j = y0; j < y1; ++j)
            for (uint32_t i = x0; i < x1; ++i) {
                float avg[4] = {0, 0, 0, 0};
                for (uint32_t sample = 0; sample < ns; ++sample) {
                    F3 org, dir;
                    M::camera_ray(cam, i, j, sample, org, dir);
                    Hit hh = trace(*s, org, dir, 0.0f, c);
                    c.paths++;
                    RGB3 col = bg;
                    float a = bg_alpha;
                    if (hit_ids) {
                        uint32_t* hp = hit_ids + ((size_t(j) * w + i) * ns + sample) * 2;
                        hp[0] = hh.geom == UINT32_MAX ? 0u : hh.geom + 1u;
                        hp[1] = hh.geom == UINT32_MAX ? 0u : hh.prim;
                    }
                    if (hh.geom != UINT32_MAX) {
                        using frm::dot;
                        const Geom& g = s->geoms[hh.geom];
                        F3 n = frm::div_each(hh.Ng, std::sqrt(dot(hh.Ng, hh.Ng)));
                        F3 v = frm::div_recip(-dir, std::sqrt(dot(dir, dir)));
                        const Mat& m = (hh.d >= g.outline_width) ? g.material : g.outline;
                        if (M::is_solid(m)) {
                            col = M::base_color(m, hh.color);
                        } else {
                            col = RGB3{0, 0, 0};
                            for (unsigned li = 0; li < lights.n; ++li) {
                                F3 l = lights.dir[li];
                                F3 r = -v + (2.0f * n * dot(n, v));
                                float half = lights.theta[li];
                                float cos_half = cosf(half);
                                float ldotr = dot(l, r);
                                if (ldotr < cos_half) {
                                    F3 ax = frm::cross(l, r);
                                    ax = frm::div_recip(ax, sqrtf(dot(ax, ax)));
                                    Quat q = M::from_axis_angle(ax, -acosf(ldotr) + half);
                                    r = M::rotate(q, r);
                                }
                                RGB3 f_d{0, 0, 0}, f_s{0, 0, 0};
                                float ndotl = dot(n, l);
                                if (ndotl >= 0.0f)
                                    f_d = M::brdf_diffuse(m, l, v, n, hh.color) * ndotl;
                                if (dot(n, r) >= 0.0f)
                                    f_s = M::brdf_specular(m, r, v, n, hh.color, half) * dot(n, r);
                                col = col + (f_d + f_s) * float(M_PI) * lights.color[li];
                            }
                        }
                        a = 1.0f;
                    }
                    avg[0] += col.r;
                    avg[1] += col.g;
                    avg[2] += col.b;
                    avg[3] += a;
                }
                float q = 1.0f / float(ns);
                float* px = linear + (size_t(j) * w + i) * 4;
                px[0] = avg[0] * q;
                px[1] = avg[1] * q;
                px[2] = avg[2] * q;
                px[3] = avg[3] * q;
                write_srgb(*p, px, srgb + (size_t(j) * w + i) * 4);
            }
    });
    if (stats) {
        for (auto& c : cnt) {
            stats->rays += c.rays;
            stats->box_tests += c.box;
            stats->prim_tests += c.prim;
            stats->paths += c.paths;
        }
    }
    return 0;
}

int or_prim_hit(const or_scene* s, uint32_t geom, uint32_t prim, const float o[3],
                const float d[3], float tnear, float out[3])
{
    if (!s || geom >= s->geoms.size())
        return 0;
    const Geom& g = s->geoms[geom];
    if (prim >= g.prim_count())
        return 0;
    Hit h;
    h.t = std::numeric_limits<float>::infinity();
    h.geom = UINT32_MAX;
    h.prim = 0;
    h.d = 0;
    F3 oo{o[0], o[1], o[2]}, dd{d[0], d[1], d[2]};
    switch (g.type) {
    case FR_GEOM_SPHERE:
        glue_sphere(g, geom, prim, oo, dd, tnear, h);
        break;
    case FR_GEOM_CYLINDER:
        glue_cylinder(g, geom, prim, oo, dd, tnear, h);
        break;
    case FR_GEOM_POLYHEDRON:
        glue_polyhedron(g, geom, prim, oo, dd, tnear, h);
        break;
    case FR_GEOM_POLYGON:
        glue_polygon(g, geom, prim, oo, dd, tnear, h);
        break;
    default:
        glue_mesh(g, geom, prim, oo, dd, tnear, h);
        break;
    }
    if (h.geom == UINT32_MAX)
        return 0;
    out[0] = h.t;
    out[1] = h.d;
    out[2] = 0.0f;
    return 1;
}

void or_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    frm::Ctr4 c{{ctr[0], ctr[1], ctr[2], ctr[3]}};
    frm::Ctr4 r = frm::philox4x32_10(c, key[0], key[1]);
    for (int k = 0; k < 4; ++k)
        out[k] = r.v[k];
}

float or_u01(uint32_t x) { return frm::u01(x); }

void or_srgb(const float rgba[4], uint8_t out[4]) { M::srgb_encode(rgba, out); }

void or_camera_ray(const fr_user_camera* c, uint32_t w, uint32_t h, uint32_t seed, int sample_aa,
                   uint32_t i, uint32_t j, uint32_t sample, float o[3], float d[3])
{
    M::Cam cam = M::make_camera(to_camera(*c), w, h, seed, sample_aa != 0);
    F3 oo, dd;
    M::camera_ray(cam, i, j, sample, oo, dd);
    o[0] = oo.x;
    o[1] = oo.y;
    o[2] = oo.z;
    d[0] = dd.x;
    d[1] = dd.y;
    d[2] = dd.z;
}

void or_mis_sample(const fr_material* m, const float v[3], const float n[3], uint32_t depth,
                   uint32_t sample, uint32_t key0, uint32_t key1, float out[5])
{
    float factor = 1.0f;
    bool transmit = false;
    F3 l = M::mis_direction(factor, transmit, F3{v[0], v[1], v[2]}, F3{n[0], n[1], n[2]}, depth,
                            sample, key0, key1, to_mat(*m));
    out[0] = l.x;
    out[1] = l.y;
    out[2] = l.z;
    out[3] = factor;
    out[4] = transmit ? 1.0f : 0.0f;
}

void or_brdf(const fr_material* m, const float l[3], const float v[3], const float n[3],
             const float sc[3], float out[3])
{
    RGB3 r = M::brdf(to_mat(*m), F3{l[0], l[1], l[2]}, F3{v[0], v[1], v[2]}, F3{n[0], n[1], n[2]},
                     RGB3{sc[0], sc[1], sc[2]});
    out[0] = r.r;
    out[1] = r.g;
    out[2] = r.b;
}

void or_set_ray_log(float* buffer, uint64_t capacity)
{
    g_ray_log = buffer;
    g_ray_log_cap = buffer ? capacity : 0;
    g_ray_log_n.store(0);
}

uint64_t or_ray_log_count(void) { return g_ray_log_n.load(); }

int or_grid_walk_stats(const or_scene* s, uint32_t sphere_geom, const float* pos, const float* rad,
                       uint32_t n, float cells_per_sphere, const float* rays, uint64_t n_rays,
                       int nthreads, double out[6])
{
    SphereGrid G;
    if (!build_sphere_grid(pos, rad, n, cells_per_sphere, G))
        return 1;
    const uint32_t chunks = uint32_t(std::min<uint64_t>(n_rays, 4096));
    std::vector<uint64_t> cells(chunks, 0), tests(chunks, 0), differ(chunks, 0);
    parallel_tiles(chunks, nthreads, [&](uint32_t ch, int) {
        const uint64_t a = n_rays * ch / chunks, b = n_rays * (ch + 1) / chunks;
        for (uint64_t i = a; i < b; ++i) {
            const float* r = rays + 7 * i;
            const F3 o{r[0], r[1], r[2]}, d{r[3], r[4], r[5]};
            const uint32_t g = walk_sphere_grid(G, o, d, r[6], cells[ch], tests[ch]);
            Counters c;
            const Hit h = trace(*s, o, d, r[6], c);
            const uint32_t b_prim = (h.geom == sphere_geom) ? h.prim : UINT32_MAX;
            if (g != b_prim)
                differ[ch]++;
        }
    });
    double tc = 0, tt = 0, td = 0;
    for (uint32_t ch = 0; ch < chunks; ++ch) {
        tc += double(cells[ch]);
        tt += double(tests[ch]);
        td += double(differ[ch]);
    }
    out[0] = double(n_rays);
    out[1] = n_rays ? tc / double(n_rays) : 0.0;
    out[2] = n_rays ? tt / double(n_rays) : 0.0;
    out[3] = td;
    out[4] = double(G.start.size() - 1);
    out[5] = double(G.refs.size());
    return 0;
}

int or_parts_grid_walk_stats(const or_scene* s, float cells_per_prim, const float* rays,
                             uint64_t n_rays, int nthreads, double out[5])
{
    std::vector<Box> boxes;
    for (const Geom& g : s->geoms) {
        if (!g.enabled || g.prim_count() == 0)
            continue;
        if (g.type == FR_GEOM_MESH) {
            for (uint32_t i = 0; i < g.n; ++i)
                boxes.push_back(instance_box(g, i));
        } else {
            for (uint32_t p = 0; p < g.prim_count(); ++p)
                boxes.push_back(prim_box(g, p));
        }
    }
    CountGrid G;
    if (!build_count_grid(boxes, cells_per_prim, G))
        return 1;
    const uint32_t chunks = uint32_t(std::min<uint64_t>(n_rays, 4096));
    std::vector<uint64_t> cells(chunks, 0), refs(chunks, 0);
    parallel_tiles(chunks, nthreads, [&](uint32_t ch, int) {
        const uint64_t a = n_rays * ch / chunks, b = n_rays * (ch + 1) / chunks;
        for (uint64_t i = a; i < b; ++i) {
            const float* r = rays + 7 * i;
            const F3 o{r[0], r[1], r[2]}, d{r[3], r[4], r[5]};
            Counters c;
            const Hit h = trace(*s, o, d, r[6], c);
            walk_count_grid(G, o, d, h.t, cells[ch], refs[ch]);
        }
    });
    double tc = 0, tr = 0;
    for (uint32_t ch = 0; ch < chunks; ++ch) {
        tc += double(cells[ch]);
        tr += double(refs[ch]);
    }
    out[0] = double(n_rays);
    out[1] = n_rays ? tc / double(n_rays) : 0.0;
    out[2] = n_rays ? tr / double(n_rays) : 0.0;
    out[3] = double(G.count.size());
    out[4] = double(G.refs);
    return 0;
}

}  // extern "C"
