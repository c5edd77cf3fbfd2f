// abi.cu -- the C ABI declared in include/fresnel_b200.h.
//
// Object model (mirrors fresnel/gpu/{Device,Scene,Geometry,Tracer}.cc):
//   fr_device    one CUDA device and one stream; shared BVH-build scratch; an error status word
//   fr_scene     ordered list of geometries (index = geometry id of the hit records) and the
//                device table of their GeomDev records
//   fr_geometry  device copies of the user arrays + the BVH (rebuilt lazily when a geometric
//                array changed, like OptiX's markDirty, fresnel/gpu/Scene.h:64-83)
//   fr_tracer    output buffers (linear RGBA f32, sRGB RGBA8) and the path tracer's per-pixel
//                wavefront state (allocated on first path render)
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "batch.hpp"
#include "bvh.hpp"
#include "fresnel_b200.h"
#include "grid.hpp"
#include "render.hpp"

using namespace fr;

namespace {

thread_local std::string g_error;

fr_status fail(fr_status s, const std::string& msg)
{
    g_error = msg;
    return s;
}

fr_status cuda_fail(cudaError_t e, const char* what)
{
    fr_status s = (e == cudaErrorMemoryAllocation) ? FR_ERR_OUT_OF_MEMORY : FR_ERR_CUDA;
    return fail(s, std::string(what) + ": " + cudaGetErrorString(e));
}

#define FR_CUDA(expr, what)                    \
    do {                                       \
        cudaError_t e_ = (expr);               \
        if (e_ != cudaSuccess)                 \
            return cuda_fail(e_, what);        \
    } while (0)

#define FR_CHECK_NULL(p)                                        \
    do {                                                        \
        if (!(p))                                               \
            return fail(FR_ERR_INVALID, #p " must not be null"); \
    } while (0)

Mat to_mat(const fr_material& m)
{
    Mat r;
    r.solid = m.solid;
    r.color = c3(m.color[0], m.color[1], m.color[2]);
    r.primitive_color_mix = m.primitive_color_mix;
    r.roughness = m.roughness;
    r.specular = m.specular;
    r.metal = m.metal;
    r.spec_trans = m.spec_trans;
    return r;
}

// fresnel::Material(color, solid) defaults (fresnel/common/Material.h:59-64)
fr_material default_material(float r, float g, float b, float solid)
{
    fr_material m;
    m.solid = solid;
    m.color[0] = r;
    m.color[1] = g;
    m.color[2] = b;
    m.primitive_color_mix = 0.0f;
    m.roughness = 0.1f;
    m.specular = 0.5f;
    m.metal = 0.0f;
    m.spec_trans = 0.0f;
    return m;
}

}  // namespace

// Wavefront state of the path tracer (PathState's arrays), grown on demand.
struct PathBuffers {
    DevArray<float4> prim_o, prim_d, ray_o, ray_d, att, result, sample;
    DevArray<uint2> prim_hit, ls_depth, hit;
    DevArray<uint32_t> q0, q1, ctr;
    // slots for n paths; `moved` is set when an array changed address
    cudaError_t reserve(size_t n, bool* moved = nullptr)
    {
        const void* before[13] = {prim_o.ptr, prim_d.ptr, ray_o.ptr, ray_d.ptr, att.ptr,
                                  result.ptr, sample.ptr, prim_hit.ptr, ls_depth.ptr, hit.ptr,
                                  q0.ptr, q1.ptr, ctr.ptr};
        cudaError_t e = cudaSuccess;
        auto r = [&](auto& a, size_t m) {
            if (e == cudaSuccess)
                e = a.reserve(m);
        };
        r(prim_o, n);
        r(prim_d, n);
        r(ray_o, n);
        r(ray_d, n);
        r(att, n);
        r(result, n);
        r(sample, n);
        r(prim_hit, n);
        r(ls_depth, n);
        r(hit, n);
        r(q0, n);
        r(q1, n);
        r(ctr, 4);
        const void* after[13] = {prim_o.ptr, prim_d.ptr, ray_o.ptr, ray_d.ptr, att.ptr,
                                 result.ptr, sample.ptr, prim_hit.ptr, ls_depth.ptr, hit.ptr,
                                 q0.ptr, q1.ptr, ctr.ptr};
        if (moved)
            for (int k = 0; k < 13; ++k)
                if (before[k] != after[k])
                    *moved = true;
        return e;
    }
    PathState state() const
    {
        PathState S;
        S.prim_o = prim_o.ptr;
        S.prim_d = prim_d.ptr;
        S.prim_hit = prim_hit.ptr;
        S.ray_o = ray_o.ptr;
        S.ray_d = ray_d.ptr;
        S.att = att.ptr;
        S.result = result.ptr;
        S.ls_depth = ls_depth.ptr;
        S.hit = hit.ptr;
        S.sample = sample.ptr;
        S.queue[0] = q0.ptr;
        S.queue[1] = q1.ptr;
        S.ctr = ctr.ptr;
        return S;
    }
};

struct fr_tracer;

struct fr_device {
    int ordinal = 0;
    cudaStream_t stream = nullptr;
    int num_sms = 0;
    cudaDeviceProp prop{};
    Scratch scratch;
    BuildParams build;
    LaunchShape shape{};
    DevArray<uint32_t> status;  // traversal error bits
    cudaEvent_t timer[2] = {nullptr, nullptr};
    bool profiling = false;
    size_t path_slots = size_t(128) << 20;  // path slots traced together (144 B each)
    int persistent = 0;                    // persistent traversal kernels for 4-wide trees
    uint32_t tile_log2 = 3;                // primary work tiles of 2^tile_log2 pixels square
    int refit = 0;                         // refit (not rebuild) trees whose primitives moved
    int shade_blocks = 3;                  // shade kernel variant (render.hpp FrameParams)
    int combined = 1;                      // one tree per scene of several geometries
    int packet = 0;                        // warp-cooperative primary traversal
    int refill = 0;                        // extension rays with per-lane refill
    int preview_warp = 1;                  // Preview: one warp per pixel at 32k samples/pixel
    int accel = 2;                         // sphere grid: 0 never, 1 whenever possible, 2 auto
    int fuse_shade = 1;                    // primary rays shaded in the primary pass
    int tail_after = 1;                    // fused bounce launches before the tail kernel (-1: none)
    float grid_cells_per_prim = 1.5f;      // grid cells per sphere
    std::vector<fr_scene*> scenes;         // to mark BVHs stale when a build option changes
    void* static_path = nullptr;           // this device's copy of g_static_path (looked up once)
    PathBuffers path;                      // wavefront state shared by the device's tracers
    uint32_t* h_count = nullptr;           // pinned word for queue-length readbacks
    const fr_tracer* path_owner = nullptr; // tracer of the last path render in `path`
    uint32_t path_k = 0;                   // samples per pixel of that render's last wavefront
    uint32_t path_tile_log2 = 3;           // and its primary tile size
};

struct fr_geometry {
    fr_scene* scene = nullptr;
    int type = 0;
    uint32_t n = 0;        // user primitives (mesh: instances)
    uint32_t n_faces = 0;  // mesh
    uint32_t n_vertices = 0;
    uint32_t n_planes = 0;
    float poly_radius = 0.0f;
    float mesh_radius = 0.0f;  // mesh: the largest vertex distance from the instance origin
    float color_by_face = 0.0f;
    bool enabled = true;
    bool removed = false;
    fr_material material{}, outline{};
    float outline_width = 0.0f;
    DevArray<float> position, radius, color, points, orientation, vertices, planes;
    DevArray<float> angle;         // polygon: [n] radians; orientation holds their quaternions
    DevArray<float4> face_box;     // mesh: per face its local box (lo, hi), padded
    float rounding_radius = 0.0f;  // polygon
    BvhBuffers bvh;
    bool bvh_dirty = true;
    uint64_t gen = 0;        // changes whenever the primitives (or the build options) change
    double last_build_ms = 0.0;
    uint32_t bvh_n = 0;      // primitives of the tree in `bvh`
    BuildParams bvh_bp{};    // and the parameters it was built with

    uint32_t bvh_prims() const { return type == FR_GEOM_MESH ? n * n_faces : n; }
    DevArray<float>* field(int f, size_t& count)
    {
        count = 0;
        switch (f) {
        case FR_FIELD_POSITION:
            if (type == FR_GEOM_CYLINDER)
                return nullptr;
            count = size_t(n) * (type == FR_GEOM_POLYGON ? 2 : 3);
            return &position;
        case FR_FIELD_RADIUS:
            if (type != FR_GEOM_SPHERE && type != FR_GEOM_CYLINDER)
                return nullptr;
            count = n;
            return &radius;
        case FR_FIELD_COLOR:
            count = type == FR_GEOM_CYLINDER ? size_t(n) * 6
                    : type == FR_GEOM_MESH   ? size_t(n_vertices) * 3
                                             : size_t(n) * 3;
            return &color;
        case FR_FIELD_POINTS:
            if (type != FR_GEOM_CYLINDER)
                return nullptr;
            count = size_t(n) * 6;
            return &points;
        case FR_FIELD_ORIENTATION:
            if (type != FR_GEOM_POLYHEDRON && type != FR_GEOM_MESH)
                return nullptr;
            count = size_t(n) * 4;
            return &orientation;
        case FR_FIELD_ANGLE:
            if (type != FR_GEOM_POLYGON)
                return nullptr;
            count = n;
            return &angle;
        }
        return nullptr;
    }
};

struct fr_scene {
    fr_device* dev = nullptr;
    std::vector<fr_geometry*> geoms;
    DevArray<GeomDev> table;
    bool table_dirty = true;
    // one tree over the primitives of all enabled geometries (scenes of 2..MAX_PARTS of them)
    BvhBuffers combined;
    bool use_combined = false;
    std::vector<uint64_t> combined_key;  // (geometry, primitives, generation) per part
    BuildParams combined_bp{};
    // uniform grid over the scene's one sphere geometry (instead of its BVH)
    GridBuffers grid;
    bool use_grid = false;
    std::vector<uint64_t> grid_key;  // (kind, (geometry, primitives, generation) per geometry,
                                     // mode, density) of the grid last tried
    uint32_t grid_geom = 0;          // sphere grid: scene index of its geometry
    GridReport grid_report;
};

struct fr_tracer {
    fr_device* dev = nullptr;
    uint32_t w = 0, h = 0;
    DevArray<float4> linear;
    DevArray<uint32_t> srgb;
    DevArray<uint2> preview_hits;
    DevArray<unsigned long long> stats;
    DevArray<uint32_t> hist;  // Tracer.histogram counts
    uint64_t launches = 0;
    uint64_t builds = 0;
    uint64_t refits = 0;
    uint64_t grid_builds = 0;
    uint32_t last_grid = 0;  // the last render's grid: 0 none, 1 sphere grid, 2 grid over parts
    double build_ms = 0.0;
    // per-kernel timing while profiling: event pairs pending readback, by kernel kind
    std::vector<cudaEvent_t> event_pool;
    struct Pending {
        cudaEvent_t a, b;
        int kind;  // 0 primary, 1 shade, 2 extend
    };
    std::vector<Pending> pending;
    double kernel_ms[3] = {0, 0, 0};
    uint64_t kernel_launches[3] = {0, 0, 0};
    ~fr_tracer()
    {
        for (cudaEvent_t e : event_pool)
            cudaEventDestroy(e);
        for (auto& p : pending) {
            cudaEventDestroy(p.a);
            cudaEventDestroy(p.b);
        }
    }
    cudaEvent_t take_event()
    {
        if (!event_pool.empty()) {
            cudaEvent_t e = event_pool.back();
            event_pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    // call after the stream has been synchronised
    void collect()
    {
        for (auto& p : pending) {
            float ms = 0.0f;
            if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
                kernel_ms[p.kind] += ms;
                kernel_launches[p.kind]++;
            }
            event_pool.push_back(p.a);
            event_pool.push_back(p.b);
        }
        pending.clear();
    }
};

// Many path renders traced together (batch.hpp). Items are queued by fr_batch_add_path and
// traced by fr_batch_render; the tracers and scenes must live until then.
struct fr_batch {
    fr_device* dev = nullptr;
    struct Item {
        fr_tracer* tr;
        fr_scene* sc;
        fr_render_params params;
        uint32_t first, n, light_samples;
    };
    std::vector<Item> items;
    // device-side plan and path state (their addresses are baked into the graph)
    DevArray<WaveJob> jobs;
    DevArray<uint32_t> wave_first, wave_items, wave_pixels;
    DevArray<BatchCtl> ctl;
    PathBuffers path;
    BatchCtl* h_ctl = nullptr;  // pinned
    cudaGraphExec_t exec = nullptr;
    int exec_width = 0;
    uint32_t exec_mask = 0;
    cudaStream_t capture = nullptr;
    fr_batch_stats stats{};
    ~fr_batch()
    {
        if (exec)
            cudaGraphExecDestroy(exec);
        if (capture)
            cudaStreamDestroy(capture);
        if (h_ctl)
            cudaFreeHost(h_ctl);
    }
};

namespace {

uint64_t g_generation = 0;  // source of fr_geometry::gen values (never repeats)

void mark_moved(fr_geometry* g)
{
    g->bvh_dirty = true;
    g->gen = ++g_generation;
}

fr_status use_device(const fr_device* d)
{
    FR_CUDA(cudaSetDevice(d->ordinal), "cudaSetDevice");
    return FR_OK;
}

fr_status alloc_field(fr_geometry* g, int f)
{
    size_t count;
    DevArray<float>* a = g->field(f, count);
    if (!a || count == 0)
        return FR_OK;
    FR_CUDA(a->reserve(count), "allocating a geometry array");
    FR_CUDA(cudaMemsetAsync(a->ptr, 0, count * sizeof(float), g->scene->dev->stream),
            "clearing a geometry array");
    return FR_OK;
}

fr_status new_geometry(fr_scene* scene, int type, uint32_t n, fr_geometry** out,
                       fr_geometry** made)
{
    FR_CHECK_NULL(scene);
    FR_CHECK_NULL(out);
    fr_geometry* g = new (std::nothrow) fr_geometry();
    if (!g)
        return fail(FR_ERR_OUT_OF_MEMORY, "out of host memory");
    g->scene = scene;
    g->type = type;
    g->n = n;
    g->material = default_material(1, 0, 1, 0);
    g->outline = default_material(0, 0, 0, 1);
    *made = g;
    return FR_OK;
}

fr_status finish_geometry(fr_geometry* g, fr_geometry** out)
{
    fr_status s = use_device(g->scene->dev);
    if (s != FR_OK) {
        delete g;
        return s;
    }
    for (int f = 0; f <= FR_FIELD_ANGLE; ++f) {
        if ((s = alloc_field(g, f)) != FR_OK) {
            delete g;
            return s;
        }
    }
    g->scene->geoms.push_back(g);
    g->scene->table_dirty = true;
    g->gen = ++g_generation;
    *out = g;
    return FR_OK;
}

BuildInput build_input(const fr_geometry* g)
{
    BuildInput in;
    in.type = g->type;
    in.position = g->position.ptr;
    in.radius = g->radius.ptr;
    in.points = g->points.ptr;
    in.orientation = g->orientation.ptr;
    in.vertices = g->vertices.ptr;
    in.n_faces = g->n_faces;
    in.poly_radius = g->poly_radius;
    in.instances = 0;
    return in;
}

bool same_params(const BuildParams& a, const BuildParams& b)
{
    return a.builder == b.builder && a.width == b.width && a.leaf_max == b.leaf_max &&
           a.c_trav == b.c_trav && a.c_isect == b.c_isect;
}

// The geometries a combined tree would cover (empty if the scene traces per-geometry trees:
// combining is off, the trees are binary, or fewer than 2 or more than MAX_PARTS geometries
// have primitives) and the key that identifies their current contents.
std::vector<fr_geometry*> combined_parts(const fr_scene* sc, std::vector<uint64_t>& key)
{
    std::vector<fr_geometry*> parts;
    key.clear();
    const fr_device* dev = sc->dev;
    if (!dev->combined || dev->build.width != 4)
        return parts;
    for (fr_geometry* g : sc->geoms)
        if (!g->removed && g->enabled && g->bvh_prims() > 0)
            parts.push_back(g);
    if (parts.size() < 2 || parts.size() > size_t(MAX_PARTS)) {
        parts.clear();
        return parts;
    }
    for (fr_geometry* g : parts) {
        key.push_back(reinterpret_cast<uintptr_t>(g));
        key.push_back(g->bvh_prims());
        key.push_back(g->gen);
    }
    return parts;
}

// What a grid may replace (nothing when the device option accel is 0): the tree of the scene's
// only enabled geometry when it holds spheres (kind 1, a sphere grid; gi receives its scene
// index), else the trees of all its enabled geometries, at most MAX_PARTS (kind 2, a grid over
// their primitives, a mesh by instance; parts receives them in scene order).  The automatic
// mode (accel 2) applies the grid's own rules (clustering, sparseness) to both kinds: measured
// against the trees, spheres and bonds of 1e4 to 2e6 primitives traced 1.5x to 1.9x faster
// through a grid over parts, the mixed scene (spheres, bonds, cubes, icosahedra) 1.15x, 10k
// icosahedra alone 1.66x, 1080 polygons with 400 spheres 1.38x.  key identifies what a grid
// build depends on.  Returns the kind, or 0 when no grid applies.
int grid_candidate(const fr_scene* sc, std::vector<uint64_t>& key, uint32_t& gi,
                   std::vector<fr_geometry*>* parts = nullptr)
{
    key.clear();
    if (parts)
        parts->clear();
    const fr_device* dev = sc->dev;
    if (dev->accel == 0)
        return 0;
    std::vector<fr_geometry*> on;
    uint32_t first = 0;
    for (uint32_t i = 0; i < sc->geoms.size(); ++i) {
        fr_geometry* g = sc->geoms[i];
        if (g->removed || !g->enabled || g->bvh_prims() == 0)
            continue;
        if (on.empty())
            first = i;
        on.push_back(g);
    }
    if (on.empty() || on.size() > size_t(MAX_PARTS))
        return 0;
    if (sc->geoms.size() >= (size_t(1) << PART_TYPE_SHIFT))
        return 0;  // a grid over parts keeps geometry indices below 2^24
    const int kind = (on.size() == 1 && on[0]->type == FR_GEOM_SPHERE) ? 1 : 2;
    uint32_t density_bits;
    std::memcpy(&density_bits, &dev->grid_cells_per_prim, sizeof(density_bits));
    key.push_back(uint64_t(kind));
    for (fr_geometry* g : on) {
        key.push_back(reinterpret_cast<uintptr_t>(g));
        key.push_back(g->bvh_prims());
        key.push_back(g->gen);
    }
    key.push_back(uint64_t(dev->accel));
    key.push_back(density_bits);
    gi = first;
    if (parts)
        *parts = on;
    return kind;
}

// Whether prepare_scene would build anything.
bool scene_needs_build(const fr_scene* sc)
{
    std::vector<uint64_t> key;
    uint32_t gi = 0;
    if (grid_candidate(sc, key, gi) != 0) {
        if (key != sc->grid_key)
            return true;
        if (sc->use_grid)
            return false;
    }
    if (!combined_parts(sc, key).empty())
        return !sc->use_combined || key != sc->combined_key;
    for (fr_geometry* g : sc->geoms)
        if (!g->removed && g->bvh_dirty)
            return true;
    return false;
}

fr_status check_build_status(fr_device* dev)
{
    uint32_t stw = 0;
    FR_CUDA(cudaMemcpy(&stw, dev->status.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost),
            "reading the build status");
    if (stw & ERR_BUILD) {
        cudaMemset(dev->status.ptr, 0, sizeof(uint32_t));
        return fail(FR_ERR_DEVICE_LIMIT, "BVH construction produced an inconsistent tree");
    }
    return FR_OK;
}

// The build input over the primitives of `parts` (at most MAX_PARTS geometries of sc); n
// receives their number.  mesh_instances: a mesh contributes one primitive per instance (grids
// over parts) rather than one per triangle (trees).
PartsInput parts_input(const fr_scene* sc, const std::vector<fr_geometry*>& parts, uint32_t& n,
                       bool mesh_instances = false)
{
    PartsInput in;
    std::memset(&in, 0, sizeof(in));
    n = 0;
    in.n_parts = uint32_t(parts.size());
    for (uint32_t p = 0; p < in.n_parts; ++p) {
        fr_geometry* g = parts[p];
        in.part[p] = build_input(g);
        const bool inst = mesh_instances && g->type == FR_GEOM_MESH;
        in.part[p].instances = inst ? 1 : 0;
        in.first[p] = n;
        uint32_t gi = 0;
        while (sc->geoms[gi] != g)
            ++gi;
        in.geom[p] = gi;
        n += inst ? g->n : g->bvh_prims();
    }
    in.first[in.n_parts] = n;
    return in;
}

// Build (or refit) the scene's combined tree over `parts`.
fr_status build_combined(fr_scene* sc, fr_tracer* tr, const std::vector<fr_geometry*>& parts,
                         const std::vector<uint64_t>& key)
{
    fr_device* dev = sc->dev;
    uint32_t n = 0;
    const PartsInput in = parts_input(sc, parts, n);
    const BuildParams& bp = dev->build;
    // same geometries and counts, other contents: the topology can be kept
    bool same_layout = sc->combined.n_nodes > 0 && sc->combined_key.size() == key.size() &&
                       same_params(sc->combined_bp, bp);
    for (size_t i = 0; same_layout && i < key.size(); i += 3)
        same_layout = sc->combined_key[i] == key[i] && sc->combined_key[i + 1] == key[i + 1];
    const bool refit = dev->refit && same_layout;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, dev->stream);
    cudaError_t e = cudaErrorInvalidValue;
    if (refit)
        e = refit_bvh(in, n, bp, sc->combined, dev->scratch, dev->status.ptr, dev->stream);
    if (!refit || e == cudaErrorInvalidValue)
        e = build_bvh(in, n, bp, sc->combined, dev->scratch, dev->status.ptr, dev->stream);
    cudaEventRecord(e1, dev->stream);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess)
        return cuda_fail(e, "building a BVH");
    fr_status s = check_build_status(dev);
    if (s != FR_OK) {
        sc->combined.n_nodes = 0;
        sc->combined.n_nodes4 = 0;
        sc->use_combined = false;
        sc->combined_key.clear();
        return s;
    }
    if (tr) {
        tr->builds++;
        if (refit)
            tr->refits++;
        tr->build_ms = ms;
    }
    sc->combined_key = key;
    sc->combined_bp = bp;
    sc->use_combined = true;
    return FR_OK;
}

// Build (or decline) the grid grid_candidate chose, of kind 1 (the sphere geometry parts[0], scene
// index gi) or 2 (over `parts`), when its inputs changed.
fr_status prepare_grid(fr_scene* sc, fr_tracer* tr, int kind, uint32_t gi,
                       const std::vector<fr_geometry*>& parts, const std::vector<uint64_t>& key)
{
    fr_device* dev = sc->dev;
    GridParams gp;
    gp.mode = dev->accel;
    gp.cells_per_prim = dev->grid_cells_per_prim;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, dev->stream);
    cudaError_t e;
    if (kind == 1) {
        const fr_geometry* g = parts[0];
        e = build_grid(g->position.ptr, g->radius.ptr, g->n, gp, sc->grid, dev->scratch,
                       dev->stream, sc->grid_report);
    } else {
        uint32_t n = 0;
        const PartsInput in = parts_input(sc, parts, n, true);
        e = build_grid(in, n, gp, sc->grid, dev->scratch, dev->stream, sc->grid_report);
    }
    cudaEventRecord(e1, dev->stream);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) {
        sc->use_grid = false;
        sc->grid_key.clear();
        return cuda_fail(e, "building a sphere grid");
    }
    sc->grid_key = key;
    sc->grid_geom = gi;
    sc->use_grid = sc->grid_report.built;
    GridBuffers& G = sc->grid;
    if (!sc->use_grid || G.parts) {  // free the arrays the grid in use does not read
        G.ref_sphere.release();
    }
    if (!sc->use_grid || !G.parts) {
        G.ref_data.release();
        G.ref_geom.release();
    }
    if (!sc->use_grid) {  // BVHs serve this scene
        G.box_lo.release();  // (kept otherwise, as the other build temporaries, for rebuilds)
        G.box_hi.release();
        G.cell_start.release();
        G.ref_prim.release();
    } else if (tr) {
        tr->grid_builds++;
        tr->build_ms = ms;
    }
    return FR_OK;
}

// Build the stale acceleration structures (grid or BVHs) and refresh the device geometry table.
fr_status prepare_scene(fr_scene* sc, fr_tracer* tr)
{
    fr_device* dev = sc->dev;
    std::vector<uint64_t> key;
    uint32_t gi = 0;
    std::vector<fr_geometry*> grid_parts;
    const int kind = grid_candidate(sc, key, gi, &grid_parts);
    if (kind == 0) {
        sc->use_grid = false;
        sc->grid_key.clear();
    } else if (key != sc->grid_key) {
        fr_status s = prepare_grid(sc, tr, kind, gi, grid_parts, key);
        if (s != FR_OK)
            return s;
    }
    const std::vector<fr_geometry*> parts =
        sc->use_grid ? std::vector<fr_geometry*>() : combined_parts(sc, key);
    if (!parts.empty()) {
        if (!sc->use_combined || key != sc->combined_key) {
            fr_status s = build_combined(sc, tr, parts, key);
            if (s != FR_OK)
                return s;
        }
    } else {
        sc->use_combined = false;
    }
    for (fr_geometry* g : sc->geoms) {
        if (sc->use_grid || sc->use_combined || g->removed || !g->bvh_dirty)
            continue;
        BuildInput in = build_input(g);
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, dev->stream);
        const BuildParams& bp = dev->build;
        const bool refit = dev->refit && g->bvh.n_nodes > 0 && g->bvh_n == g->bvh_prims() &&
                           same_params(g->bvh_bp, bp);
        cudaError_t e = cudaErrorInvalidValue;
        if (refit)
            e = refit_bvh(in, g->bvh_prims(), bp, g->bvh, dev->scratch, dev->status.ptr,
                          dev->stream);
        if (!refit || e == cudaErrorInvalidValue)
            e = build_bvh(in, g->bvh_prims(), bp, g->bvh, dev->scratch, dev->status.ptr,
                          dev->stream);
        cudaEventRecord(e1, dev->stream);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (e != cudaSuccess)
            return cuda_fail(e, "building a BVH");
        g->last_build_ms = ms;
        {
            uint32_t stw = 0;
            FR_CUDA(cudaMemcpy(&stw, dev->status.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost),
                    "reading the build status");
            if (stw & ERR_BUILD) {
                cudaMemset(dev->status.ptr, 0, sizeof(uint32_t));
                g->bvh.n_nodes = 0;
                g->bvh.n_nodes4 = 0;
                return fail(FR_ERR_DEVICE_LIMIT, "BVH construction produced an inconsistent tree");
            }
        }
        if (tr) {
            tr->builds++;
            if (refit)
                tr->refits++;
            tr->build_ms = ms;
        }
        g->bvh_n = g->bvh_prims();
        g->bvh_bp = bp;
        g->bvh_dirty = false;
        sc->table_dirty = true;
    }
    if (sc->table_dirty) {
        std::vector<GeomDev> host(sc->geoms.size());
        for (size_t i = 0; i < sc->geoms.size(); ++i) {
            fr_geometry* g = sc->geoms[i];
            GeomDev& d = host[i];
            std::memset(&d, 0, sizeof(d));
            d.type = g->type;
            d.enabled = (g->enabled && !g->removed) ? 1 : 0;
            d.n_prims = g->bvh_prims();
            d.n_nodes = g->bvh.n_nodes;
            d.n_nodes4 = g->bvh.n_nodes4;
            d.nodes = g->bvh.nodes.ptr;
            d.nodes4 = g->bvh.nodes4.ptr;
            d.leaf_data = g->bvh.leaf_data.ptr;
            d.order = g->bvh.order.ptr;
            d.position = g->position.ptr;
            d.radius = g->radius.ptr;
            d.color = g->color.ptr;
            d.points = g->points.ptr;
            d.orientation = g->orientation.ptr;
            d.vertices = g->vertices.ptr;
            d.planes = g->planes.ptr;
            d.n_faces = g->n_faces;
            d.n_planes = g->n_planes;
            d.n_vertices = g->type == FR_GEOM_POLYGON ? g->n_vertices : 0u;
            d.rounding_radius = g->rounding_radius;
            d.bound_radius = g->type == FR_GEOM_MESH ? g->mesh_radius : g->poly_radius;
            d.face_box = g->face_box.ptr;
            d.color_by_face = g->color_by_face;
            d.outline_width = g->outline_width;
            d.material = to_mat(g->material);
            d.outline = to_mat(g->outline);
        }
        if (!host.empty()) {
            FR_CUDA(sc->table.reserve(host.size()), "allocating the geometry table");
            FR_CUDA(cudaMemcpyAsync(sc->table.ptr, host.data(), host.size() * sizeof(GeomDev),
                                    cudaMemcpyHostToDevice, dev->stream),
                    "uploading the geometry table");
            FR_CUDA(cudaStreamSynchronize(dev->stream), "uploading the geometry table");
        }
        sc->table_dirty = false;
    }
    return FR_OK;
}

FrameParams frame_params(fr_tracer* tr, fr_scene* sc, const fr_render_params* p, bool preview,
                         uint32_t aa_n)
{
    FrameParams P;
    std::memset(&P, 0, sizeof(P));
    P.scene.geoms = sc->table.ptr;
    P.scene.n_geoms = uint32_t(sc->geoms.size());
    P.scene.status = sc->dev->status.ptr;
    P.type_mask = 0;
    P.bvh_width = 2;
    P.persistent = sc->dev->persistent;
    P.refill_geom = -1;  // no tree the refill kernel can walk (set below when there is one)
    if (sc->use_grid) {
        const GridBuffers& G = sc->grid;
        GridDev& d = P.scene.grid;
        d.n_cells = G.n_cells;
        d.nx = G.dims[0];
        d.ny = G.dims[1];
        d.nz = G.dims[2];
        d.lox = G.lo[0];
        d.loy = G.lo[1];
        d.loz = G.lo[2];
        d.hix = G.hi[0];
        d.hiy = G.hi[1];
        d.hiz = G.hi[2];
        d.hx = G.cell[0];
        d.hy = G.cell[1];
        d.hz = G.cell[2];
        d.ihx = 1.0f / G.cell[0];
        d.ihy = 1.0f / G.cell[1];
        d.ihz = 1.0f / G.cell[2];
        d.geom = sc->grid_geom;
        d.cell_start = G.cell_start.ptr;
        d.ref_sphere = G.ref_sphere.ptr;
        d.ref_prim = G.ref_prim.ptr;
        d.parts = G.parts ? 1u : 0u;
        if (G.parts) {  // the references read as a combined tree's leaf slots
            for (fr_geometry* g : sc->geoms)
                if (g->enabled && !g->removed && g->bvh_prims() > 0)
                    P.type_mask |= 1u << g->type;
            P.scene.n_prims = G.n_refs;
            P.scene.leaf_data = G.ref_data.ptr;
            P.scene.leaf_geom = G.ref_geom.ptr;
            P.scene.order = G.ref_prim.ptr;
        } else {
            P.type_mask = 1u << FR_GEOM_SPHERE;
        }
        P.bvh_width = 4;
        P.persistent = 0;  // the persistent and packet kernels walk trees
    } else if (sc->use_combined && sc->combined.n_nodes4 > 0) {
        for (fr_geometry* g : sc->geoms)
            if (g->enabled && !g->removed && g->bvh_prims() > 0)
                P.type_mask |= 1u << g->type;
        P.bvh_width = 4;
        P.persistent = 0;  // the persistent kernels step through per-geometry trees
        P.scene.n_nodes4 = sc->combined.n_nodes4;
        uint32_t n = 0;
        for (size_t i = 1; i < sc->combined_key.size(); i += 3)
            n += uint32_t(sc->combined_key[i]);
        P.scene.n_prims = n;
        P.scene.nodes4 = sc->combined.nodes4.ptr;
        P.scene.leaf_data = sc->combined.leaf_data.ptr;
        P.scene.leaf_geom = sc->combined.leaf_geom.ptr;
        P.scene.order = sc->combined.order.ptr;
        P.refill_geom = -2;
    } else {
        bool all4 = true;
        for (fr_geometry* g : sc->geoms) {
            if (!g->enabled || g->removed || g->bvh.n_nodes == 0)
                continue;
            P.type_mask |= 1u << g->type;
            all4 = all4 && g->bvh.n_nodes4 > 0;
        }
        if (P.type_mask != 0 && all4)
            P.bvh_width = 4;
        int only = -1, n_enabled = 0;
        for (size_t i = 0; i < sc->geoms.size(); ++i) {
            const fr_geometry* g = sc->geoms[i];
            if (g->enabled && !g->removed && g->bvh.n_nodes > 0) {
                only = int(i);
                ++n_enabled;
            }
        }
        if (n_enabled == 1)
            P.refill_geom = only;
    }
    P.tile_log2 = sc->dev->tile_log2;
    P.shade_blocks = sc->dev->shade_blocks;
    P.packet = sc->use_grid ? 0 : sc->dev->packet;
    P.refill = sc->dev->refill;
    P.preview_warp = sc->dev->preview_warp;
    tr->last_grid = sc->use_grid ? (sc->grid.parts ? 2u : 1u) : 0u;
    const fr_user_camera& c = p->camera;
    float f_stop = preview ? std::numeric_limits<float>::infinity() : c.f_stop;  // no depth of field in preview
    bool sample_aa = preview ? (aa_n != 1) : true;
    P.cam = make_camera(v3(c.position[0], c.position[1], c.position[2]),
                        v3(c.look_at[0], c.look_at[1], c.look_at[2]),
                        v3(c.up[0], c.up[1], c.up[2]), c.h, c.f, f_stop, c.focus_distance, c.model,
                        tr->w, tr->h, p->seed, sample_aa);
    V3 dirs[4];
    C3 cols[4];
    float th[4];
    uint32_t n = p->lights.n > 4 ? 4 : p->lights.n;
    for (uint32_t i = 0; i < 4; ++i) {
        dirs[i] = v3(p->lights.direction[i][0], p->lights.direction[i][1], p->lights.direction[i][2]);
        cols[i] = c3(p->lights.color[i][0], p->lights.color[i][1], p->lights.color[i][2]);
        th[i] = p->lights.theta[i];
    }
    P.lights = lights_to_world(dirs, cols, th, n, P.cam);
    P.bg = c3(p->background_color[0], p->background_color[1], p->background_color[2]);
    P.bg_alpha = p->background_alpha;
    P.w = tr->w;
    P.h = tr->h;
    P.highlight = p->highlight_warning;
    P.hl_color = c3(p->highlight_color[0], p->highlight_color[1], p->highlight_color[2]);
    P.linear = tr->linear.ptr;
    P.srgb = tr->srgb.ptr;
    P.stats = tr->stats.ptr;
    return P;
}

fr_status check_status(fr_device* dev)
{
    uint32_t st = 0;
    FR_CUDA(cudaMemcpyAsync(&st, dev->status.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                            dev->stream),
            "reading the device status");
    FR_CUDA(cudaStreamSynchronize(dev->stream), "render");
    if (st) {
        FR_CUDA(cudaMemsetAsync(dev->status.ptr, 0, sizeof(uint32_t), dev->stream), "status reset");
        return fail(FR_ERR_DEVICE_LIMIT,
                    (st & ERR_STACK_OVERFLOW) ? "BVH traversal stack overflow (tree too deep)"
                    : (st & ERR_BAD_NODE)     ? "BVH traversal met an out-of-range node"
                    : (st & ERR_KERNEL)       ? "a kernel met an acceleration structure it lacks"
                                              : "BVH traversal iteration cap reached");
    }
    return FR_OK;
}

fr_status alloc_outputs(fr_tracer* tr, uint32_t w, uint32_t h)
{
    size_t n = size_t(w) * h;
    FR_CUDA(tr->linear.reserve(n), "allocating the linear output");
    FR_CUDA(tr->srgb.reserve(n), "allocating the sRGB output");
    FR_CUDA(cudaMemsetAsync(tr->linear.ptr, 0, n * sizeof(float4), tr->dev->stream), "clear");
    FR_CUDA(cudaMemsetAsync(tr->srgb.ptr, 0, n * sizeof(uint32_t), tr->dev->stream), "clear");
    tr->w = w;
    tr->h = h;
    return FR_OK;
}

// Path slots per sample of a w x h image: the pixels of its 8x8 tiles (edge tiles padded).
size_t padded_pixels(uint32_t w, uint32_t h, uint32_t tl)
{
    const size_t t = size_t(1) << tl;
    return ((w + t - 1) / t) * ((h + t - 1) / t) * t * t;
}

// Samples traced together: a batch of K samples of every pixel fills about
// dev->path_slots slots (about 144 bytes each).
uint32_t batch_size(const fr_tracer* tr, uint32_t remaining)
{
    size_t wh = padded_pixels(tr->w, tr->h, tr->dev->tile_log2);
    size_t k = tr->dev->path_slots / wh;
    if (k < 1)
        k = 1;
    if (k > 4096)
        k = 4096;  // the primary kernel's grid z dimension
    if (k > remaining)
        k = remaining;
    return uint32_t(k);
}

fr_status alloc_path_state(fr_tracer* tr, uint32_t batch)
{
    size_t n = padded_pixels(tr->w, tr->h, tr->dev->tile_log2) * batch;
    FR_CUDA(tr->dev->path.reserve(n), "allocating the path state");
    return FR_OK;
}

fr_status check_params(const fr_tracer* tr, const fr_scene* sc, const fr_render_params* p)
{
    FR_CHECK_NULL(tr);
    FR_CHECK_NULL(sc);
    FR_CHECK_NULL(p);
    if (sc->dev != tr->dev)
        return fail(FR_ERR_INVALID, "Scene and Tracer devices do not match");
    return FR_OK;
}

}  // namespace

// =============================================================================================
extern "C" {

const char* fr_last_error(void) { return g_error.c_str(); }
int fr_abi_version(void) { return FR_ABI_VERSION; }

fr_status fr_get_num_available_devices(int* n)
{
    FR_CHECK_NULL(n);
    *n = 0;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        cudaGetLastError();
        return FR_OK;  // no driver or no device: zero GPUs
    }
    for (int i = 0; i < count; ++i) {
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, i) == cudaSuccess && prop.major == 10)
            ++*n;
    }
    return FR_OK;
}

fr_status fr_get_all_gpus(char* buf, size_t cap)
{
    FR_CHECK_NULL(buf);
    std::string s;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        cudaGetLastError();
        count = 0;
    }
    for (int i = 0; i < count; ++i) {
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, i) == cudaSuccess && prop.major == 10) {
            s += "[" + std::to_string(i) + "]: " + prop.name + " " +
                 std::to_string(prop.multiProcessorCount) + " SM_" + std::to_string(prop.major) +
                 "." + std::to_string(prop.minor) + "\n";
        }
    }
    if (cap == 0)
        return fail(FR_ERR_INVALID, "buffer capacity is zero");
    std::snprintf(buf, cap, "%s", s.c_str());
    return FR_OK;
}

fr_status fr_device_create(int n, fr_device** out)
{
    FR_CHECK_NULL(out);
    *out = nullptr;
    int avail = 0;
    fr_get_num_available_devices(&avail);
    if (avail == 0)
        return fail(FR_ERR_UNSUPPORTED, "No GPUs are available (an sm_100 device is required)");
    if (n == 0 || n < -1)
        return fail(FR_ERR_INVALID, "the number of GPUs must be positive or -1");
    int count = 0;
    FR_CUDA(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
    int ordinal = -1;
    for (int i = 0; i < count && ordinal < 0; ++i) {
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, i) == cudaSuccess && prop.major == 10)
            ordinal = i;
    }
    fr_device* d = new (std::nothrow) fr_device();
    if (!d)
        return fail(FR_ERR_OUT_OF_MEMORY, "out of host memory");
    d->ordinal = ordinal;
    cudaError_t e = cudaSetDevice(ordinal);
    if (e == cudaSuccess)
        e = cudaGetDeviceProperties(&d->prop, ordinal);
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = d->status.reserve(1);
    if (e == cudaSuccess)
        e = cudaMemset(d->status.ptr, 0, sizeof(uint32_t));
    if (e == cudaSuccess)
        e = cudaMallocHost((void**)&d->h_count, 4 * sizeof(uint32_t));
    if (e != cudaSuccess) {
        delete d;
        return cuda_fail(e, "creating the device");
    }
    d->num_sms = d->prop.multiProcessorCount;
    d->shape = path_launch_shape(d->num_sms);
    *out = d;
    return FR_OK;
}

fr_status fr_device_destroy(fr_device* d)
{
    if (!d)
        return FR_OK;
    cudaSetDevice(d->ordinal);
    if (d->stream) {
        cudaStreamSynchronize(d->stream);
        cudaStreamDestroy(d->stream);
    }
    for (int k = 0; k < 2; ++k)
        if (d->timer[k])
            cudaEventDestroy(d->timer[k]);
    if (d->h_count)
        cudaFreeHost(d->h_count);
    delete d;
    return FR_OK;
}

fr_status fr_device_describe(const fr_device* d, char* buf, size_t cap)
{
    FR_CHECK_NULL(d);
    FR_CHECK_NULL(buf);
    if (cap == 0)
        return fail(FR_ERR_INVALID, "buffer capacity is zero");
    std::snprintf(buf, cap, "Enabled GPUs:\n[%d]: %s %d SM_%d.%d\n", d->ordinal, d->prop.name,
                  d->num_sms, d->prop.major, d->prop.minor);
    return FR_OK;
}

fr_status fr_device_synchronize(fr_device* d)
{
    FR_CHECK_NULL(d);
    FR_CUDA(cudaSetDevice(d->ordinal), "cudaSetDevice");
    FR_CUDA(cudaStreamSynchronize(d->stream), "cudaStreamSynchronize");
    return FR_OK;
}

fr_status fr_device_timer_start(fr_device* d)
{
    FR_CHECK_NULL(d);
    FR_CUDA(cudaSetDevice(d->ordinal), "cudaSetDevice");
    for (int k = 0; k < 2; ++k)
        if (!d->timer[k])
            FR_CUDA(cudaEventCreate(&d->timer[k]), "creating a timer event");
    FR_CUDA(cudaEventRecord(d->timer[0], d->stream), "recording the timer start");
    return FR_OK;
}

fr_status fr_device_timer_stop(fr_device* d, float* ms)
{
    FR_CHECK_NULL(d);
    FR_CHECK_NULL(ms);
    if (!d->timer[0] || !d->timer[1])
        return fail(FR_ERR_STATE, "the timer was not started");
    FR_CUDA(cudaSetDevice(d->ordinal), "cudaSetDevice");
    FR_CUDA(cudaEventRecord(d->timer[1], d->stream), "recording the timer stop");
    FR_CUDA(cudaEventSynchronize(d->timer[1]), "waiting for the timer stop");
    FR_CUDA(cudaEventElapsedTime(ms, d->timer[0], d->timer[1]), "reading the timer");
    return FR_OK;
}

fr_status fr_device_set_option(fr_device* d, const char* name, double value)
{
    FR_CHECK_NULL(d);
    FR_CHECK_NULL(name);
    std::string n(name);
    bool tree = false;
    if (n == "bvh_width") {
        if (value != 2.0 && value != 4.0)
            return fail(FR_ERR_INVALID, "bvh_width must be 2 or 4");
        tree = d->build.width != int(value);
        d->build.width = int(value);
    } else if (n == "leaf_max") {
        if (!(value >= 1.0 && value <= 16.0))
            return fail(FR_ERR_INVALID, "leaf_max must be in [1, 16]");
        tree = d->build.leaf_max != int(value);
        d->build.leaf_max = int(value);
    } else if (n == "c_trav") {
        if (!(value > 0.0 && value < 100.0))
            return fail(FR_ERR_INVALID, "c_trav must be in (0, 100)");
        tree = d->build.c_trav != float(value);
        d->build.c_trav = float(value);
    } else if (n == "refill") {
        if (value != 0.0 && value != 1.0)
            return fail(FR_ERR_INVALID, "refill must be 0 or 1");
        d->refill = int(value);
    } else if (n == "packet") {
        if (value != 0.0 && value != 1.0)
            return fail(FR_ERR_INVALID, "packet must be 0 or 1");
        d->packet = int(value);
    } else if (n == "combined") {
        if (value != 0.0 && value != 1.0)
            return fail(FR_ERR_INVALID, "combined must be 0 or 1");
        tree = d->combined != int(value);
        d->combined = int(value);
    } else if (n == "shade_blocks") {
        if (value != 0.0 && value != 3.0 && value != 4.0)
            return fail(FR_ERR_INVALID, "shade_blocks must be 0, 3 or 4");
        d->shade_blocks = int(value);
    } else if (n == "refit") {
        if (value != 0.0 && value != 1.0)
            return fail(FR_ERR_INVALID, "refit must be 0 or 1");
        d->refit = int(value);
    } else if (n == "tile") {
        if (value != 4.0 && value != 8.0 && value != 16.0)
            return fail(FR_ERR_INVALID, "tile must be 4, 8 or 16");
        d->tile_log2 = value == 4.0 ? 2u : value == 8.0 ? 3u : 4u;
    } else if (n == "builder") {
        if (value != 0.0 && value != 1.0)
            return fail(FR_ERR_INVALID, "builder must be 0 (LBVH) or 1 (PLOC)");
        tree = d->build.builder != int(value);
        d->build.builder = int(value);
    } else if (n == "persistent") {
        if (value != 0.0 && value != 1.0)
            return fail(FR_ERR_INVALID, "persistent must be 0 or 1");
        d->persistent = int(value);
    } else if (n == "fuse_shade") {
        if (!(value == 0.0 || value == 1.0 || value == 2.0))
            return fail(FR_ERR_INVALID, "fuse_shade must be 0, 1 or 2");
        d->fuse_shade = int(value);
    } else if (n == "preview_warp") {
        if (value != 0.0 && value != 1.0)
            return fail(FR_ERR_INVALID, "preview_warp must be 0 or 1");
        d->preview_warp = int(value);
    } else if (n == "tail") {
        if (!(value >= -1.0 && value <= 64.0 && value == double(int(value))))
            return fail(FR_ERR_INVALID, "tail must be an integer in [-1, 64]");
        d->tail_after = int(value);
    } else if (n == "accel") {
        if (!(value == 0.0 || value == 1.0 || value == 2.0))
            return fail(FR_ERR_INVALID, "accel must be 0 (BVH), 1 (sphere grid) or 2 (automatic)");
        d->accel = int(value);
    } else if (n == "grid_density") {
        if (!(value > 0.0 && value <= 64.0))
            return fail(FR_ERR_INVALID, "grid_density must be in (0, 64]");
        d->grid_cells_per_prim = float(value);
    } else if (n == "path_slots") {
        if (!(value >= 1.0 && value <= 1e9))
            return fail(FR_ERR_INVALID, "path_slots must be in [1, 1e9]");
        d->path_slots = size_t(value);
    } else {
        return fail(FR_ERR_INVALID, "unknown option " + n);
    }
    if (tree)
        for (fr_scene* sc : d->scenes)
            for (fr_geometry* g : sc->geoms)
                mark_moved(g);
    return FR_OK;
}

fr_status fr_device_get_option(const fr_device* d, const char* name, double* value)
{
    FR_CHECK_NULL(d);
    FR_CHECK_NULL(name);
    FR_CHECK_NULL(value);
    std::string n(name);
    if (n == "bvh_width")
        *value = d->build.width;
    else if (n == "leaf_max")
        *value = d->build.leaf_max;
    else if (n == "c_trav")
        *value = d->build.c_trav;
    else if (n == "path_slots")
        *value = double(d->path_slots);
    else if (n == "accel")
        *value = d->accel;
    else if (n == "tail")
        *value = d->tail_after;
    else if (n == "preview_warp")
        *value = d->preview_warp;
    else if (n == "fuse_shade")
        *value = d->fuse_shade;
    else if (n == "grid_density")
        *value = d->grid_cells_per_prim;
    else if (n == "builder")
        *value = d->build.builder;
    else if (n == "tile")
        *value = double(1u << d->tile_log2);
    else if (n == "refit")
        *value = d->refit;
    else if (n == "shade_blocks")
        *value = d->shade_blocks;
    else if (n == "combined")
        *value = d->combined;
    else if (n == "packet")
        *value = d->packet;
    else if (n == "refill")
        *value = d->refill;
    else if (n == "persistent")
        *value = d->persistent;
    else
        return fail(FR_ERR_INVALID, "unknown option " + n);
    return FR_OK;
}

fr_status fr_device_set_profiling(fr_device* d, int enable)
{
    FR_CHECK_NULL(d);
    d->profiling = enable != 0;
    return FR_OK;
}

// ---------------------------------------------------------------------------------------------
fr_status fr_scene_create(fr_device* dev, fr_scene** out)
{
    FR_CHECK_NULL(dev);
    FR_CHECK_NULL(out);
    fr_scene* s = new (std::nothrow) fr_scene();
    if (!s)
        return fail(FR_ERR_OUT_OF_MEMORY, "out of host memory");
    s->dev = dev;
    dev->scenes.push_back(s);
    *out = s;
    return FR_OK;
}

fr_status fr_scene_destroy(fr_scene* s)
{
    if (!s)
        return FR_OK;
    auto& v = s->dev->scenes;
    for (size_t i = 0; i < v.size(); ++i)
        if (v[i] == s) {
            v.erase(v.begin() + long(i));
            break;
        }
    cudaSetDevice(s->dev->ordinal);
    cudaStreamSynchronize(s->dev->stream);
    for (fr_geometry* g : s->geoms)
        g->scene = nullptr;  // geometries outlive nothing: the owner destroys them explicitly
    delete s;
    return FR_OK;
}

fr_status fr_scene_build(fr_scene* s)
{
    FR_CHECK_NULL(s);
    fr_status st = use_device(s->dev);
    if (st != FR_OK)
        return st;
    return prepare_scene(s, nullptr);
}

// ---------------------------------------------------------------------------------------------
fr_status fr_geometry_create_sphere(fr_scene* scene, uint32_t n, fr_geometry** out)
{
    fr_geometry* g = nullptr;
    fr_status s = new_geometry(scene, FR_GEOM_SPHERE, n, out, &g);
    return s != FR_OK ? s : finish_geometry(g, out);
}

fr_status fr_geometry_create_cylinder(fr_scene* scene, uint32_t n, fr_geometry** out)
{
    fr_geometry* g = nullptr;
    fr_status s = new_geometry(scene, FR_GEOM_CYLINDER, n, out, &g);
    return s != FR_OK ? s : finish_geometry(g, out);
}

fr_status fr_geometry_create_polyhedron(fr_scene* scene, const float* origins, const float* normals,
                                        const float* colors, uint32_t n_planes, uint32_t n,
                                        float radius, fr_geometry** out)
{
    FR_CHECK_NULL(origins);
    FR_CHECK_NULL(normals);
    FR_CHECK_NULL(colors);
    if (n_planes == 0)
        return fail(FR_ERR_INVALID, "a convex polyhedron needs at least one plane");
    fr_geometry* g = nullptr;
    fr_status s = new_geometry(scene, FR_GEOM_POLYHEDRON, n, out, &g);
    if (s != FR_OK)
        return s;
    g->n_planes = n_planes;
    g->poly_radius = radius;
    // [origin, unit normal, colour] per plane; normals scaled by 1/|n|
    // (fresnel/cpu/GeometryConvexPolyhedron.cc:81-91)
    std::vector<float> pl(size_t(n_planes) * 9);
    for (uint32_t i = 0; i < n_planes; ++i) {
        V3 nn = v3(normals[3 * i], normals[3 * i + 1], normals[3 * i + 2]);
        nn = div_recip(nn, sqrtf(dot(nn, nn)));
        float* q = pl.data() + 9 * i;
        q[0] = origins[3 * i];
        q[1] = origins[3 * i + 1];
        q[2] = origins[3 * i + 2];
        q[3] = nn.x;
        q[4] = nn.y;
        q[5] = nn.z;
        q[6] = colors[3 * i];
        q[7] = colors[3 * i + 1];
        q[8] = colors[3 * i + 2];
    }
    cudaError_t e = use_device(scene->dev) == FR_OK ? g->planes.reserve(pl.size()) : cudaErrorUnknown;
    if (e == cudaSuccess)
        e = cudaMemcpy(g->planes.ptr, pl.data(), pl.size() * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        delete g;
        return cuda_fail(e, "uploading polyhedron planes");
    }
    return finish_geometry(g, out);
}

fr_status fr_geometry_create_mesh(fr_scene* scene, const float* vertices, uint32_t n_vertices,
                                  uint32_t n, fr_geometry** out)
{
    FR_CHECK_NULL(vertices);
    if (n_vertices % 3 != 0)
        return fail(FR_ERR_INVALID, "the number of triangle vertices must be a multiple of three.");
    fr_geometry* g = nullptr;
    fr_status s = new_geometry(scene, FR_GEOM_MESH, n, out, &g);
    if (s != FR_OK)
        return s;
    g->n_vertices = n_vertices;
    g->n_faces = n_vertices / 3;
    double r2 = 0.0;  // a NaN vertex is passed over: its triangles have no valid box anyway
    for (uint32_t i = 0; i < n_vertices; ++i) {
        const double x = vertices[3 * size_t(i)], y = vertices[3 * size_t(i) + 1],
                     z = vertices[3 * size_t(i) + 2];
        const double q = x * x + y * y + z * z;
        if (q > r2)
            r2 = q;
    }
    g->mesh_radius = float(std::sqrt(r2) * (1.0 + 1e-6));
    // each face's box in the instance frame, padded like the tree builds' boxes (a filter in
    // front of the face's test in grids over parts; a face with a NaN vertex gets an empty box)
    std::vector<float4> boxes(2 * size_t(g->n_faces));
    for (uint32_t f = 0; f < g->n_faces; ++f) {
        float lo[3], hi[3];
        bool ok = true;
        for (int k = 0; k < 3; ++k) {
            lo[k] = INFINITY;
            hi[k] = -INFINITY;
            for (int v = 0; v < 3; ++v) {
                const float x = vertices[3 * (3 * size_t(f) + v) + k];
                ok = ok && std::isfinite(x);
                lo[k] = std::min(lo[k], x);
                hi[k] = std::max(hi[k], x);
            }
        }
        float scale = 0.0f, ext = 0.0f;
        for (int k = 0; k < 3; ++k) {
            scale = std::max(scale, std::max(std::fabs(lo[k]), std::fabs(hi[k])));
            ext += hi[k] - lo[k];
        }
        const float pad = 1e-5f * scale + 1e-6f * ext + 1e-30f;
        if (!ok) {
            boxes[2 * size_t(f)] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
            boxes[2 * size_t(f) + 1] = make_float4(-1.0f, -1.0f, -1.0f, 0.0f);
        } else {
            boxes[2 * size_t(f)] = make_float4(lo[0] - pad, lo[1] - pad, lo[2] - pad, 0.0f);
            boxes[2 * size_t(f) + 1] = make_float4(hi[0] + pad, hi[1] + pad, hi[2] + pad, 0.0f);
        }
    }
    cudaError_t e = use_device(scene->dev) == FR_OK ? g->vertices.reserve(size_t(n_vertices) * 3)
                                                    : cudaErrorUnknown;
    if (e == cudaSuccess && n_vertices)
        e = cudaMemcpy(g->vertices.ptr, vertices, size_t(n_vertices) * 3 * sizeof(float),
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess && g->n_faces)
        e = g->face_box.reserve(boxes.size());
    if (e == cudaSuccess && g->n_faces)
        e = cudaMemcpy(g->face_box.ptr, boxes.data(), boxes.size() * sizeof(float4),
                       cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        delete g;
        return cuda_fail(e, "uploading mesh vertices");
    }
    return finish_geometry(g, out);
}

fr_status fr_scene_get_accel(const fr_scene* sc, int* grid, char* reason, size_t cap)
{
    FR_CHECK_NULL(sc);
    FR_CHECK_NULL(grid);
    *grid = sc->use_grid ? (sc->grid.parts ? 2 : 1) : 0;
    if (reason && cap) {
        const char* r = (!sc->use_grid && !sc->grid_key.empty()) ? sc->grid_report.reason : "";
        std::snprintf(reason, cap, "%s", r);
    }
    return FR_OK;
}

fr_status fr_geometry_create_polygon(fr_scene* scene, const float* vertices, uint32_t n_vertices,
                                     float rounding_radius, uint32_t n, fr_geometry** out)
{
    if (n_vertices)
        FR_CHECK_NULL(vertices);
    fr_geometry* g = nullptr;
    fr_status s = new_geometry(scene, FR_GEOM_POLYGON, n, out, &g);
    if (s != FR_OK)
        return s;
    g->n_vertices = n_vertices;
    g->rounding_radius = rounding_radius;
    // bounding radius: the farthest vertex plus the rounding (fresnel/cpu/GeometryPolygon.cc:58-67)
    float r = 0.0f;
    for (uint32_t i = 0; i < n_vertices; ++i) {
        const float x = vertices[2 * i], y = vertices[2 * i + 1];
        r = std::max(r, sqrtf(x * x + y * y));
    }
    g->poly_radius = r + rounding_radius;
    // every angle starts at 0: its quaternion is the identity
    std::vector<float> q(size_t(n) * 4, 0.0f);
    for (uint32_t i = 0; i < n; ++i)
        q[4 * size_t(i)] = 1.0f;
    cudaError_t e = use_device(scene->dev) == FR_OK ? g->vertices.reserve(size_t(n_vertices) * 2)
                                                    : cudaErrorUnknown;
    if (e == cudaSuccess && n_vertices)
        e = cudaMemcpy(g->vertices.ptr, vertices, size_t(n_vertices) * 2 * sizeof(float),
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = g->orientation.reserve(q.size());
    if (e == cudaSuccess && n)
        e = cudaMemcpy(g->orientation.ptr, q.data(), q.size() * sizeof(float),
                       cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        delete g;
        return cuda_fail(e, "uploading polygon vertices");
    }
    return finish_geometry(g, out);
}

fr_status fr_geometry_get_radius(const fr_geometry* g, float* radius)
{
    FR_CHECK_NULL(g);
    FR_CHECK_NULL(radius);
    if (g->type != FR_GEOM_POLYGON)
        return fail(FR_ERR_INVALID, "only polygon geometries have a radius");
    *radius = g->poly_radius;
    return FR_OK;
}

fr_status fr_geometry_destroy(fr_geometry* g)
{
    if (!g)
        return FR_OK;
    if (g->scene) {
        cudaSetDevice(g->scene->dev->ordinal);
        cudaStreamSynchronize(g->scene->dev->stream);
        auto& v = g->scene->geoms;
        for (size_t i = 0; i < v.size(); ++i)
            if (v[i] == g) {
                v.erase(v.begin() + long(i));
                break;
            }
        g->scene->table_dirty = true;
    }
    delete g;
    return FR_OK;
}

fr_status fr_geometry_field_size(const fr_geometry* g, int field, size_t* nbytes)
{
    FR_CHECK_NULL(g);
    FR_CHECK_NULL(nbytes);
    size_t count = 0;
    const_cast<fr_geometry*>(g)->field(field, count);
    *nbytes = count * sizeof(float);
    return FR_OK;
}

fr_status fr_geometry_write(fr_geometry* g, int field, const void* host, size_t offset,
                            size_t nbytes)
{
    FR_CHECK_NULL(g);
    FR_CHECK_NULL(host);
    if (!g->scene)
        return fail(FR_ERR_STATE, "the geometry's scene was destroyed");
    size_t count = 0;
    DevArray<float>* a = g->field(field, count);
    if (!a)
        return fail(FR_ERR_INVALID, "this geometry has no such array");
    if (offset + nbytes > count * sizeof(float))
        return fail(FR_ERR_INVALID, "write past the end of the array");
    if (nbytes == 0)
        return FR_OK;
    fr_status s = use_device(g->scene->dev);
    if (s != FR_OK)
        return s;
    if (field == FR_FIELD_ANGLE && (offset % sizeof(float) != 0 || nbytes % sizeof(float) != 0))
        return fail(FR_ERR_INVALID, "angle writes must cover whole floats");
    FR_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(a->ptr) + offset, host, nbytes,
                            cudaMemcpyHostToDevice, g->scene->dev->stream),
            "uploading a geometry array");
    if (field == FR_FIELD_ANGLE) {
        // the rotation quaternion of each angle, computed here on the host as the reference's
        // CPU path does, quat::fromAxisAngle((0, 0, 1), angle) (fresnel/cpu/GeometryPolygon.cc:
        // 153, fresnel/common/VectorMath.h:924-928 with cosf/sinf)
        const float* a_host = static_cast<const float*>(host);
        const size_t first = offset / sizeof(float), count = nbytes / sizeof(float);
        std::vector<float> q(count * 4);
        for (size_t k = 0; k < count; ++k) {
            const float half = a_host[k] / 2.0f;
            const float sh = sinf(half);
            q[4 * k] = cosf(half);
            q[4 * k + 1] = sh * 0.0f;
            q[4 * k + 2] = sh * 0.0f;
            q[4 * k + 3] = sh * 1.0f;
        }
        FR_CUDA(cudaMemcpyAsync(g->orientation.ptr + 4 * first, q.data(), q.size() * sizeof(float),
                                cudaMemcpyHostToDevice, g->scene->dev->stream),
                "uploading polygon rotations");
    }
    FR_CUDA(cudaStreamSynchronize(g->scene->dev->stream), "uploading a geometry array");
    if (field != FR_FIELD_COLOR)
        mark_moved(g);  // colours do not move primitives
    return FR_OK;
}

fr_status fr_geometry_read(fr_geometry* g, int field, void* host, size_t offset, size_t nbytes)
{
    FR_CHECK_NULL(g);
    FR_CHECK_NULL(host);
    if (!g->scene)
        return fail(FR_ERR_STATE, "the geometry's scene was destroyed");
    size_t count = 0;
    DevArray<float>* a = g->field(field, count);
    if (!a)
        return fail(FR_ERR_INVALID, "this geometry has no such array");
    if (offset + nbytes > count * sizeof(float))
        return fail(FR_ERR_INVALID, "read past the end of the array");
    if (nbytes == 0)
        return FR_OK;
    fr_status s = use_device(g->scene->dev);
    if (s != FR_OK)
        return s;
    FR_CUDA(cudaMemcpyAsync(host, reinterpret_cast<const char*>(a->ptr) + offset, nbytes,
                            cudaMemcpyDeviceToHost, g->scene->dev->stream),
            "downloading a geometry array");
    FR_CUDA(cudaStreamSynchronize(g->scene->dev->stream), "downloading a geometry array");
    return FR_OK;
}

fr_status fr_geometry_set_enabled(fr_geometry* g, int enabled)
{
    FR_CHECK_NULL(g);
    if (g->removed || !g->scene)
        return fail(FR_ERR_STATE, enabled ? "Cannot enable inactive Geometry"
                                          : "Cannot disable inactive Geometry");
    g->enabled = enabled != 0;
    g->scene->table_dirty = true;
    return FR_OK;
}

fr_status fr_geometry_remove(fr_geometry* g)
{
    FR_CHECK_NULL(g);
    if (!g->removed && g->scene) {
        g->removed = true;
        g->scene->table_dirty = true;
    }
    return FR_OK;
}

fr_status fr_geometry_set_material(fr_geometry* g, const fr_material* m, const fr_material* outline,
                                   float outline_width)
{
    FR_CHECK_NULL(g);
    if (m)
        g->material = *m;
    if (outline)
        g->outline = *outline;
    g->outline_width = outline_width;
    if (g->scene)
        g->scene->table_dirty = true;
    return FR_OK;
}

fr_status fr_geometry_set_color_by_face(fr_geometry* g, float f)
{
    FR_CHECK_NULL(g);
    g->color_by_face = f;
    if (g->scene)
        g->scene->table_dirty = true;
    return FR_OK;
}

fr_status fr_geometry_update(fr_geometry* g)
{
    FR_CHECK_NULL(g);
    mark_moved(g);
    return FR_OK;
}

// ---------------------------------------------------------------------------------------------
fr_status fr_tracer_create(fr_device* dev, uint32_t w, uint32_t h, fr_tracer** out)
{
    FR_CHECK_NULL(dev);
    FR_CHECK_NULL(out);
    *out = nullptr;
    if (w == 0 || h == 0)
        return fail(FR_ERR_INVALID, "Invalid dimensions");
    fr_status s = use_device(dev);
    if (s != FR_OK)
        return s;
    fr_tracer* t = new (std::nothrow) fr_tracer();
    if (!t)
        return fail(FR_ERR_OUT_OF_MEMORY, "out of host memory");
    t->dev = dev;
    cudaError_t e = t->stats.reserve(8);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(t->stats.ptr, 0, 8 * sizeof(unsigned long long), dev->stream);
    if (e != cudaSuccess) {
        delete t;
        return cuda_fail(e, "creating a tracer");
    }
    if ((s = alloc_outputs(t, w, h)) != FR_OK) {
        delete t;
        return s;
    }
    *out = t;
    return FR_OK;
}

fr_status fr_tracer_destroy(fr_tracer* t)
{
    if (!t)
        return FR_OK;
    cudaSetDevice(t->dev->ordinal);
    cudaStreamSynchronize(t->dev->stream);
    if (t->dev->path_owner == t)
        t->dev->path_owner = nullptr;
    delete t;
    return FR_OK;
}

fr_status fr_tracer_resize(fr_tracer* t, uint32_t w, uint32_t h)
{
    FR_CHECK_NULL(t);
    if (w == 0 || h == 0)
        return fail(FR_ERR_INVALID, "Invalid dimensions");
    fr_status s = use_device(t->dev);
    if (s != FR_OK)
        return s;
    s = alloc_outputs(t, w, h);
    if (s != FR_OK)
        return s;
    FR_CUDA(cudaStreamSynchronize(t->dev->stream), "resize");
    return FR_OK;
}

fr_status fr_tracer_clear(fr_tracer* t)
{
    FR_CHECK_NULL(t);
    fr_status s = use_device(t->dev);
    if (s != FR_OK)
        return s;
    size_t n = size_t(t->w) * t->h;
    FR_CUDA(cudaMemsetAsync(t->linear.ptr, 0, n * sizeof(float4), t->dev->stream), "clear");
    FR_CUDA(cudaMemsetAsync(t->srgb.ptr, 0, n * sizeof(uint32_t), t->dev->stream), "clear");
    FR_CUDA(cudaStreamSynchronize(t->dev->stream), "clear");
    return FR_OK;
}

fr_status fr_tracer_render_path(fr_tracer* t, fr_scene* sc, const fr_render_params* p,
                                uint32_t first_sample, uint32_t n_render, uint32_t light_samples)
{
    fr_status s = check_params(t, sc, p);
    if (s != FR_OK)
        return s;
    if (light_samples == 0)
        return fail(FR_ERR_INVALID, "light_samples must be positive");
    if (first_sample == 0)
        return fail(FR_ERR_INVALID, "sample numbers start at 1");
    if ((s = use_device(t->dev)) != FR_OK)
        return s;
    if ((s = prepare_scene(sc, t)) != FR_OK)
        return s;
    uint32_t batch = batch_size(t, n_render);
    if ((s = alloc_path_state(t, batch)) != FR_OK)
        return s;
    FrameParams P = frame_params(t, sc, p, false, 1);
    P.light_samples = light_samples;
    PathState S = t->dev->path.state();
    t->dev->path_owner = t;
    cudaStream_t st = t->dev->stream;
    FR_CUDA(cudaMemsetAsync(S.ctr, 0, 4 * sizeof(uint32_t), st), "clearing queue lengths");
    const int CHECK_EVERY = 8;
    const int MAX_ITER = 1 << 20;
    const bool prof = t->dev->profiling;
    auto timed = [&](int kind, auto&& launch) {
        if (!prof) {
            launch();
            return;
        }
        cudaEvent_t a = t->take_event(), b = t->take_event();
        cudaEventRecord(a, st);
        launch();
        cudaEventRecord(b, st);
        t->pending.push_back({a, b, kind});
    };
    for (uint32_t done = 0; done < n_render;) {
        P.n_samples = first_sample + done;
        P.batch = batch < n_render - done ? batch : n_render - done;
        // primary rays shaded at once: the first shade pass is folded into the primary pass
        const bool fused = t->dev->fuse_shade && !P.persistent && !P.packet;
        if (fused) {
            FR_CUDA(cudaMemsetAsync(S.ctr, 0, 4 * sizeof(uint32_t), st), "clearing the queues");
            timed(0, [&] { launch_path_primary_shade(P, S, st); });
        } else {
            FR_CUDA(cudaMemsetAsync(S.ctr + 3, 0, sizeof(uint32_t), st), "clearing a counter");
            timed(0, [&] { launch_path_primary(P, S, t->dev->shape, st); });
        }
        t->launches++;
        int it = 0;
        // bounces fused too: by default for sphere-grid scenes only (a BVH walk in a kernel
        // compiled for 3 blocks per SM is slower than the separate passes)
        const bool bounces =
            fused && (t->dev->fuse_shade == 2 || (P.scene.grid.n_cells != 0 && !P.refill));
        if (bounces && t->dev->tail_after >= 0) {
            // a few bounce launches while the queues are long, then every path's remaining
            // bounces in one launch: the wavefront needs no queue-length read-back
            for (int b = 0; b < t->dev->tail_after; ++b, ++it) {
                FR_CUDA(cudaMemsetAsync(S.ctr + ((it & 1) ^ 1), 0, sizeof(uint32_t), st),
                        "clearing a queue");
                FR_CUDA(cudaMemsetAsync(S.ctr + 2, 0, sizeof(uint32_t), st), "clearing a counter");
                timed(2, [&] { launch_path_bounce(P, S, it, t->dev->shape, st); });
                t->launches += 1;
            }
            FR_CUDA(cudaMemsetAsync(S.ctr + 2, 0, sizeof(uint32_t), st), "clearing a counter");
            timed(2, [&] { launch_path_tail(P, S, it, t->dev->shape, st); });
            t->launches += 1;
            FR_CUDA(cudaGetLastError(), "launching the path tracer");
            launch_path_fold(P, S, st);
            t->launches++;
            t->dev->path_k = P.batch;
            t->dev->path_tile_log2 = P.tile_log2;
            done += P.batch;
            continue;
        }
        while (true) {
            for (int b = 0; b < CHECK_EVERY; ++b, ++it) {
                if (bounces) {
                    // trace and shade queue it&1 into queue (it&1)^1, cleared first with the
                    // work counter
                    FR_CUDA(cudaMemsetAsync(S.ctr + ((it & 1) ^ 1), 0, sizeof(uint32_t), st),
                            "clearing a queue");
                    FR_CUDA(cudaMemsetAsync(S.ctr + 2, 0, sizeof(uint32_t), st),
                            "clearing a counter");
                    timed(2, [&] { launch_path_bounce(P, S, it, t->dev->shape, st); });
                    t->launches += 1;
                    continue;
                }
                if (!(fused && it == 0))
                    timed(1, [&] { launch_path_shade(P, S, it, t->dev->shape, st); });
                timed(2, [&] { launch_path_extend(P, S, it, t->dev->shape, st); });
                t->launches += 2;
            }
            FR_CUDA(cudaGetLastError(), "launching the path tracer");
            // the output queue of the last shade pass (or of the last bounce)
            const int last_q = bounces ? (((it - 1) & 1) ^ 1) : ((it - 1) & 1);
            FR_CUDA(cudaMemcpyAsync(t->dev->h_count, S.ctr + last_q, sizeof(uint32_t),
                                    cudaMemcpyDeviceToHost, st),
                    "reading the queue length");
            FR_CUDA(cudaStreamSynchronize(st), "path tracer");
            t->collect();
            if (*t->dev->h_count == 0)
                break;
            if (it >= MAX_ITER)
                return fail(FR_ERR_DEVICE_LIMIT, "path tracer exceeded the bounce iteration cap");
        }
        launch_path_fold(P, S, st);
        t->launches++;
        t->dev->path_k = P.batch;
        t->dev->path_tile_log2 = P.tile_log2;
        done += P.batch;
    }
    s = check_status(t->dev);
    t->collect();  // the stream is synchronised: profiling events of the tail launches are done
    return s;
}

// ---------------------------------------------------------------------------------------------
// Allocation-free path render.  The wavefront state of fr_tracer_render_path_static lives in
// g_static_path: 16 bytes of queue/work counters, then each per-slot array sized for
// FR_STATIC_PATH_SLOTS slots at a 256-byte aligned offset.  A __device__ array is created with
// the module (one copy per GPU), so the call allocates nothing.
}  // extern "C"

namespace {

constexpr size_t kStaticSlots = FR_STATIC_PATH_SLOTS;
constexpr size_t kStaticBytes = 256 + kStaticSlots * (7 * sizeof(float4) + 3 * sizeof(uint2) +
                                                      2 * sizeof(uint32_t));

__device__ __align__(256) unsigned char g_static_path[kStaticBytes];

// Carves the per-slot arrays out of the static block; false if they would not fit.
bool static_path_state(void* base, PathState& S)
{
    ScratchLayout L;
    uint32_t* ctr = L.take<uint32_t>(4);
    S.prim_o = L.take<float4>(kStaticSlots);
    S.prim_d = L.take<float4>(kStaticSlots);
    S.ray_o = L.take<float4>(kStaticSlots);
    S.ray_d = L.take<float4>(kStaticSlots);
    S.att = L.take<float4>(kStaticSlots);
    S.result = L.take<float4>(kStaticSlots);
    S.sample = L.take<float4>(kStaticSlots);
    S.prim_hit = L.take<uint2>(kStaticSlots);
    S.ls_depth = L.take<uint2>(kStaticSlots);
    S.hit = L.take<uint2>(kStaticSlots);
    S.queue[0] = L.take<uint32_t>(kStaticSlots);
    S.queue[1] = L.take<uint32_t>(kStaticSlots);
    L.bind(base);
    S.ctr = L.at(ctr);
    S.prim_o = L.at(S.prim_o);
    S.prim_d = L.at(S.prim_d);
    S.ray_o = L.at(S.ray_o);
    S.ray_d = L.at(S.ray_d);
    S.att = L.at(S.att);
    S.result = L.at(S.result);
    S.sample = L.at(S.sample);
    S.prim_hit = L.at(S.prim_hit);
    S.ls_depth = L.at(S.ls_depth);
    S.hit = L.at(S.hit);
    S.queue[0] = L.at(S.queue[0]);
    S.queue[1] = L.at(S.queue[1]);
    return L.bytes <= kStaticBytes;
}

// With a multiple of 64 slots every per-slot array ends on a 256-byte boundary, so the only
// padding is the 240 bytes after the counters and the layout is exactly kStaticBytes.
static_assert(kStaticSlots % 64 == 0, "static path layout");

}  // namespace

extern "C" {

fr_status fr_tracer_render_path_static(fr_tracer* t, fr_scene* sc, const fr_render_params* p,
                                       uint32_t first_sample, uint32_t n_render,
                                       uint32_t light_samples)
{
    fr_status s = check_params(t, sc, p);
    if (s != FR_OK)
        return s;
    if (light_samples == 0)
        return fail(FR_ERR_INVALID, "light_samples must be positive");
    if (first_sample == 0)
        return fail(FR_ERR_INVALID, "sample numbers start at 1");
    const size_t wh = padded_pixels(t->w, t->h, t->dev->tile_log2);
    if (wh > kStaticSlots)
        return fail(FR_ERR_INVALID, "image of " + std::to_string(t->w) + "x" +
                                        std::to_string(t->h) +
                                        " pixels exceeds the allocation-free render's limit of " +
                                        std::to_string(kStaticSlots) +
                                        " pixels (counted in whole primary tiles)");
    if (scene_needs_build(sc))
        return fail(FR_ERR_STATE, "the allocation-free render needs a built scene: call "
                                  "fr_scene_build after changing geometry");
    if (sc->table_dirty)
        return fail(FR_ERR_STATE, "the allocation-free render needs a built scene: call "
                                  "fr_scene_build after changing geometry");
    if ((s = use_device(t->dev)) != FR_OK)
        return s;
    if (!t->dev->static_path) {
        void* base = nullptr;
        FR_CUDA(cudaGetSymbolAddress(&base, g_static_path), "looking up the static path state");
        t->dev->static_path = base;
    }
    // The device's allocating path state may still hold this tracer's earlier render; its
    // primary hits do not describe the image this call writes.
    if (t->dev->path_owner == t)
        t->dev->path_owner = nullptr;
    if (n_render == 0)
        return FR_OK;
    PathState S;
    if (!static_path_state(t->dev->static_path, S))
        return fail(FR_ERR_STATE, "static path state layout exceeds its array");
    size_t k = kStaticSlots / wh;
    if (k > 4096)
        k = 4096;  // the primary kernel's grid z dimension
    const uint32_t batch = uint32_t(k);
    FrameParams P = frame_params(t, sc, p, false, 1);
    P.light_samples = light_samples;
    cudaStream_t st = t->dev->stream;
    FR_CUDA(cudaMemsetAsync(S.ctr, 0, 4 * sizeof(uint32_t), st), "clearing queue lengths");
    const int CHECK_EVERY = 8;
    const int MAX_ITER = 1 << 20;
    for (uint32_t done = 0; done < n_render;) {
        P.n_samples = first_sample + done;
        P.batch = batch < n_render - done ? batch : n_render - done;
        FR_CUDA(cudaMemsetAsync(S.ctr + 3, 0, sizeof(uint32_t), st), "clearing a counter");
        launch_path_primary(P, S, t->dev->shape, st);
        t->launches++;
        int it = 0;
        while (true) {
            for (int b = 0; b < CHECK_EVERY; ++b, ++it) {
                launch_path_shade(P, S, it, t->dev->shape, st);
                launch_path_extend(P, S, it, t->dev->shape, st);
                t->launches += 2;
            }
            FR_CUDA(cudaGetLastError(), "launching the path tracer");
            FR_CUDA(cudaMemcpyAsync(t->dev->h_count, S.ctr + ((it - 1) & 1), sizeof(uint32_t),
                                    cudaMemcpyDeviceToHost, st),
                    "reading the queue length");
            FR_CUDA(cudaStreamSynchronize(st), "path tracer");
            if (*t->dev->h_count == 0)
                break;
            if (it >= MAX_ITER)
                return fail(FR_ERR_DEVICE_LIMIT, "path tracer exceeded the bounce iteration cap");
        }
        launch_path_fold(P, S, st);
        t->launches++;
        done += P.batch;
    }
    return check_status(t->dev);
}

fr_status fr_tracer_render_preview(fr_tracer* t, fr_scene* sc, const fr_render_params* p,
                                   uint32_t aa_n, uint32_t* hit_ids)
{
    fr_status s = check_params(t, sc, p);
    if (s != FR_OK)
        return s;
    if (aa_n == 0)
        return fail(FR_ERR_INVALID, "the anti-aliasing level must be positive");
    if ((s = use_device(t->dev)) != FR_OK)
        return s;
    if ((s = prepare_scene(sc, t)) != FR_OK)
        return s;
    FrameParams P = frame_params(t, sc, p, true, aa_n);
    size_t nh = size_t(t->w) * t->h * aa_n * aa_n;
    uint2* hits = nullptr;
    if (hit_ids) {
        FR_CUDA(t->preview_hits.reserve(nh), "allocating the hit-id buffer");
        hits = t->preview_hits.ptr;
    }
    launch_preview(P, aa_n, hits, t->dev->stream);
    t->launches++;
    FR_CUDA(cudaGetLastError(), "launching the preview tracer");
    if (hit_ids)
        FR_CUDA(cudaMemcpyAsync(hit_ids, hits, nh * sizeof(uint2), cudaMemcpyDeviceToHost,
                                t->dev->stream),
                "downloading hit ids");
    return check_status(t->dev);
}

fr_status fr_tracer_read_linear(fr_tracer* t, float* host, size_t nbytes)
{
    FR_CHECK_NULL(t);
    FR_CHECK_NULL(host);
    if (nbytes != size_t(t->w) * t->h * sizeof(float4))
        return fail(FR_ERR_INVALID, "linear output size mismatch");
    fr_status s = use_device(t->dev);
    if (s != FR_OK)
        return s;
    FR_CUDA(cudaMemcpyAsync(host, t->linear.ptr, nbytes, cudaMemcpyDeviceToHost, t->dev->stream),
            "downloading the linear output");
    FR_CUDA(cudaStreamSynchronize(t->dev->stream), "downloading the linear output");
    return FR_OK;
}

fr_status fr_tracer_read_srgb(fr_tracer* t, uint8_t* host, size_t nbytes)
{
    FR_CHECK_NULL(t);
    FR_CHECK_NULL(host);
    if (nbytes != size_t(t->w) * t->h * 4)
        return fail(FR_ERR_INVALID, "sRGB output size mismatch");
    fr_status s = use_device(t->dev);
    if (s != FR_OK)
        return s;
    FR_CUDA(cudaMemcpyAsync(host, t->srgb.ptr, nbytes, cudaMemcpyDeviceToHost, t->dev->stream),
            "downloading the sRGB output");
    FR_CUDA(cudaStreamSynchronize(t->dev->stream), "downloading the sRGB output");
    return FR_OK;
}

fr_status fr_tracer_histogram(fr_tracer* t, uint32_t* counts, size_t nbytes)
{
    FR_CHECK_NULL(t);
    FR_CHECK_NULL(counts);
    if (nbytes != size_t(HIST_BINS) * 4 * sizeof(uint32_t))
        return fail(FR_ERR_INVALID, "histogram size mismatch: " + std::to_string(HIST_BINS) +
                                        " x 4 counts of 4 bytes");
    fr_status s = use_device(t->dev);
    if (s != FR_OK)
        return s;
    FR_CUDA(t->hist.reserve(size_t(HIST_BINS) * 4), "allocating the histogram");
    cudaStream_t st = t->dev->stream;
    FR_CUDA(cudaMemsetAsync(t->hist.ptr, 0, nbytes, st), "clearing the histogram");
    launch_histogram(t->linear.ptr, t->w * t->h, t->hist.ptr, t->dev->num_sms, st);
    FR_CUDA(cudaGetLastError(), "launching the histogram");
    FR_CUDA(cudaMemcpyAsync(counts, t->hist.ptr, nbytes, cudaMemcpyDeviceToHost, st),
            "downloading the histogram");
    FR_CUDA(cudaStreamSynchronize(st), "histogram");
    return FR_OK;
}

fr_status fr_host_alloc(size_t nbytes, void** out)
{
    FR_CHECK_NULL(out);
    *out = nullptr;
    if (nbytes == 0)
        return fail(FR_ERR_INVALID, "host allocation of 0 bytes");
    FR_CUDA(cudaHostAlloc(out, nbytes, cudaHostAllocPortable), "allocating page-locked host memory");
    return FR_OK;
}

fr_status fr_host_free(void* host)
{
    if (host)
        FR_CUDA(cudaFreeHost(host), "freeing page-locked host memory");
    return FR_OK;
}

fr_status fr_tracer_write_linear(fr_tracer* t, const float* host, size_t nbytes)
{
    FR_CHECK_NULL(t);
    FR_CHECK_NULL(host);
    if (nbytes != size_t(t->w) * t->h * sizeof(float4))
        return fail(FR_ERR_INVALID, "linear output size mismatch");
    fr_status s = use_device(t->dev);
    if (s != FR_OK)
        return s;
    FR_CUDA(cudaMemcpyAsync(t->linear.ptr, host, nbytes, cudaMemcpyHostToDevice, t->dev->stream),
            "uploading the linear output");
    FR_CUDA(cudaStreamSynchronize(t->dev->stream), "uploading the linear output");
    return FR_OK;
}

fr_status fr_tracer_write_srgb(fr_tracer* t, const uint8_t* host, size_t nbytes)
{
    FR_CHECK_NULL(t);
    FR_CHECK_NULL(host);
    if (nbytes != size_t(t->w) * t->h * 4)
        return fail(FR_ERR_INVALID, "sRGB output size mismatch");
    fr_status s = use_device(t->dev);
    if (s != FR_OK)
        return s;
    FR_CUDA(cudaMemcpyAsync(t->srgb.ptr, host, nbytes, cudaMemcpyHostToDevice, t->dev->stream),
            "uploading the sRGB output");
    FR_CUDA(cudaStreamSynchronize(t->dev->stream), "uploading the sRGB output");
    return FR_OK;
}

fr_status fr_tracer_get_stats(const fr_tracer* t, fr_stats* out)
{
    FR_CHECK_NULL(t);
    FR_CHECK_NULL(out);
    unsigned long long v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    FR_CUDA(cudaSetDevice(t->dev->ordinal), "cudaSetDevice");
    FR_CUDA(cudaMemcpyAsync(v, t->stats.ptr, sizeof(v), cudaMemcpyDeviceToHost, t->dev->stream),
            "reading tracer counters");
    FR_CUDA(cudaStreamSynchronize(t->dev->stream), "reading tracer counters");
    out->rays = v[0];
    out->paths = v[1];
    out->dropped = v[2];
    out->box_tests = v[3];
    out->prim_tests = v[4];
    out->kernel_launches = t->launches;
    out->bvh_builds = t->builds;
    out->bvh_refits = t->refits;
    out->bvh_build_ms = t->build_ms;
    out->primary_ms = t->kernel_ms[0];
    out->shade_ms = t->kernel_ms[1];
    out->extend_ms = t->kernel_ms[2];
    out->primary_launches = t->kernel_launches[0];
    out->shade_launches = t->kernel_launches[1];
    out->extend_launches = t->kernel_launches[2];
    out->grid_builds = t->grid_builds;
    out->last_render_grid = t->last_grid;
    return FR_OK;
}

fr_status fr_tracer_read_primary_hits(fr_tracer* t, uint32_t* host, size_t nbytes)
{
    FR_CHECK_NULL(t);
    FR_CHECK_NULL(host);
    size_t n = size_t(t->w) * t->h;
    if (nbytes != n * sizeof(uint2))
        return fail(FR_ERR_INVALID, "primary hit buffer size mismatch");
    const size_t K = t->dev->path_k;
    const uint32_t tl = t->dev->path_tile_log2;
    const size_t slots = padded_pixels(t->w, t->h, tl) * K;
    if (t->dev->path_owner != t || K == 0 || t->dev->path.prim_hit.cap < slots)
        return fail(FR_ERR_STATE, "the device's last path render was not this tracer's");
    fr_status s = use_device(t->dev);
    if (s != FR_OK)
        return s;
    std::vector<uint2> all(slots);
    FR_CUDA(cudaMemcpyAsync(all.data(), t->dev->path.prim_hit.ptr, slots * sizeof(uint2),
                            cudaMemcpyDeviceToHost, t->dev->stream),
            "downloading primary hits");
    FR_CUDA(cudaStreamSynchronize(t->dev->stream), "downloading primary hits");
    // sample 0 of pixel (i, j) sits at the start of the pixel's K slots in its tile
    const size_t T = size_t(1) << tl, mask = T - 1;
    const size_t tiles_x = (t->w + T - 1) / T;
    for (uint32_t j = 0; j < t->h; ++j)
        for (uint32_t i = 0; i < t->w; ++i) {
            const size_t slot =
                ((((j >> tl) * tiles_x + (i >> tl)) << (2 * tl)) + ((j & mask) << tl) + (i & mask)) * K;
            host[2 * (size_t(j) * t->w + i)] = all[slot].x;
            host[2 * (size_t(j) * t->w + i) + 1] = all[slot].y;
        }
    return FR_OK;
}

fr_status fr_debug_traversal_compare(fr_scene* sc, const float* rays, uint32_t n, uint32_t* out)
{
    FR_CHECK_NULL(sc);
    FR_CHECK_NULL(rays);
    FR_CHECK_NULL(out);
    fr_status s = use_device(sc->dev);
    if (s != FR_OK || (s = prepare_scene(sc, nullptr)) != FR_OK)
        return s;
    DevArray<float> d_rays;
    DevArray<uint32_t> d_out;
    FR_CUDA(d_rays.reserve(size_t(n) * 6), "alloc");
    FR_CUDA(d_out.reserve(size_t(n) * 6), "alloc");
    FR_CUDA(cudaMemcpy(d_rays.ptr, rays, size_t(n) * 6 * 4, cudaMemcpyHostToDevice), "copy");
    SceneDev sd;
    sd.geoms = sc->table.ptr;
    sd.n_geoms = uint32_t(sc->geoms.size());
    sd.status = sc->dev->status.ptr;
    launch_traversal_compare(sd, d_rays.ptr, n, d_out.ptr, sc->dev->stream);
    FR_CUDA(cudaStreamSynchronize(sc->dev->stream), "compare");
    FR_CUDA(cudaMemcpy(out, d_out.ptr, size_t(n) * 6 * 4, cudaMemcpyDeviceToHost), "copy");
    return FR_OK;
}

fr_status fr_tracer_reset_stats(fr_tracer* t)
{
    FR_CHECK_NULL(t);
    FR_CUDA(cudaSetDevice(t->dev->ordinal), "cudaSetDevice");
    FR_CUDA(cudaMemsetAsync(t->stats.ptr, 0, 8 * sizeof(unsigned long long), t->dev->stream),
            "clearing tracer counters");
    FR_CUDA(cudaStreamSynchronize(t->dev->stream), "clearing tracer counters");
    t->launches = 0;
    t->builds = 0;
    t->refits = 0;
    for (int k = 0; k < 3; ++k) {
        t->kernel_ms[k] = 0.0;
        t->kernel_launches[k] = 0;
    }
    return FR_OK;
}

// ---------------------------------------------------------------------------------------------
// Batched path renders
// ---------------------------------------------------------------------------------------------
fr_status fr_batch_create(fr_device* dev, fr_batch** out)
{
    FR_CHECK_NULL(dev);
    FR_CHECK_NULL(out);
    *out = nullptr;
    fr_status s = use_device(dev);
    if (s != FR_OK)
        return s;
    fr_batch* b = new fr_batch;
    b->dev = dev;
    cudaError_t e = cudaMallocHost((void**)&b->h_ctl, sizeof(BatchCtl));
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = b->ctl.reserve(1);
    if (e != cudaSuccess) {
        delete b;
        return cuda_fail(e, "creating a batch");
    }
    *out = b;
    return FR_OK;
}

fr_status fr_batch_destroy(fr_batch* b)
{
    if (!b)
        return FR_OK;
    cudaSetDevice(b->dev->ordinal);
    cudaStreamSynchronize(b->dev->stream);
    delete b;
    return FR_OK;
}

fr_status fr_batch_clear(fr_batch* b)
{
    FR_CHECK_NULL(b);
    b->items.clear();
    return FR_OK;
}

fr_status fr_batch_add_path(fr_batch* b, fr_tracer* t, fr_scene* sc, const fr_render_params* p,
                            uint32_t first_sample, uint32_t n_render, uint32_t light_samples)
{
    FR_CHECK_NULL(b);
    fr_status s = check_params(t, sc, p);
    if (s != FR_OK)
        return s;
    if (t->dev != b->dev)
        return fail(FR_ERR_INVALID, "the tracer belongs to another device than the batch");
    if (light_samples == 0)
        return fail(FR_ERR_INVALID, "light_samples must be positive");
    if (first_sample == 0)
        return fail(FR_ERR_INVALID, "sample numbers start at 1");
    if (n_render == 0)
        return FR_OK;
    b->items.push_back({t, sc, *p, first_sample, n_render, light_samples});
    return FR_OK;
}

}  // extern "C"

namespace {

// Grow a batch buffer; reports whether its address changed (the graph then has to be redone).
template <class T> cudaError_t grow(DevArray<T>& a, size_t n, bool& moved)
{
    T* old = a.ptr;
    cudaError_t e = a.reserve(n);
    if (a.ptr != old)
        moved = true;
    return e;
}

}  // namespace

extern "C" {

fr_status fr_batch_render(fr_batch* b)
{
    FR_CHECK_NULL(b);
    fr_status s = use_device(b->dev);
    if (s != FR_OK)
        return s;
    fr_device* dev = b->dev;
    if (b->items.empty())
        return FR_OK;

    // scenes: build what is stale (each scene once)
    std::vector<fr_scene*> scenes;
    for (auto& it : b->items)
        if (std::find(scenes.begin(), scenes.end(), it.sc) == scenes.end())
            scenes.push_back(it.sc);
    for (size_t i = 0; i < scenes.size(); ++i) {
        fr_tracer* owner = nullptr;
        for (auto& it : b->items)
            if (it.sc == scenes[i]) {
                owner = it.tr;
                break;
            }
        if ((s = prepare_scene(scenes[i], owner)) != FR_OK)
            return s;
    }

    // path-state capacity: the device's wavefront size, but no more than the batch can fill,
    // and at least one sample of its largest image
    size_t need = 0, largest = 0;
    for (auto& it : b->items) {
        const size_t px = padded_pixels(it.tr->w, it.tr->h, dev->tile_log2);
        need += px * it.n;
        largest = std::max(largest, px);
    }
    size_t cap = std::max(largest, std::min(dev->path_slots, need));

    // plan: every item's samples go to waves in sample order, at most one slice of a tracer
    // per wave, K samples of all pixels per slice; first fit over the waves
    struct Slice {
        size_t item;
        uint32_t first, k;
    };
    std::vector<std::vector<Slice>> waves;
    std::vector<size_t> used;
    std::vector<std::pair<const fr_tracer*, size_t>> last_wave;  // tracer -> next allowed wave
    for (size_t i = 0; i < b->items.size(); ++i) {
        const auto& it = b->items[i];
        const size_t wh = padded_pixels(it.tr->w, it.tr->h, dev->tile_log2);
        size_t min_wave = 0;
        for (auto& lw : last_wave)
            if (lw.first == it.tr)
                min_wave = lw.second;
        uint32_t done = 0;
        while (done < it.n) {
            size_t w = min_wave;
            while (w < waves.size() && cap - used[w] < wh)
                ++w;
            if (w == waves.size()) {
                waves.emplace_back();
                used.push_back(0);
            }
            size_t k = (cap - used[w]) / wh;
            k = std::min<size_t>(k, 4096);
            k = std::min<size_t>(k, it.n - done);
            waves[w].push_back({i, it.first + done, uint32_t(k)});
            used[w] += k * wh;
            done += uint32_t(k);
            min_wave = w + 1;
        }
        bool found = false;
        for (auto& lw : last_wave)
            if (lw.first == it.tr) {
                lw.second = min_wave;
                found = true;
            }
        if (!found)
            last_wave.push_back({it.tr, min_wave});
    }

    // render table
    std::vector<WaveJob> jobs;
    std::vector<uint32_t> wave_first, wave_items, wave_pixels;
    int width = 4;
    uint32_t mask = 0;
    bool all_grid = true;   // every render traces a sphere grid: the grid-only kernels serve
    bool all_parts = true;  // every render traces a grid over its parts
    for (auto& wv : waves) {
        wave_first.push_back(uint32_t(jobs.size()));
        uint64_t slot = 0, item = 0, pixel = 0;
        for (auto& sl : wv) {
            const auto& it = b->items[sl.item];
            WaveJob J;
            std::memset(&J, 0, sizeof(J));
            J.P = frame_params(it.tr, it.sc, &it.params, false, 1);
            J.P.light_samples = it.light_samples;
            J.P.n_samples = sl.first;
            J.P.batch = sl.k;
            if (J.P.bvh_width != 4)
                width = 2;
            mask |= J.P.type_mask;
            all_grid = all_grid && J.P.scene.grid.n_cells != 0 && !J.P.scene.grid.parts;
            all_parts = all_parts && J.P.scene.grid.n_cells != 0 && J.P.scene.grid.parts;
            J.slot_base = uint32_t(slot);
            J.item_base = uint32_t(item);
            J.pixel_base = uint32_t(pixel);
            item += uint64_t(padded_pixels(it.tr->w, it.tr->h, dev->tile_log2)) * sl.k;
            slot = item;
            pixel += uint64_t(it.tr->w) * it.tr->h;
            if (slot > 0xFFFFFFFFull || item > 0xFFFFFFFFull || pixel > 0xFFFFFFFFull)
                return fail(FR_ERR_INVALID, "a batch wave exceeds 2^32 slots");
            jobs.push_back(J);
        }
        wave_items.push_back(uint32_t(item));
        wave_pixels.push_back(uint32_t(pixel));
    }
    if (all_grid && !jobs.empty())
        mask = dev->fuse_shade ? MASK_GRID_FUSED : MASK_GRID;
    else if (all_parts && !jobs.empty() && dev->fuse_shade)
        mask = (mask & (1u << FR_GEOM_MESH)) ? MASK_GRID_PARTS_FUSED : MASK_GRID_PARTS_NO_MESH_FUSED;
    wave_first.push_back(uint32_t(jobs.size()));
    if (mask == 0)
        mask = MASK_SPHERES;  // empty scenes: every ray misses

    bool moved = false;
    FR_CUDA(grow(b->jobs, jobs.size(), moved), "allocating the batch plan");
    FR_CUDA(grow(b->wave_first, wave_first.size(), moved), "allocating the batch plan");
    FR_CUDA(grow(b->wave_items, wave_items.size(), moved), "allocating the batch plan");
    FR_CUDA(grow(b->wave_pixels, wave_pixels.size(), moved), "allocating the batch plan");
    FR_CUDA(b->path.reserve(cap, &moved), "allocating the batch path state");

    cudaStream_t st = dev->stream;
    FR_CUDA(cudaMemcpyAsync(b->jobs.ptr, jobs.data(), jobs.size() * sizeof(WaveJob),
                            cudaMemcpyHostToDevice, st), "uploading the batch plan");
    FR_CUDA(cudaMemcpyAsync(b->wave_first.ptr, wave_first.data(), wave_first.size() * 4,
                            cudaMemcpyHostToDevice, st), "uploading the batch plan");
    FR_CUDA(cudaMemcpyAsync(b->wave_items.ptr, wave_items.data(), wave_items.size() * 4,
                            cudaMemcpyHostToDevice, st), "uploading the batch plan");
    FR_CUDA(cudaMemcpyAsync(b->wave_pixels.ptr, wave_pixels.data(), wave_pixels.size() * 4,
                            cudaMemcpyHostToDevice, st), "uploading the batch plan");
    std::memset(b->h_ctl, 0, sizeof(BatchCtl));
    b->h_ctl->n_waves = uint32_t(waves.size());
    FR_CUDA(cudaMemcpyAsync(b->ctl.ptr, b->h_ctl, sizeof(BatchCtl), cudaMemcpyHostToDevice, st),
            "uploading the batch plan");

    if (b->exec && (moved || b->exec_width != width || b->exec_mask != mask)) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    if (!b->exec) {
        BatchDev B;
        B.jobs = b->jobs.ptr;
        B.wave_first = b->wave_first.ptr;
        B.wave_items = b->wave_items.ptr;
        B.wave_pixels = b->wave_pixels.ptr;
        B.ctl = b->ctl.ptr;
        B.S = b->path.state();
        FR_CUDA(batch_graph_create(B, width, mask, dev->num_sms, b->capture, &b->exec),
                "capturing the batch graph");
        b->exec_width = width;
        b->exec_mask = mask;
        b->stats.graph_captures++;
    }
    cudaEvent_t e0, e1;
    FR_CUDA(cudaEventCreate(&e0), "batch timing");
    FR_CUDA(cudaEventCreate(&e1), "batch timing");
    cudaEventRecord(e0, st);
    cudaError_t le = cudaGraphLaunch(b->exec, st);
    cudaEventRecord(e1, st);
    if (le == cudaSuccess)
        le = cudaMemcpyAsync(b->h_ctl, b->ctl.ptr, sizeof(BatchCtl), cudaMemcpyDeviceToHost, st);
    if (le == cudaSuccess)
        le = cudaStreamSynchronize(st);
    float ms = 0.0f;
    if (le == cudaSuccess)
        cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (le != cudaSuccess)
        return cuda_fail(le, "running the batch graph");

    const BatchCtl& c = *b->h_ctl;
    b->stats.renders += uint32_t(b->items.size());
    b->stats.waves += uint32_t(waves.size());
    b->stats.graph_launches += 1;
    b->stats.shade_extend_pairs += c.pairs;
    // fused grid waves: begin, primary, 3 queue clears, 2 bounces, tail, fold, end;
    // otherwise per wave: begin, primary, fold, end, and per pass: 2 shade, 2 extend, 1
    // condition; 1 start
    if (b->exec_mask == MASK_GRID_FUSED || b->exec_mask == MASK_GRID_PARTS_FUSED ||
        b->exec_mask == MASK_GRID_PARTS_NO_MESH_FUSED)
        b->stats.kernel_launches += 1 + 10 * uint64_t(waves.size());
    else
        b->stats.kernel_launches += 1 + 4 * uint64_t(waves.size()) + 5 * c.pairs;
    b->stats.box_tests += c.box_tests;
    b->stats.prim_tests += c.prim_tests;
    b->stats.last_ms = ms;
    b->stats.total_ms += ms;
    if (c.error)
        return fail(FR_ERR_DEVICE_LIMIT, "batched path tracer exceeded the bounce iteration cap");
    return check_status(dev);
}

fr_status fr_batch_reserve(fr_batch* b, size_t slots)
{
    FR_CHECK_NULL(b);
    fr_status s = use_device(b->dev);
    if (s != FR_OK)
        return s;
    bool moved = false;
    FR_CUDA(b->path.reserve(slots, &moved), "allocating the batch path state");
    if (moved && b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    return FR_OK;
}

fr_status fr_batch_get_stats(const fr_batch* b, fr_batch_stats* out)
{
    FR_CHECK_NULL(b);
    FR_CHECK_NULL(out);
    *out = b->stats;
    return FR_OK;
}

}  // extern "C"
