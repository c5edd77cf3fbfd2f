/*
 * fresnel_b200.h -- C ABI of the B200 (sm_100a) path-tracing engine.
 *
 * Every entry point takes plain pointers, sizes and opaque handles, returns an
 * fr_status, and never lets a C++ exception cross the boundary.  The text of
 * the last error on the calling thread is available from fr_last_error().
 *
 * The entry points replace the backend classes that fresnel's Python layer
 * binds through its `_gpu` pybind11 module (fresnel/gpu/module-gpu.cc:27-43).
 * Each declaration names the reference method it stands in for.  Geometry
 * buffers live in device memory owned by the library; the host side copies
 * whole arrays (or byte ranges of them) in and out, which is what the
 * reference's Array map()/unmap() pair does (fresnel/gpu/Array.h:190-215).
 *
 * All work of one fr_device is ordered on one CUDA stream owned by that device.
 */
#ifndef FRESNEL_B200_H
#define FRESNEL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FR_ABI_VERSION 1

#if defined(__GNUC__)
#define FR_API __attribute__((visibility("default")))
#else
#define FR_API
#endif

typedef enum fr_status {
    FR_OK = 0,
    FR_ERR_INVALID = 1,      /* bad argument (shape, size, null handle ...) */
    FR_ERR_CUDA = 2,         /* a CUDA runtime call failed */
    FR_ERR_OUT_OF_MEMORY = 3,
    FR_ERR_STATE = 4,        /* operation not allowed in the object's state */
    FR_ERR_DEVICE_LIMIT = 5, /* a kernel hit a bounded limit (stack, iteration cap) */
    FR_ERR_UNSUPPORTED = 6
} fr_status;

/* ------------------------------------------------------------------------ */
/* Plain data shared with the host layer (layouts follow the reference's    */
/* POD structs so they can be filled field by field from Python).           */
/* ------------------------------------------------------------------------ */

enum { FR_CAMERA_ORTHOGRAPHIC = 0, FR_CAMERA_PERSPECTIVE = 1 };

/* fresnel::UserCamera (fresnel/common/Camera.h:55-77). */
typedef struct fr_user_camera {
    float position[3];
    float look_at[3];
    float up[3];
    float h;
    float f;
    float f_stop;
    float focus_distance;
    int32_t model; /* FR_CAMERA_* */
} fr_user_camera;

/* fresnel::Lights (fresnel/common/Light.h:36-40): up to 4 area lights given in camera space. */
typedef struct fr_lights {
    float direction[4][3];
    float color[4][3];
    float theta[4];
    uint32_t n;
} fr_lights;

/* fresnel::Material (fresnel/common/Material.h:47-55). */
typedef struct fr_material {
    float solid;
    float color[3];
    float primitive_color_mix;
    float roughness;
    float specular;
    float metal;
    float spec_trans;
} fr_material;

/* Per-render scene-wide inputs (fresnel/gpu/TracerPath.cc:60-101 uploads the same values as
 * OptiX variables before each launch). */
typedef struct fr_render_params {
    fr_user_camera camera;
    fr_lights lights;
    float background_color[3];
    float background_alpha;
    uint32_t seed;
    int32_t highlight_warning;
    float highlight_color[3];
} fr_render_params;

/* Geometry kinds (fresnel/gpu/module-gpu.cc:33-38). */
enum {
    FR_GEOM_SPHERE = 0,
    FR_GEOM_CYLINDER = 1,
    FR_GEOM_POLYHEDRON = 2,
    FR_GEOM_MESH = 3,
    FR_GEOM_POLYGON = 4
};

/* Per-geometry arrays exposed through the Python Array proxy. */
enum {
    FR_FIELD_POSITION = 0,    /* sphere/polyhedron/mesh: [N][3] f32; polygon: [N][2] f32 */
    FR_FIELD_RADIUS = 1,      /* sphere/cylinder: [N] f32 */
    FR_FIELD_COLOR = 2,       /* sphere/polyhedron/polygon: [N][3]; cylinder: [N][2][3]; mesh: [n_verts][3] */
    FR_FIELD_POINTS = 3,      /* cylinder: [N][2][3] f32 */
    FR_FIELD_ORIENTATION = 4, /* polyhedron/mesh: [N][4] f32 quaternion (s, x, y, z) */
    FR_FIELD_ANGLE = 5        /* polygon: [N] f32, rotation about z in radians */
};

/* Counters accumulated by a tracer since creation (or the last fr_tracer_reset_stats). */
typedef struct fr_stats {
    uint64_t rays;          /* closest-hit queries (primary rays shared across light samples) */
    uint64_t paths;         /* pixel samples x light samples */
    uint64_t dropped;       /* non-finite pixel samples not folded into the mean */
    uint64_t box_tests;     /* ray/AABB tests of the BVH traversals */
    uint64_t prim_tests;    /* ray/primitive intersection tests */
    uint64_t kernel_launches;
    uint64_t bvh_builds;
    double bvh_build_ms;    /* device time of the last BVH build of any geometry */
    /* per-kernel device time, accumulated only while profiling is on (fr_device_set_profiling) */
    double primary_ms, shade_ms, extend_ms;
    uint64_t primary_launches, shade_launches, extend_launches;
    uint64_t bvh_refits;    /* of bvh_builds, how many refitted an existing tree */
    uint64_t grid_builds;   /* grids built (device option "accel") */
    uint32_t last_render_grid; /* the last render's grid: 0 none (BVHs), 1 sphere grid, 2 grid
                                * over the scene's parts */
} fr_stats;

typedef struct fr_device fr_device;
typedef struct fr_scene fr_scene;
typedef struct fr_geometry fr_geometry;
typedef struct fr_tracer fr_tracer;

/* Text of the last failed call on this thread ("" if none). */
FR_API const char* fr_last_error(void);
FR_API int fr_abi_version(void);

/* ---------------- device: fresnel/gpu/Device.cc ---------------- */

/* get_num_available_devices (fresnel/gpu/module-gpu.cc:22-25): number of sm_100 devices. */
FR_API fr_status fr_get_num_available_devices(int* n);
/* Device::getAllGPUs (fresnel/gpu/Device.cc:186-192): one line per GPU, each ending in '\n'. */
FR_API fr_status fr_get_all_gpus(char* buf, size_t cap);
/* Device::Device(ptx_root, n) (fresnel/gpu/Device.cc:29-54).  n = -1 selects all; the engine
 * renders on the first selected GPU. */
FR_API fr_status fr_device_create(int n, fr_device** out);
FR_API fr_status fr_device_destroy(fr_device* dev);
/* Device::describe (fresnel/gpu/Device.cc:114-128). */
FR_API fr_status fr_device_describe(const fr_device* dev, char* buf, size_t cap);
FR_API fr_status fr_device_synchronize(fr_device* dev);
/* Device time between two points of the engine's stream: start records a CUDA event, stop
 * records another, waits for it and returns the elapsed milliseconds.  No counterpart in the
 * reference (its OptiX launches are synchronous); used to time renders on the device. */
FR_API fr_status fr_device_timer_start(fr_device* dev);
FR_API fr_status fr_device_timer_stop(fr_device* dev, float* ms);
/* Engine tuning options of a device (no counterpart in the reference, whose OptiX and Embree
 * backends tune themselves); they apply to BVHs built and renders started afterwards:
 *   "bvh_width"     2 or 4: binary or 4-wide tree traversed by the renderers (default 4)
 *   "leaf_max"      largest leaf the SAH collapse may form (1..16, default 2)
 *   "c_trav"        SAH cost of one node visit relative to one primitive test (default 1)
 *   "path_slots"    path slots traced together by the path tracer, 144 bytes each
 *                   (default 134217728: 18.4 GB; a batch takes at most what it can fill)
 *   "persistent"    1: 4-wide traversal in persistent warps with per-lane refill;
 *                   0: one ray per thread (default)
 *   "builder"       0: LBVH (Karras hierarchy, default); 1: PLOC (locally-ordered clustering)
 *   "tile"          4, 8 (default) or 16: primary rays are traced in square pixel tiles of this
 *                   size, the samples of a pixel in neighbouring threads
 *   "packet"        1: primary rays traced warp-cooperatively (one node sequence per warp, a
 *                   shared stack); 0: one ray per thread (default)
 *   "refill"        1: extension rays with per-lane refill (a warp's idle lanes take new rays
 *                   without waiting for its slowest ray; scenes with one tree, and sphere-grid
 *                   scenes, whose bounces then trace and shade in separate passes); 0: default
 *   "combined"      1 (default): a scene of 2 to 8 enabled geometries gets one BVH over all
 *                   their primitives; 0: each geometry's own BVH, traversed in turn
 *   "shade_blocks"  3 (default) or 4: the shade kernel compiled to fit that many 256-thread
 *                   blocks per SM; 0: as the compiler chooses
 *   "refit"         1: when a geometry's arrays change but its primitive count and the build
 *                   options do not, refit its tree (new boxes, same topology) instead of
 *                   rebuilding it; 0: always rebuild, as the reference does (default)
 *   "accel"         acceleration structure: 0: BVHs; 1: a uniform grid (walked cell by cell
 *                   along each ray) over the spheres of a scene whose only enabled geometry
 *                   holds spheres, else over the primitives of all its enabled geometries (at
 *                   most 8; a mesh by instance); 2 (default): the same grids unless the
 *                   primitives are
 *                   clustered (a cell with more than 64 of them) or a ray would cross more
 *                   than 1024 cells on average; else BVHs.  A primitive spanning more than
 *                   4096 cells leaves any scene to its BVHs.
 *                   The closest hits do not depend on the choice: primitives hit at exactly
 *                   the same distance go to the lower (geometry, primitive) index in every
 *                   structure.
 *   "grid_density"  grid cells per primitive (default 1.5; (0, 64])
 *   "fuse_shade"    1 (default): the primary pass also shades each primary hit and queues the
 *                   continuing paths itself (the first shade pass of a wavefront is not
 *                   launched), and for scenes traced through a sphere grid each bounce traces
 *                   and shades in one kernel; 2: bounces fused for every scene; 0: separate
 *                   passes.  The same images in every case.
 *   "preview_warp"  1 (default): Preview with a multiple of 16 samples per pixel traces each
 *                   pixel with a group of 32 lanes (8x8 anti-aliasing) or 16 (4x4), that many
 *                   of its samples at a time, summed in sample order; 0: one pixel per
 *                   thread.  The same outputs.
 *   "tail"          fused sphere-grid bounces: after this many bounce launches per wavefront
 *                   (0..64, default 1), one persistent launch follows every remaining path to
 *                   its end (a lane takes the next path once its own ends), with no queue
 *                   read-back; -1: a bounce launch per bounce until the queue is empty.  The
 *                   same images in every case.
 * Setting an option marks every BVH of the device's scenes for rebuild when it changes the
 * tree.  Unknown names or out-of-range values return FR_ERR_INVALID. */
FR_API fr_status fr_device_set_option(fr_device* dev, const char* name, double value);
FR_API fr_status fr_device_get_option(const fr_device* dev, const char* name, double* value);
/* When enabled, every kernel launch of the path tracer is bracketed by CUDA events and its
 * device time is accumulated in fr_stats (primary/shade/extend).  Off by default. */
FR_API fr_status fr_device_set_profiling(fr_device* dev, int enable);

/* ---------------- scene: fresnel/gpu/Scene.cc ---------------- */

/* Scene::Scene (fresnel/gpu/Scene.cc:15-28). */
FR_API fr_status fr_scene_create(fr_device* dev, fr_scene** out);
/* Which acceleration structure the scene's last build chose (no counterpart in the reference):
 * *grid = 1 for a sphere grid, 2 for a grid over the primitives of several geometries (or of one
 * non-sphere geometry), 0 for BVHs; reason (nullable, cap bytes) receives why a grid was not
 * chosen when one was considered ("" otherwise). */
FR_API fr_status fr_scene_get_accel(const fr_scene* scene, int* grid, char* reason, size_t cap);
FR_API fr_status fr_scene_destroy(fr_scene* scene);

/* ---------------- geometry: fresnel/gpu/Geometry*.cc ---------------- */

/* GeometrySphere(Scene, N) (fresnel/gpu/GeometrySphere.cc:17-49). */
FR_API fr_status fr_geometry_create_sphere(fr_scene* scene, uint32_t n, fr_geometry** out);
/* GeometryCylinder(Scene, N) (fresnel/gpu/GeometryCylinder.cc). */
FR_API fr_status fr_geometry_create_cylinder(fr_scene* scene, uint32_t n, fr_geometry** out);
/* GeometryConvexPolyhedron(Scene, origins, normals, colors, N, r)
 * (fresnel/cpu/GeometryConvexPolyhedron.cc:22-103; normals are normalised on ingest). */
FR_API fr_status fr_geometry_create_polyhedron(fr_scene* scene, const float* plane_origins,
                                        const float* plane_normals, const float* plane_colors,
                                        uint32_t n_planes, uint32_t n, float radius,
                                        fr_geometry** out);
/* GeometryMesh(Scene, vertices[nv][3], N) (fresnel/cpu/GeometryMesh.cc:20-72; nv % 3 == 0). */
FR_API fr_status fr_geometry_create_mesh(fr_scene* scene, const float* vertices, uint32_t n_vertices,
                                  uint32_t n, fr_geometry** out);
/* GeometryPolygon(Scene, vertices[nv][2], rounding_radius, N) (fresnel/cpu/GeometryPolygon.cc:
 * 20-82): simple polygons (vertices counter-clockwise, concave allowed) in the xy plane, each
 * placed at its 2-D position and rotated about z by its angle, rounded by rounding_radius
 * (spheropolygons), double sided.  n_vertices >= 1. */
FR_API fr_status fr_geometry_create_polygon(fr_scene* scene, const float* vertices,
                                            uint32_t n_vertices, float rounding_radius, uint32_t n,
                                            fr_geometry** out);
/* GeometryPolygon::getRadius: the largest vertex distance from the origin plus the rounding
 * radius (the half extent of each polygon's bounding square). */
FR_API fr_status fr_geometry_get_radius(const fr_geometry* geom, float* radius);
/* ~Geometry / Geometry::remove (fresnel/gpu/Geometry.cc:18-58). */
FR_API fr_status fr_geometry_destroy(fr_geometry* geom);
/* Geometry::remove (fresnel/gpu/Geometry.cc:47-58): detach for good; enable/disable then fail. */
FR_API fr_status fr_geometry_remove(fr_geometry* geom);
/* Array<T>::unmap of a geometry buffer: copy host bytes into the device array and mark the
 * geometry's BVH stale (fresnel/util.py:54-62, fresnel/gpu/Geometry.h:85-89). */
FR_API fr_status fr_geometry_write(fr_geometry* geom, int field, const void* host, size_t offset_bytes,
                            size_t nbytes);
/* Array<T>::map of a geometry buffer: copy device bytes to the host. */
FR_API fr_status fr_geometry_read(fr_geometry* geom, int field, void* host, size_t offset_bytes,
                           size_t nbytes);
/* Byte size of a field (0 if the geometry kind has no such field). */
FR_API fr_status fr_geometry_field_size(const fr_geometry* geom, int field, size_t* nbytes);
/* Geometry::enable / disable (fresnel/gpu/Geometry.cc:24-45). */
FR_API fr_status fr_geometry_set_enabled(fr_geometry* geom, int enabled);
/* Geometry::setMaterial / setOutlineMaterial / setOutlineWidth (fresnel/gpu/Geometry.h:43-80). */
FR_API fr_status fr_geometry_set_material(fr_geometry* geom, const fr_material* material,
                                   const fr_material* outline_material, float outline_width);
/* GeometryConvexPolyhedron::setColorByFace (fresnel/cpu/GeometryConvexPolyhedron.h:69-72). */
FR_API fr_status fr_geometry_set_color_by_face(fr_geometry* geom, float f);
/* Geometry::update (fresnel/gpu/Geometry.h:85-89): mark the BVH stale. */
FR_API fr_status fr_geometry_update(fr_geometry* geom);
/* Build (or rebuild) every stale BVH of the scene now instead of at the next render. */
FR_API fr_status fr_scene_build(fr_scene* scene);

/* ---------------- tracers: fresnel/gpu/Tracer*.cc ---------------- */

/* Tracer::Tracer(device, w, h) (fresnel/gpu/Tracer.cc:14-22). */
FR_API fr_status fr_tracer_create(fr_device* dev, uint32_t w, uint32_t h, fr_tracer** out);
FR_API fr_status fr_tracer_destroy(fr_tracer* tr);
/* Tracer::resize (fresnel/gpu/Tracer.cc:26-51); w or h == 0 is an error. Clears both outputs. */
FR_API fr_status fr_tracer_resize(fr_tracer* tr, uint32_t w, uint32_t h);
/* TracerPath::reset's buffer clear (fresnel/cpu/TracerPath.cc:31-47). */
FR_API fr_status fr_tracer_clear(fr_tracer* tr);

/* TracerPath::render (fresnel/gpu/TracerPath.cc:60-102), called n_render times in a row:
 * render k (k = 0..n_render-1) takes pixel sample number first_sample + k (1-based, the
 * value of m_n_samples after its increment) and folds it into the running mean. */
FR_API fr_status fr_tracer_render_path(fr_tracer* tr, fr_scene* scene, const fr_render_params* params,
                                uint32_t first_sample, uint32_t n_render,
                                uint32_t light_samples);

/* TracerDirect::render (fresnel/gpu/TracerDirect.cc): aa_n x aa_n primary samples per pixel.
 * If hit_ids is not NULL it receives, for each pixel and AA sample, the pair
 * (geometry index + 1, primitive index) of the closest hit ((0, 0) on a miss), laid out
 * [h][w][aa_n*aa_n][2] (host memory, 8 bytes per sample). */
FR_API fr_status fr_tracer_render_preview(fr_tracer* tr, fr_scene* scene, const fr_render_params* params,
                                   uint32_t aa_n, uint32_t* hit_ids);

/* Output buffers: linear RGBA f32 [h][w][4] and sRGB RGBA u8 [h][w][4]
 * (fresnel/gpu/Tracer.cc:26-51, the reference's getLinearOutputBuffer/getSRGBOutputBuffer). */
FR_API fr_status fr_tracer_read_linear(fr_tracer* tr, float* host, size_t nbytes);
FR_API fr_status fr_tracer_read_srgb(fr_tracer* tr, uint8_t* host, size_t nbytes);
FR_API fr_status fr_tracer_write_linear(fr_tracer* tr, const float* host, size_t nbytes);
FR_API fr_status fr_tracer_write_srgb(fr_tracer* tr, const uint8_t* host, size_t nbytes);
/* Tracer.histogram (fresnel/tracer.py:79-108) computed on the device from the linear output:
 * counts[512][4] (nbytes = 8192) of the pixels with alpha > 0, columns lightness
 * l = 0.21 r + 0.72 g + 0.07 b, R, G, B, each value raised to 1/2.2 and binned over [0, 1] in
 * 512 equal bins as numpy.histogram does (float32 arithmetic as numpy's; the power rounded
 * once from double precision, where numpy's float32 power may differ by an ulp). */
FR_API fr_status fr_tracer_histogram(fr_tracer* tr, uint32_t* counts, size_t nbytes);
/* Page-locked host memory (no counterpart in the reference, whose arrays live in pageable
 * memory, fresnel/gpu/Array.h:98-223): fr_tracer_read_* and fr_geometry_write copy to and
 * from it at full link speed without a staging copy.  fr_host_free(NULL) does nothing. */
FR_API fr_status fr_host_alloc(size_t nbytes, void** out);
FR_API fr_status fr_host_free(void* host);
FR_API fr_status fr_tracer_get_stats(const fr_tracer* tr, fr_stats* out);
/* Parity hook (no counterpart in the reference): the closest hits of the primary rays of the
 * first sample of the last wavefront of the device's last path render, which must have been
 * this tracer's (else FR_ERR_STATE), [h][w][2] = (geometry index or 0xFFFFFFFF, primitive
 * index), for comparing traversal variants and the CPU oracle. */
FR_API fr_status fr_tracer_read_primary_hits(fr_tracer* tr, uint32_t* host, size_t nbytes);
FR_API fr_status fr_tracer_reset_stats(fr_tracer* tr);

/* ---------------- allocation-free path render ----------------
 * No counterpart in the reference.  fr_tracer_render_path keeps its wavefront state (rays,
 * throughputs, queues) in device memory shared by the device's tracers, which it allocates on
 * first use and reallocates when a call needs a larger wavefront; cudaFree of the old block
 * waits for the whole GPU.  fr_tracer_render_path_static renders the same images without allocating any memory: the
 * wavefront state lives in one fixed array of FR_STATIC_PATH_SLOTS slots of 144 bytes (37.7 MB)
 * inside the library's device module.  It is for callers that must not allocate inside a render
 * call: a runtime that reserves the GPU's memory up front for its own pool, or a frame loop
 * that shares the GPU with other streams and cannot let a cudaFree stall them.
 *
 *  - Limit: the image may have at most FR_STATIC_PATH_SLOTS pixels, counted with the image
 *    rounded up to whole primary tiles (8 x 8 by default): 512 x 512 fits; larger images
 *    return FR_ERR_INVALID.  Each wavefront traces FR_STATIC_PATH_SLOTS / (padded pixels)
 *    samples of every pixel (at most 4096).
 *  - The scene must be built (fr_scene_build after its last change): a build allocates, so a
 *    scene with stale BVHs or geometry table returns FR_ERR_STATE.
 *  - The first call on each device looks up the array's address (cudaGetSymbolAddress, which
 *    may load the library's device module).  Make that first call outside any CUDA stream
 *    capture.
 *  - The array is shared by all tracers of the process on one GPU.  Calls that overlap in time
 *    (several host threads, or several fr_device handles on the same GPU) race on it and give
 *    wrong images: serialise them.
 *  - The queue-length counters at the start of the array are cleared by every call; nothing
 *    else needs to start at zero.  Kernel profiling (fr_device_set_profiling) is ignored here.
 * Arguments and results are those of fr_tracer_render_path. */
#define FR_STATIC_PATH_SLOTS 262144u
FR_API fr_status fr_tracer_render_path_static(fr_tracer* tr, fr_scene* scene,
                                              const fr_render_params* params, uint32_t first_sample,
                                              uint32_t n_render, uint32_t light_samples);

/* ---------------- batched path renders ----------------
 * No counterpart in the reference, which renders one Tracer.Path call at a time.  A batch
 * queues path renders of any tracers, scenes and image sizes on one device and traces them
 * together: their pixel samples share wavefronts and kernel launches, and the whole batch is
 * one CUDA graph launch (device-side loops over waves and bounces, no host round trips).  Each
 * render's output equals what fr_tracer_render_path gives for the same arguments.  Renders of
 * one tracer are traced in the order they were added.  Tracers and scenes must stay alive until
 * fr_batch_render returns; fr_batch_render keeps the queue (fr_batch_clear empties it). */
typedef struct fr_batch fr_batch;
typedef struct fr_batch_stats {
    uint32_t renders;             /* renders traced */
    uint32_t waves;               /* wavefronts (renders that fit the path state together) */
    uint64_t graph_launches;
    uint64_t graph_captures;
    uint64_t kernel_launches;     /* kernels executed inside the graphs */
    uint64_t shade_extend_pairs;  /* device-side loop passes (two bounces each) */
    uint64_t box_tests, prim_tests;
    float last_ms;                /* device time of the last fr_batch_render */
    double total_ms;
} fr_batch_stats;
FR_API fr_status fr_batch_create(fr_device* dev, fr_batch** out);
FR_API fr_status fr_batch_destroy(fr_batch* batch);
/* Queue n_render TracerPath::render calls of tr on scene (as fr_tracer_render_path). */
FR_API fr_status fr_batch_add_path(fr_batch* batch, fr_tracer* tr, fr_scene* scene,
                                   const fr_render_params* params, uint32_t first_sample,
                                   uint32_t n_render, uint32_t light_samples);
FR_API fr_status fr_batch_clear(fr_batch* batch);
/* Build stale scenes, then trace every queued render. */
FR_API fr_status fr_batch_render(fr_batch* batch);
/* Allocate the batch's path state for `slots` path slots now (144 bytes each), so that later
 * fr_batch_render calls whose waves fit need no allocation (a render grows it on demand). */
FR_API fr_status fr_batch_reserve(fr_batch* batch, size_t slots);
FR_API fr_status fr_batch_get_stats(const fr_batch* batch, fr_batch_stats* out);

/* ---------------- self-tests ---------------- */

/* Diagnostic (no counterpart in the reference): trace n rays (o.xyz, d.xyz, 6 floats each,
 * host) through a sphere scene's 4-wide trees with the one-ray-per-thread traversal and with
 * the step-wise traversal of the persistent kernels; out (host, 6 words per ray) receives
 * (geometry, primitive, box tests) of each. */
FR_API fr_status fr_debug_traversal_compare(fr_scene* scene, const float* rays, uint32_t n,
                                            uint32_t* out);

/* Runs the engine's device Philox4x32-10 and cuRAND's curand_Philox4x32_10 on n inputs
 * in[i] = (ctr0, ctr1, ctr2, ctr3, key0, key1) (host arrays; outputs n x 4 words each).
 * No counterpart in the reference: Random123's known-answer vectors are not in its tree, and
 * this is how the generator behind fresnel/common/RayGen.h:49-61 is checked on the device. */
FR_API fr_status fr_selftest_philox(const uint32_t* in, uint32_t n, uint32_t* engine_out,
                                    uint32_t* curand_out);

#ifdef __cplusplus
}
#endif

#endif /* FRESNEL_B200_H */
