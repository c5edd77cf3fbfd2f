/*
 * oracle.h -- TEST INFRASTRUCTURE.  C interface of the CPU oracle: a scalar restatement of
 * fresnel's CPU (Embree) path tracer and preview tracer, used only by tests/, by the smoke
 * check and by bench.py's CPU-baseline leg.  Never linked into the product.
 *
 * Two builds share this interface:
 *   oracle/_build/liboracle.so      restated math (oracle/restated_math.hpp)
 *   oracle/_ref/libfresnel_ref.so   the reference's own fresnel/common headers
 * Both use the same BVH, the same per-geometry hit glue (restated from
 * fresnel/cpu/Geometry*.cc) and the same tile loops (restated from fresnel/cpu/Tracer*.cc).
 */
#ifndef FR_ORACLE_H
#define FR_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "../include/fresnel_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_geometry_desc {
    int32_t type; /* FR_GEOM_* */
    int32_t enabled;
    uint32_t n;               /* primitives (mesh: instances) */
    const float* position;    /* [n][3] sphere / polyhedron / mesh */
    const float* radius;      /* [n] sphere / cylinder */
    const float* color;       /* sphere, polyhedron [n][3]; cylinder [n][2][3]; mesh [n_vertices][3] */
    const float* points;      /* cylinder [n][2][3] */
    const float* orientation; /* polyhedron / mesh [n][4] (s, x, y, z) */
    const float* vertices;    /* mesh [n_vertices][3] */
    uint32_t n_vertices;
    const float* plane_origin; /* polyhedron [n_planes][3] */
    const float* plane_normal; /* polyhedron [n_planes][3], already unit length */
    const float* plane_color;  /* polyhedron [n_planes][3] */
    uint32_t n_planes;
    float poly_radius;
    float color_by_face;
    fr_material material;
    fr_material outline_material;
    float outline_width;
    /* polygon: position is [n][2], vertices [n_vertices][2], colour [n][3] */
    const float* angle; /* polygon [n] radians */
    float rounding_radius;
} or_geometry_desc;

typedef struct or_stats {
    uint64_t rays;       /* closest-hit queries */
    uint64_t box_tests;  /* AABB tests */
    uint64_t prim_tests; /* primitive intersection tests */
    uint64_t paths;      /* pixel samples x light samples */
    uint64_t nonfinite;  /* pixel samples whose value was not finite */
} or_stats;

typedef struct or_scene or_scene;

/* Copies the arrays and builds a binned-SAH BVH2 (leaves of at most leaf_max primitives)
 * over every enabled geometry.  Returns NULL on invalid input. */
or_scene* or_scene_create(const or_geometry_desc* geoms, uint32_t n_geoms, int leaf_max);
void or_scene_destroy(or_scene* s);
/* Number of BVH nodes and primitive references (for reporting). */
void or_scene_info(const or_scene* s, uint64_t* nodes, uint64_t* prims);

/* n_render consecutive TracerPath::render calls (fresnel/cpu/TracerPath.cc:56-256): render k
 * uses pixel sample number first_sample + k (1-based).  linear [H][W][4] is the running mean
 * (read and written), srgb [H][W][4] is written.  When pixels != NULL only the listed pixel
 * indices (j*w + i) are rendered and linear/srgb (and m2, if given) are [n_pixels][...].
 * m2 (nullable, [.][3]) accumulates Welford's sum of squared deviations of the RGB samples.
 * nan_guard != 0 skips non-finite samples the way fresnel/gpu/path.cu:111-113 does.
 * nthreads <= 0 uses all hardware threads. */
int or_render_path(const or_scene* s, const fr_render_params* p, uint32_t w, uint32_t h,
                   uint32_t first_sample, uint32_t n_render, uint32_t light_samples,
                   float* linear, uint8_t* srgb, float* m2, const uint32_t* pixels,
                   uint32_t n_pixels, int nan_guard, int nthreads, or_stats* stats);

/* TracerDirect::render (fresnel/cpu/TracerDirect.cc:33-222).  hit_ids (nullable) receives
 * [h][w][aa_n*aa_n][2] = (geometry index + 1, primitive index), (0, 0) on a miss. */
int or_render_preview(const or_scene* s, const fr_render_params* p, uint32_t w, uint32_t h,
                      uint32_t aa_n, float* linear, uint8_t* srgb, uint32_t* hit_ids,
                      int nthreads, or_stats* stats);

/* Single closest-hit query (tests): returns 1 on a hit and fills t, geometry, primitive. */
int or_trace(const or_scene* s, const float o[3], const float d[3], float tnear, float* t,
             uint32_t* geom, uint32_t* prim);

/* Closest-hit glue of one primitive alone (tests): 1 if the ray hits it in (tnear, inf), with
 * out[0] = t and out[1] = the outline distance d. */
int or_prim_hit(const or_scene* s, uint32_t geom, uint32_t prim, const float o[3],
                const float d[3], float tnear, float out[3]);

/* Raw building blocks exposed for unit tests. */
void or_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
float or_u01(uint32_t x);
void or_srgb(const float rgba[4], uint8_t out[4]);
void or_camera_ray(const fr_user_camera* c, uint32_t w, uint32_t h, uint32_t seed, int sample_aa,
                   uint32_t i, uint32_t j, uint32_t sample, float o[3], float d[3]);
/* One MIS bounce decision (fresnel/common/RayGen.h:110-157) for unit tests:
 * out[0..2] = direction, out[3] = factor, out[4] = transmit. */
void or_mis_sample(const fr_material* m, const float v[3], const float n[3], uint32_t depth,
                   uint32_t sample, uint32_t key0, uint32_t key1, float out[5]);
void or_brdf(const fr_material* m, const float l[3], const float v[3], const float n[3],
             const float shading_color[3], float out[3]);
const char* or_math_kind(void);

/* Record the rays trace() answers (7 floats each: origin, direction, tnear) into buffer, up to
   capacity; NULL stops recording.  or_ray_log_count: rays seen since the buffer was set. */
void or_set_ray_log(float* buffer, uint64_t capacity);
uint64_t or_ray_log_count(void);

/* The engine's uniform sphere grid over (pos, rad), restated, walked by n_rays logged rays: out =
   {rays, cells per ray, spheres tested per ray, rays whose grid hit differs from the oracle's BVH
   hit on geometry sphere_geom, cells, references}.  Returns 0 on success. */
int or_grid_walk_stats(const or_scene* s, uint32_t sphere_geom, const float* pos, const float* rad,
                       uint32_t n, float cells_per_sphere, const float* rays, uint64_t n_rays,
                       int nthreads, double out[6]);
/* The engine's uniform grid over the scene's parts (every enabled geometry's primitives, a mesh
   by instance), restated, walked by n_rays logged rays up to the oracle's closest hit: out =
   {rays, cells per ray, references per ray (listed in the cells walked), cells, references}.
   Returns 0 on success. */
int or_parts_grid_walk_stats(const or_scene* s, float cells_per_prim, const float* rays,
                             uint64_t n_rays, int nthreads, double out[5]);

#ifdef __cplusplus
}
#endif

#endif
