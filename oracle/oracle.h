/*
 * oracle.h - CPU restatement of Pencil's per-pixel path-tracing loop.
 *
 * TEST INFRASTRUCTURE ONLY. This code is the checker for the GPU core in
 * pencil_b200/: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it. The product never calls it.
 *
 * It restates, in plain C with Pencil's float32 operation order, the
 * functions on the hot path (file:line in the reference project):
 *   Rng                      src/rng.hpp:13-45
 *   Vec3 helpers, schlick    src/vec3.hpp:24-92
 *   Camera basis / ray_at    src/camera.hpp:67-86, src/camera.cpp:48-68
 *   AABB::hit                src/primitives.hpp:38-49
 *   Sphere/Triangle/Cube/Plane/Cylinder/Cone::hit
 *                            src/primitives.hpp:98-120,145-170,201-238,
 *                            261-272,406-504,517-605
 *   BVHNode::hit/occluded    src/bvh.hpp:31-48
 *   render_tile_region       src/renderer.hpp:309-390 (non-adaptive branch)
 *   trace (Whitted)          src/renderer.hpp:403-822 (supported subset)
 *   trace_path               src/renderer.hpp:829-972
 *   trace_dielectric         src/renderer.hpp:1582-1627
 *   ACES + gamma + 8-bit     src/tonemap.hpp:27-61, src/image_io.hpp:63-113
 * It is compiled with -ffp-contract=off so that no multiply-add is fused,
 * as in the reference's x86-64 build.
 */
#ifndef PENCIL_ORACLE_H
#define PENCIL_ORACLE_H

#include <stdint.h>
#include "../include/pencil_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Scene as the oracle sees it: primitives in the unified index space (mesh
 * triangles expanded to PGPU_PRIM_TRIANGLE records), the DFS node table,
 * and the camera basis from orc_camera_basis(). */
typedef struct orc_scene {
    const pgpu_prim*     prims;     int32_t n_prims;
    const pgpu_bvh_node* nodes;     int32_t n_nodes;
    const pgpu_material* materials; int32_t n_materials;
    const pgpu_light*    lights;    int32_t n_lights;
    float cam[21];   /* origin, lower_left, horizontal, vertical, u, v, w */
    float background[3];
    float ambient[3];
} orc_scene;

enum orc_counter {
    ORC_CNT_REFERENCE_RAYS = 0,   /* trace / trace_path calls              */
    ORC_CNT_EXTENSION_RAYS = 1,   /* Scene::hit calls                      */
    ORC_CNT_SHADOW_RAYS    = 2,   /* Scene::occluded calls                 */
    ORC_CNT_NODE_VISITS    = 3,   /* BVH nodes whose box was tested        */
    ORC_CNT_PRIM_TESTS     = 4,   /* primitive hit tests                   */
    /* The same work split by kind of traversal, and the bytes of the
     * primitive records tested (sphere 16 B = center + radius, triangle
     * 36 B = three float3 vertices, cube 16 B, plane 24 B, cylinder and
     * cone 32 B): the algorithmic traffic of a reference-order walk. */
    ORC_CNT_EXT_NODES      = 5,   /* node visits by Scene::hit             */
    ORC_CNT_EXT_PRIMS      = 6,   /* primitive tests by Scene::hit         */
    ORC_CNT_EXT_PRIM_BYTES = 7,
    ORC_CNT_SH_NODES       = 8,   /* node visits by Scene::occluded        */
    ORC_CNT_SH_PRIMS       = 9,
    ORC_CNT_SH_PRIM_BYTES  = 10,
    ORC_CNT_PRIM_BYTES     = 11,  /* primitive bytes, both kinds           */
    ORC_CNT_N              = 12
};

void orc_camera_basis(const pgpu_camera* cam, float out[21]);

/* Render rows [0, height) with the reference algorithm: per-pixel xorshift32
 * stream over the pixel's samples, both dielectric branches traced.
 * mode = PGPU_MODE_PATHTRACE or PGPU_MODE_WHITTED. out_m2 may be NULL.
 * counters (ORC_CNT_N entries) may be NULL. */
int32_t orc_render(const orc_scene* s, const pgpu_render_params* p,
                   float* out_rgb, float* out_m2, int32_t n_threads,
                   uint64_t* counters);

/* The GPU core's production estimator restated on the CPU (test-only):
 * counter RNG (orc_path_seed), one Fresnel-chosen dielectric branch,
 * quad-light NEE; per-pixel sums in the GPU megakernel's lane order. */
int32_t orc_render_split(const orc_scene* s, const pgpu_render_params* p,
                         float* out_rgb, float* out_m2, int32_t n_threads,
                         uint64_t* counters);

/* The same two renders restricted to a window win = {x, y, w, h} of the
 * image p describes (pixels keep their full-image seeds and jitter);
 * out_rgb / out_m2 hold the window's w*h*3 floats, row-major. */
int32_t orc_render_window(const orc_scene* s, const pgpu_render_params* p,
                          const int32_t* win, float* out_rgb, float* out_m2,
                          int32_t n_threads, uint64_t* counters);
int32_t orc_render_split_window(const orc_scene* s, const pgpu_render_params* p,
                                const int32_t* win, float* out_rgb, float* out_m2,
                                int32_t n_threads, uint64_t* counters);

/* FP64 adjoint of the production estimator (test-only): replays each path
 * with the float32 geometry and decisions of orc_render_split and
 * accumulates, in double, dLoss/d(albedo), dLoss/d(emission) (3 per
 * material) and dLoss/d(intensity) (3 per light) for the pixel weights
 * dl (= dLoss/dimage, W*H*3). out_img (optional) gets the replayed image. */
int32_t orc_adjoint(const orc_scene* s, const pgpu_render_params* p, const float* dl,
                    double* d_albedo, double* d_emission, double* d_light,
                    double* out_img, int32_t n_threads);

/* Closest hit in the reference's traversal order (left subtree first,
 * t_max clipped by the left result), t_min 1e-4, t_max 1e9. */
void orc_trace_rays(const orc_scene* s, const float* rays, int32_t n,
                    int32_t* prim_id, float* t, uint64_t* counters);

/* Camera::ray_at(u, v) then closest hit. */
void orc_primary_hits(const orc_scene* s, const float* uv, int32_t n,
                      int32_t* prim_id, float* t);

/* Camera rays for n (u, v) points: origin[3], direction[3] per ray. */
void orc_camera_rays(const orc_scene* s, const float* uv, int32_t n,
                     float* rays);

/* Hit distance of `ray` (origin[3], direction[3], float32 values) against
 * one primitive, recomputed in double precision; -1 if no hit in
 * [1e-4, 1e9]. */
double orc_hit_t_fp64(const pgpu_prim* prim, const float* ray);

/* HDR -> 8-bit RGB as write_image does. tonemap: 0 none, 1 ACES,
 * 2 Reinhard. */
int32_t orc_render_tile(const orc_scene* s, const pgpu_render_params* p, int32_t tx, int32_t ty,
                        int32_t tw, int32_t th, float* out_rgb);
uint32_t orc_gamma_monotone(void);
void orc_rgb8(const float* hdr, int32_t n_pixels, uint8_t* out,
              int32_t tonemap, float exposure);

/* Counter-RNG path seed shared with the GPU core: the xorshift32 state of
 * the path for sample `sample` of pixel (i, j). */
uint32_t orc_path_seed(int32_t i, int32_t j, int32_t sample, uint32_t salt);

#ifdef __cplusplus
}
#endif

#endif
