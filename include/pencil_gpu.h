/*
 * pencil_gpu.h - C-ABI of the B200 path-tracing core for the Pencil ray tracer.
 *
 * This library replaces Pencil's CPU render loop:
 *
 *   pencil::Renderer::Renderer(const Scene&, const Camera&, RenderSettings)
 *                                                   src/renderer.hpp:155-169
 *   void pencil::Renderer::render(std::vector<Color>& out, RenderStats*)
 *                                                   src/renderer.hpp:198-295
 *
 * and everything below it on the per-pixel path: the tile/pixel/sample loop
 * (render_tile_region, src/renderer.hpp:309-390), camera rays
 * (Camera::ray_at, src/camera.cpp:48-68), the path tracer
 * (trace_path, src/renderer.hpp:829-972), the Whitted tracer used after glass
 * and as the default CLI mode (trace / trace_dielectric,
 * src/renderer.hpp:403-822, 1582-1627), closest/any-hit BVH traversal
 * (Scene::hit/occluded, src/scene.hpp:55-81; BVHNode::hit/occluded,
 * src/bvh.hpp:31-48) and primitive intersection (src/primitives.hpp).
 *
 * Conventions
 *  - Every function returns a pgpu_status (0 = OK, negative = error) unless
 *    stated otherwise; pgpu_last_error() gives a one-line reason.
 *  - All host buffers are caller-owned: they are copied in, or filled before
 *    the call returns; no pointer is retained after a call.
 *  - Calls are synchronous with respect to their outputs.
 *  - A context is single-threaded (not re-entrant); separate contexts may be
 *    used from separate threads.
 *  - Unsupported scene features are rejected (PGPU_ERR_UNSUPPORTED), never
 *    approximated.
 *  - No CPU fallback exists: without a usable CUDA device pgpu_create fails.
 */
#ifndef PENCIL_GPU_H
#define PENCIL_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PGPU_ABI_VERSION 2

/* ---- status codes ------------------------------------------------------ */
enum pgpu_status {
    PGPU_OK                  =  0,
    PGPU_ERR_INVALID_ARG     = -1,  /* null pointer, bad size, bad enum      */
    PGPU_ERR_UNSUPPORTED     = -2,  /* scene feature outside the GPU core    */
    PGPU_ERR_CUDA            = -3,  /* a CUDA runtime call failed            */
    PGPU_ERR_QUEUE_OVERFLOW  = -4,  /* a device queue ran out of capacity    */
    PGPU_ERR_TIMEOUT         = -5,  /* device work exceeded the time budget
                                       of pgpu_set_timeout                   */
    PGPU_ERR_NO_SCENE        = -6,  /* unknown or freed scene id             */
    PGPU_ERR_OUT_OF_MEMORY   = -7,  /* device allocation failed              */
    PGPU_ERR_BVH_INVALID     = -8   /* node table is not a valid DFS tree    */
};

/* ---- scene description ------------------------------------------------- */

/* Primitive kinds (src/primitives.hpp). A quad (make_quad,
 * src/primitives.hpp:390-396) is passed as its two triangles. */
enum pgpu_prim_type {
    PGPU_PRIM_SPHERE   = 0,  /* p: center[3], radius                         */
    PGPU_PRIM_TRIANGLE = 1,  /* p: v0[3], v1[3], v2[3]                       */
    PGPU_PRIM_CUBE     = 2,  /* p: center[3], half_extent                    */
    PGPU_PRIM_PLANE    = 3,  /* p: point[3], unit normal[3]                  */
    PGPU_PRIM_CYLINDER = 4,  /* p: center[3], unit axis[3], radius, half_h   */
    PGPU_PRIM_CONE     = 5   /* p: apex[3], unit axis[3], radius, height     */
};

/* One primitive, holding the primitive's stored state after its C++
 * constructor ran (normalised normal/axis, half height), so that hit
 * arithmetic reproduces Pencil's bit for bit. Use pgpu_make_prim() to
 * build one from constructor arguments. 64 bytes. */
typedef struct pgpu_prim {
    int32_t type;       /* enum pgpu_prim_type                             */
    int32_t material;   /* index into pgpu_scene.materials                 */
    float   p[14];      /* parameters, see enum pgpu_prim_type             */
} pgpu_prim;

/* One node of Pencil's binary BVH (src/bvh.hpp:22-49) in DFS pre-order,
 * left subtree before right subtree, one primitive per leaf. This is the
 * order in which BVH::build_range (src/bvh.hpp:74-104) creates nodes, so a
 * walk of Pencil's own tree emits it directly. 32 bytes. */
typedef struct pgpu_bvh_node {
    float   bmin[3];
    int32_t left;       /* interior: index of left child (= own index + 1);
                           leaf: -1                                         */
    float   bmax[3];
    int32_t right;      /* interior: index of right child;
                           leaf: primitive index (into the unified index
                           space: prims first, then mesh triangles)         */
} pgpu_bvh_node;

enum pgpu_material_kind {     /* src/material.hpp:17-22 */
    PGPU_MAT_DIFFUSE    = 0,
    PGPU_MAT_METAL      = 1,
    PGPU_MAT_DIELECTRIC = 2
};

/* Material (src/material.hpp:29-80, the fields the GPU core supports).
 * Textures, normal maps, SSS, dispersion and principled BSDFs are outside
 * the core: scenes using them are rejected by the Pencil-side bridge.
 * 64 bytes. */
typedef struct pgpu_material {
    int32_t kind;               /* enum pgpu_material_kind                 */
    float   albedo[3];
    float   emission[3];
    float   reflectivity;       /* metal mirror factor (1 - fuzz)          */
    float   ior;
    float   specular;           /* Phong intensity (Whitted shading)       */
    float   shininess;          /* Phong exponent                          */
    float   specular_color[3];
    int32_t flags;              /* reserved, must be 0                     */
    int32_t reserved;
} pgpu_material;

enum pgpu_light_kind {        /* src/light.hpp:15-46, plus area quads */
    PGPU_LIGHT_POINT       = 0,
    PGPU_LIGHT_DIRECTIONAL = 1,
    /* A rectangular emitter used for next-event estimation in path-trace
     * mode. Pencil has no such light: its emissive quads are reached only by
     * BSDF sampling. The quad estimator (radiance * cos * cos' / r^2 * area,
     * diffuse BRDF albedo/pi) has the same expectation; BSDF-sampled hits on
     * the emitter's material after a diffuse bounce then skip its emission. */
    PGPU_LIGHT_QUAD        = 2
};

/* 64 bytes. */
typedef struct pgpu_light {
    int32_t kind;           /* enum pgpu_light_kind                          */
    float   pos[3];         /* point: position; directional: unit direction
                               the light travels; quad: corner              */
    float   intensity[3];   /* point/directional: intensity; quad: radiance */
    float   radius;         /* point: soft-shadow disc radius (0 = hard)    */
    int32_t is_emissive;    /* point: skip the shadow test                  */
    float   edge_u[3];      /* quad: first edge from the corner             */
    float   edge_v[3];      /* quad: second edge from the corner            */
    int32_t material;       /* quad: material of the emitter surface        */
} pgpu_light;

/* Camera constructor arguments (src/camera.hpp:29-36). The library derives
 * the basis and frustum exactly as Camera::recompute_basis/recompute_frustum
 * do (src/camera.hpp:67-86). */
typedef struct pgpu_camera {
    float eye[3];
    float look[3];
    float up[3];
    float vfov_deg;
    float aspect;
    float aperture;         /* must be 0: depth of field is outside the core */
    float focus_dist;
} pgpu_camera;

typedef struct pgpu_scene {
    const pgpu_prim*     prims;           int32_t n_prims;
    /* Optional indexed triangle mesh: float32 vertices, int32 indices.
     * Mesh triangle k has unified primitive index n_prims + k. */
    const float*         mesh_vertices;   int32_t n_mesh_vertices;  /* xyz  */
    const int32_t*       mesh_indices;    int32_t n_mesh_triangles; /* 3/tri*/
    const int32_t*       mesh_materials;  /* one per mesh triangle           */
    /* Pencil's BVH in DFS pre-order. NULL: the library builds the same
     * tree itself (pgpu_build_bvh). */
    const pgpu_bvh_node* nodes;           int32_t n_nodes;
    const pgpu_material* materials;       int32_t n_materials;
    const pgpu_light*    lights;          int32_t n_lights;
    pgpu_camera          camera;
    float                background[3];   /* Scene::background              */
    float                ambient[3];      /* Scene::ambient                 */
} pgpu_scene;

/* ---- render parameters ------------------------------------------------- */

enum pgpu_mode {
    PGPU_MODE_PATHTRACE = 0,   /* trace_path (RenderSettings::pathtrace)     */
    PGPU_MODE_WHITTED   = 1    /* trace (the CLI default)                    */
};

enum pgpu_engine {
    PGPU_ENGINE_WAVEFRONT  = 0, /* persistent generate/extend/shade/shadow    */
    PGPU_ENGINE_MEGAKERNEL = 1  /* one thread per path, all bounces in one
                                   kernel                                    */
};

enum pgpu_rng {
    /* Each path (pixel, sample) seeds its own xorshift32 stream from
     * Pencil's per-pixel seed i*97861 + j*1973 + 1 (src/renderer.hpp:313)
     * mixed with the sample index. */
    PGPU_RNG_COUNTER          = 0,
    /* One xorshift32 stream per pixel consumed sequentially over the
     * pixel's samples, exactly as Pencil does. Megakernel only. */
    PGPU_RNG_PIXEL_SEQUENTIAL = 1
};

enum pgpu_glass {
    /* At a dielectric hit the Whitted continuation follows the reflected
     * ray with probability kr and the refracted ray otherwise (weight
     * albedo; total internal reflection always reflects). Unbiased for
     * trace_dielectric's expectation. */
    PGPU_GLASS_FRESNEL_SPLIT  = 0,
    /* Both branches are traced, as trace_dielectric does (megakernel only). */
    PGPU_GLASS_BOTH_BRANCHES  = 1
};

enum pgpu_flags {
    PGPU_FLAG_DEVICE_OUTPUT = 1,  /* out_rgb / out_m2 are device pointers   */
    PGPU_FLAG_COUNT_RAYS    = 2,  /* fill the ray counters in pgpu_stats    */
    PGPU_FLAG_COUNT_NODES   = 4,  /* also count node visits / prim tests    */
    PGPU_FLAG_NO_GRAPH      = 8,  /* wavefront: launch kernels one by one
                                     instead of replaying a CUDA graph       */
    PGPU_FLAG_PROFILE_KERNELS = 16, /* time each kernel class (implies
                                     NO_GRAPH); see pgpu_stats.kernel_ms     */
    PGPU_FLAG_NO_PACKETS    = 32, /* wavefront: trace camera rays one per lane
                                     instead of as warp packets              */
    PGPU_FLAG_MIS           = 64, /* path tracing with trace_path_mis's light
                                     weights (RenderSettings::mis,
                                     src/renderer.hpp:55, 1205-1346)         */
    PGPU_FLAG_BINARY_TREE   = 128 /* megakernel: traverse Pencil's binary tree
                                     (src/bvh.hpp:31-48) instead of the 4-wide
                                     tree collapsed from it, which both
                                     engines use by default                  */
};

typedef struct pgpu_render_params {
    int32_t  width;
    int32_t  height;
    int32_t  samples;           /* n: n*n stratified samples per pixel       */
    int32_t  depth;             /* path-trace bounces / Whitted max depth    */
    int32_t  mode;              /* enum pgpu_mode                            */
    int32_t  engine;            /* enum pgpu_engine                          */
    int32_t  rng;               /* enum pgpu_rng                             */
    int32_t  glass;             /* enum pgpu_glass                           */
    float    shadow_bias;       /* RenderSettings::shadow_bias (1e-3)        */
    int32_t  soft_shadow_samples; /* RenderSettings::soft_shadow_samples (4) */
    uint32_t seed;              /* salt mixed into the counter RNG (0: none) */
    int32_t  sample_offset;     /* first sample index (progressive renders)  */
    int32_t  flags;             /* enum pgpu_flags                           */
    int32_t  queue_capacity;    /* wavefront paths in flight, 0..2^28 (0:
                                   automatic)                                */
    int32_t  refill_below;      /* wavefront: a warp takes new rays once at
                                   most this many of its 32 lanes are still
                                   traversing (0: automatic)                 */
    int32_t  sort_key;          /* wavefront ray order: 0 queue order, 1 binned
                                   by direction octant, 2 shadow work sorted
                                   by origin (Morton code) and octant, 3 also
                                   the extension rays of bounces >= 1        */
    int32_t  block_size;        /* wavefront threads per block: 64, 128 or 256
                                   (0: 128; pgpu_render_noalloc always 128)  */
} pgpu_render_params;

typedef struct pgpu_stats {
    uint64_t paths;            /* camera paths rendered                      */
    uint64_t extension_rays;   /* closest-hit rays traced                    */
    uint64_t shadow_rays;      /* any-hit rays traced                        */
    uint64_t reference_rays;   /* Pencil's count: one per trace* call
                                  (src/renderer.hpp:404, 830)               */
    uint64_t node_visits;      /* interior nodes fetched (COUNT_NODES)       */
    uint64_t prim_tests;       /* primitive tests (COUNT_NODES)              */
    uint64_t ext_node_visits;  /* of which by closest-hit traversal          */
    uint64_t ext_leaf_bytes;   /* leaf bytes read by closest-hit traversal   */
    uint64_t shadow_node_visits; /* of which by any-hit traversal            */
    uint64_t shadow_leaf_bytes;  /* leaf bytes read by any-hit traversal     */
    double   device_ms;        /* device time of the render kernels          */
    double   total_ms;         /* wall time of the call                      */
    /* PGPU_FLAG_PROFILE_KERNELS: device time per kernel class (generate,
     * extend, shade, shadow, accumulate, megakernel), from CUDA events
     * around every launch (kernels are then launched one by one). */
    double   kernel_ms[6];
    int32_t  kernel_launches;  /* kernels launched by the call               */
    int32_t  reserved;
} pgpu_stats;

typedef struct pgpu_ctx pgpu_ctx;

/* ---- functions --------------------------------------------------------- */

int32_t pgpu_abi_version(void);

/* Create a context on CUDA device `device`. */
int32_t pgpu_create(int32_t device, pgpu_ctx** out);
void    pgpu_destroy(pgpu_ctx* ctx);
const char* pgpu_last_error(const pgpu_ctx* ctx);

/* Use a caller-provided cudaStream_t (NULL: the context's own stream). */
int32_t pgpu_set_stream(pgpu_ctx* ctx, void* cuda_stream);
void*   pgpu_get_stream(pgpu_ctx* ctx);

/* Wall-clock budget, in milliseconds, of the device work of one render,
 * batch or adjoint call (0, the default: none). A call whose kernels have
 * not finished within it returns PGPU_ERR_TIMEOUT before anything is copied
 * to the caller's host buffers (device outputs are still written as the
 * work completes); the context's next call first waits for that work. The
 * kernels themselves always end: none waits on a flag or on another block.
 * Counterpart of the reference's socket timeouts for workers that stop
 * answering (src/distributed.hpp:527-545). */
int32_t pgpu_set_timeout(pgpu_ctx* ctx, int32_t ms);

/* The tree the wide traversals walk (both engines), for scenes uploaded
 * after the call. Either way the leaves are the uploaded tree's: its leaf
 * boxes, bit for bit, and its DFS leaf order, which decides among hits at
 * equal distance as BVHNode::hit does (src/bvh.hpp:31-37), so hit
 * distances are the same and images agree but where rounding at a box face
 * makes the order of the walk matter. The binary tree the upload keeps
 * (PGPU_FLAG_BINARY_TREE, the adjoint) is the uploaded one in both modes.
 *   PGPU_TRAVERSAL_UPLOADED (0, default): the uploaded tree (Pencil's SAH
 *       tree), collapsed to wide nodes.
 *   PGPU_TRAVERSAL_LBVH (1): a linear BVH over the uploaded leaves, built on
 *       the device at upload (Morton order of the box centres), then
 *       collapsed: on meshes where Pencil's 12-bucket split binning over the
 *       parent box groups badly, far fewer node visits per ray.
 *   PGPU_TRAVERSAL_SAH (2): a binned SAH tree over the uploaded leaves,
 *       built on the device at upload: 16 buckets over each node's centroid
 *       bounds on all three axes, Pencil's cost function, one primitive per
 *       leaf; slower to build than the LBVH, fewer node visits.
 * No counterpart in the reference, whose renderer walks the tree it built. */
enum pgpu_traversal_tree {
    PGPU_TRAVERSAL_UPLOADED = 0,
    PGPU_TRAVERSAL_LBVH     = 1,
    PGPU_TRAVERSAL_SAH      = 2
};
int32_t pgpu_set_traversal_tree(pgpu_ctx* ctx, int32_t mode);

/* Build the primitive's stored state from its constructor arguments, with
 * the same float arithmetic as the C++ constructors (plane normal and
 * cylinder/cone axis normalised; cylinder height halved).
 *   sphere:   a = center, s0 = radius
 *   triangle: a, b, c = vertices
 *   cube:     a = center, s0 = half extent
 *   plane:    a = point, b = normal
 *   cylinder: a = center, b = axis, s0 = radius, s1 = height
 *   cone:     a = apex, b = axis, s0 = radius, s1 = height            */
int32_t pgpu_make_prim(int32_t type, int32_t material, const float* a,
                       const float* b, const float* c, float s0, float s1,
                       pgpu_prim* out);

/* Build Pencil's SAH BVH (BVH::build, src/bvh.hpp:54-192: longest axis,
 * 12 buckets, median split for <= 4 primitives) over the unified primitive
 * index space and write it in DFS pre-order. `out_nodes` must hold
 * 2*(n_prims + n_mesh_triangles) - 1 nodes. Host only. */
int32_t pgpu_build_bvh(const pgpu_scene* scene, pgpu_bvh_node* out_nodes,
                       int32_t* out_n_nodes, int32_t* out_depth);

/* A BVH built on the GPU in the same table format (DFS pre-order, one
 * primitive per leaf): a linear BVH over the Morton codes of the primitive
 * boxes' centres (Karras 2012), for scenes whose host SAH build
 * (pgpu_build_bvh, Pencil's tree) costs too much, e.g. many scenes or every
 * frame of an animation. No counterpart in the reference, which builds on
 * the host only (src/bvh.hpp:54-192). It is a different tree: renders agree
 * with those on Pencil's tree up to hit ties within rounding. out_nodes NULL:
 * *out_n_nodes gets the table size only. */
int32_t pgpu_build_bvh_device(pgpu_ctx* ctx, const pgpu_scene* scene,
                              pgpu_bvh_node* out_nodes, int32_t* out_n_nodes,
                              int32_t* out_depth);

/* Pencil's own SAH tree (BVH::build, src/bvh.hpp:74-192: 12 buckets along
 * the longest axis, cost 1 + (nL SA_L + nR SA_R) / SA_P, median split for
 * <= 4 primitives and when no bucket boundary separates) built on the GPU,
 * one tree level at a time, in the same table format. Splits are those of
 * the host build; the sides of a split keep their primitives in a stable
 * order where Pencil's std::partition does not, so trees agree node for node
 * unless two primitives tie in a median split's centroid key. out_nodes
 * NULL: *out_n_nodes gets the table size only. */
int32_t pgpu_build_bvh_device_sah(pgpu_ctx* ctx, const pgpu_scene* scene,
                                  pgpu_bvh_node* out_nodes, int32_t* out_n_nodes,
                                  int32_t* out_depth);

/* Upload a scene; returns a scene id valid until pgpu_free_scene. */
int32_t pgpu_upload_scene(pgpu_ctx* ctx, const pgpu_scene* scene,
                          int32_t* out_scene_id);
int32_t pgpu_free_scene(pgpu_ctx* ctx, int32_t scene_id);

/* Sizes of an uploaded scene. No counterpart in the reference (Pencil keeps
 * its scene on the host): it reports what pgpu_upload_scene built. */
typedef struct pgpu_scene_info {
    int64_t device_bytes;      /* bytes of the scene's device arena, all copied
                                  from pinned host memory by the upload      */
    int32_t n_leaves;          /* primitives (one per BVH leaf)              */
    int32_t n_interior;        /* interior nodes of the binary tree          */
    int32_t n_wide;            /* wide nodes collapsed from it               */
    int32_t bvh_depth;         /* levels of the binary tree                  */
    int32_t wide_stack;        /* traversal stack entries the wide tree needs */
    int32_t wide_width;        /* children per wide node (4 or 8)            */
} pgpu_scene_info;
int32_t pgpu_get_scene_info(pgpu_ctx* ctx, int32_t scene_id, pgpu_scene_info* out);

/* Render one image: out_rgb gets width*height*3 floats, row-major, row 0 at
 * the top, each pixel the mean of its n*n samples (the layout of
 * Renderer::render's std::vector<Color>). out_m2 (optional) gets the
 * per-pixel mean of the squared sample radiance. */
int32_t pgpu_render(pgpu_ctx* ctx, int32_t scene_id,
                    const pgpu_render_params* params,
                    float* out_rgb, float* out_m2, pgpu_stats* stats);

/* Render the window [x, x+w) x [y, y+h) of the image `params` describes:
 * every pixel is seeded, jittered and traced as in pgpu_render of the whole
 * image (the same values, bit for bit); out_rgb / out_m2 get w*h*3 floats,
 * row-major. A frame split into windows over several GPUs (tiles, rows) is
 * the fixed-frame counterpart of Pencil's tile farm, whose workers render
 * 64x64 tiles of the frame (src/distributed.hpp:642-718, 380-434). */
int32_t pgpu_render_window(pgpu_ctx* ctx, int32_t scene_id,
                           const pgpu_render_params* params, int32_t x, int32_t y,
                           int32_t w, int32_t h, float* out_rgb, float* out_m2,
                           pgpu_stats* stats);

/* Render several (scene, params) jobs of uneven size in one persistent
 * wavefront launch sequence. outs[i] receives job i's image. */
int32_t pgpu_render_batch(pgpu_ctx* ctx, int32_t n_jobs,
                          const int32_t* scene_ids,
                          const pgpu_render_params* params,
                          float* const* outs, pgpu_stats* stats);

/* Closest hit for n arbitrary rays (origin[3], direction[3] per ray;
 * directions are used as given): primitive index (unified index space,
 * -1 = miss) and hit distance, with t_min 1e-4 and t_max 1e9 as
 * Scene::hit is called (src/renderer.hpp:407). */
int32_t pgpu_trace_rays(pgpu_ctx* ctx, int32_t scene_id, const float* rays,
                        int32_t n, int32_t* prim_id, float* t);

/* Primary hits for n image-plane points (u, v): the camera ray
 * Camera::ray_at(u, v) followed by the closest hit. */
int32_t pgpu_primary_hits(pgpu_ctx* ctx, int32_t scene_id, const float* uv,
                          int32_t n, int32_t* prim_id, float* t);

/* Path-replay adjoint of a path-traced render (mode PATHTRACE, counter RNG,
 * Fresnel-split glass). Given dL/dimage (width*height*3 floats, host), it
 * accumulates dL/d(albedo) and dL/d(emission) per material (3 doubles per
 * material each) and dL/d(intensity) per light (3 doubles per light).
 * Gradient buffers are overwritten. Optional out_rgb receives the forward
 * image of the same samples. */
int32_t pgpu_adjoint(pgpu_ctx* ctx, int32_t scene_id,
                     const pgpu_render_params* params, const float* dl_dimage,
                     double* d_albedo, double* d_emission, double* d_light,
                     float* out_rgb, pgpu_stats* stats);

/* Render without allocating. No counterpart in the reference: Pencil renders
 * on the CPU and never touches device memory.
 *
 * pgpu_render may allocate device memory on the way (its output staging and
 * the wavefront's path queues grow with the image), and cudaMalloc/cudaFree
 * synchronize the device. Some callers cannot allow that while a frame is in
 * flight: a host whose device memory is owned by another allocator (a
 * framework's caching allocator that has reserved the GPU), a real-time loop
 * that must not stall on an allocation, or code that runs between
 * allocation-free phases of a larger pipeline. This entry point renders with
 * the wavefront engine over one file-scope device array of fixed size
 * (24.5 MiB: 65,536 paths in flight, processed chunk after chunk; every GPU
 * that loads the library holds it until exit). It calls no cudaMalloc,
 * cudaFree or other allocating routine; the scene must already be uploaded
 * and the outputs are caller-owned DEVICE buffers (out_rgb_device:
 * width*height*3 floats; out_m2_device optional).
 *
 * Limits, rejected with PGPU_ERR_INVALID_ARG and a message: at most 4 shadow
 * rays per path vertex (path-trace: one per light; Whitted: the soft-shadow
 * samples of every light), depth <= 64, no ray counting, profiling or ray
 * sorting. Counter RNG and Fresnel-split glass, as the wavefront engine.
 *
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) and reserves the context's error-message buffer;
 * make that first call before any stream capture. The address is kept for
 * the life of the process, so do not cudaDeviceReset a device while the
 * library is in use on it. Each call synchronizes its stream before it
 * returns, and a call made while that stream is being captured is refused
 * (PGPU_ERR_INVALID_ARG). Every call shares the one array and leaves its
 * contents behind (each call clears what it reads before it is written);
 * calls that overlap on the GPU -- from two contexts or two streams at
 * once -- race on it and must be serialized. */
int32_t pgpu_render_noalloc(pgpu_ctx* ctx, int32_t scene_id,
                            const pgpu_render_params* params,
                            float* out_rgb_device, float* out_m2_device);

/* One tile of the distributed worker (render_tile, src/distributed.hpp:
 * 380-434): params.width/height are the full image, out_rgb receives
 * tile_w*tile_h*3 floats of pixels [tile_x, tile_x+tile_w) x [tile_y,
 * tile_y+tile_h), each seeded and jittered as render_tile does (half-pixel
 * jitter). The worker traces with the Whitted tracer (params.mode
 * PGPU_MODE_WHITTED, depth = max_depth). Runs on the megakernel. */
int32_t pgpu_render_tile(pgpu_ctx* ctx, int32_t scene_id, const pgpu_render_params* params,
                         int32_t tile_x, int32_t tile_y, int32_t tile_w, int32_t tile_h,
                         float* out_rgb);

/* Pencil's output path on the device: exposure, tone curve, clamp, gamma 2.2
 * and 8 bits per channel, the bytes write_image / color_to_rgb8 produce
 * (src/image_io.hpp:40-113, src/tonemap.hpp:27-61) for the same HDR input.
 * tonemap: 0 none, 1 ACES (Pencil's default), 2 Reinhard; exposure in stops.
 * hdr: n_pixels*3 floats, out_rgb8: n_pixels*3 bytes; with
 * PGPU_TONEMAP_DEVICE_INPUT / _OUTPUT the pointers are device memory. */
enum pgpu_tonemap_flags {
    PGPU_TONEMAP_DEVICE_INPUT  = 1,
    PGPU_TONEMAP_DEVICE_OUTPUT = 2
};
int32_t pgpu_tonemap(pgpu_ctx* ctx, const float* hdr, int32_t n_pixels, int32_t tonemap,
                     float exposure, int32_t flags, uint8_t* out_rgb8);

/* Replace material table entries of an uploaded scene (same count), e.g.
 * between inverse-rendering steps. */
int32_t pgpu_update_materials(pgpu_ctx* ctx, int32_t scene_id,
                              const pgpu_material* materials, int32_t n);

#ifdef __cplusplus
}
#endif

#endif /* PENCIL_GPU_H */
