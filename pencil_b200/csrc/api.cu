// api.cu - the C-ABI of libpencil_gpu.so (include/pencil_gpu.h): contexts,
// scene upload (validation and conversion of Pencil's DFS BVH into the
// device layout of scene_layout.h), render dispatch and ray queries.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "host_internal.h"

namespace pgpu {

cudaError_t launch_megakernel(const SceneView& S, const RenderCfg& c, float* out, float* m2,
                              unsigned long long* counters, cudaStream_t st);
cudaError_t launch_query(const SceneView& S, bool camera, const float* in, int n, int* prim,
                         float* t, cudaStream_t st);

struct WfScratch;
WfScratch* wavefront_new();
void wavefront_delete(WfScratch* W);
cudaError_t wavefront_render(WfScratch& W, const std::vector<SceneView>& views,
                             const std::vector<std::vector<DevLight>>& lights,
                             const std::vector<int>& job_view, const std::vector<RenderCfg>& cfgs,
                             const std::vector<float*>& outs, const std::vector<float*>& m2s,
                             unsigned long long* counters, cudaStream_t st, bool use_graph,
                             int* launches, int* status_out, double* kernel_ms);

cudaError_t wavefront_render_static(int device, const SceneView& view, const DevLight* lights,
                                    int n_lights, bool has_glass, const RenderCfg& c, float* out,
                                    float* m2, cudaStream_t st, int* status_host, int* launches,
                                    const char** why);
size_t static_scratch_bytes();
cudaError_t launch_adjoint(const SceneView& S, const RenderCfg& c, const float* dl,
                           double* d_albedo, double* d_emission, double* d_light, float* out,
                           unsigned long long* counters, cudaStream_t st);
int adjoint_max_depth();
int adjoint_max_lights();
cudaError_t launch_tonemap(const float* d_hdr, long long n_pixels, int mode, float exposure,
                           uint8_t* d_out, const float* d_thr, cudaStream_t st);
const float* gamma_thresholds_host();
cudaError_t device_sah(const pgpu_scene& s, int n_unified, pgpu_bvh_node* out, int& depth,
                       cudaStream_t st, cudaMemPool_t pool, bool quality);
cudaError_t device_lbvh(const pgpu_scene& s, int n_unified, pgpu_bvh_node* out, int& depth,
                        cudaStream_t st, cudaMemPool_t pool);

constexpr int kMaxDepth = 64;          // traversal stack bound (kMaxStack)
constexpr int kMaxTreeFrames = 32;     // Whitted recursion bound of the two-branch mode

struct DeviceScene {
    void* arena = nullptr;             // binary nodes, leaves, vertices, materials, lights
    void* arena_wide = nullptr;        // 4-wide nodes (null when the root is a leaf)
    size_t bytes = 0;                  // both arenas
    SceneView view{};
    int n_unified = 0;
    int n_leaves = 0;
    int n_interior = 0;
    int n_wide = 0;
    int wide_stack = 0;
    int depth = 0;
    int n_materials = 0;
    bool has_glass = false;            // a dielectric material (two-branch glass needs it)
    std::vector<DevLight> lights;
    std::vector<int> quad_mats;        // material ids of quad-light emitters
    DevMaterial* d_mats = nullptr;
};

// Host mirror of Pencil's Vec3 arithmetic (src/vec3.hpp), for the camera
// basis: compiled with -ffp-contract=off, it rounds as the reference does.
struct HV {
    float x, y, z;
};
static inline HV hv(const float* p) { return HV{p[0], p[1], p[2]}; }
static inline HV operator+(HV a, HV b) { return HV{a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline HV operator-(HV a, HV b) { return HV{a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline HV operator*(HV a, float s) { return HV{a.x * s, a.y * s, a.z * s}; }
static inline HV hcross(HV a, HV b) {
    return HV{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
static inline HV hnorm(HV a) {
    float l = std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
    return (l > 1e-12f) ? HV{a.x / l, a.y / l, a.z / l} : HV{0.0f, 0.0f, 0.0f};
}

// Camera constructor: recompute_basis + recompute_frustum (src/camera.hpp:67-86).
static void camera_basis(const pgpu_camera& c, float out[21]) {
    HV eye = hv(c.eye), look = hv(c.look), up = hv(c.up);
    HV w = hnorm(eye - look);
    HV u = hnorm(hcross(up, w));
    HV v = hcross(w, u);
    float theta = c.vfov_deg * 3.14159265358979323846f / 180.0f;
    float half_h = std::tan(theta * 0.5f);
    float half_w = c.aspect * half_h;
    HV hor = u * (2.0f * half_w * c.focus_dist);
    HV ver = v * (2.0f * half_h * c.focus_dist);
    HV ll = eye - hor * 0.5f - ver * 0.5f - w * c.focus_dist;
    HV all[7] = {eye, ll, hor, ver, u, v, w};
    for (int k = 0; k < 7; ++k) {
        out[3 * k] = all[k].x;
        out[3 * k + 1] = all[k].y;
        out[3 * k + 2] = all[k].z;
    }
}

static inline bool finite3(const float* p) {
    return std::isfinite(p[0]) && std::isfinite(p[1]) && std::isfinite(p[2]);
}

}  // namespace pgpu

using namespace pgpu;

struct pgpu_ctx {
    int device = 0;
    cudaStream_t own = nullptr;
    cudaStream_t stream = nullptr;
    std::string err;
    std::map<int, std::unique_ptr<DeviceScene>> scenes;
    int next_id = 1;
    float* d_out = nullptr;
    size_t out_cap = 0;
    float* d_m2 = nullptr;
    size_t m2_cap = 0;
    unsigned long long* d_cnt = nullptr;
    void* d_query = nullptr;
    size_t query_cap = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    WfScratch* wf = nullptr;
    int* h_status = nullptr;          // pinned
    unsigned char* h_stage = nullptr; // pinned staging of scene uploads
    size_t stage_cap = 0;
    unsigned char* d_adj = nullptr;   // adjoint inputs and gradient sums
    size_t adj_cap = 0;
    uint8_t* d_rgb8 = nullptr;        // tonemap output staging
    size_t rgb8_cap = 0;
    float* d_thr = nullptr;           // tonemap gamma thresholds (256 floats)
    size_t thr_cap = 0;
    // scene arenas come from a stream-ordered pool owned by the context, so
    // that upload / free cycles reuse device memory without cudaMalloc or
    // cudaFree (each of which synchronises the device)
    cudaMemPool_t pool = nullptr;
    // host workspace of uploads, kept between calls (no page faults on reuse)
    std::vector<int> ws_idx, ws_leaf_ref;
    std::vector<int2> ws_size_height;
    std::vector<char> ws_seen;
    WideScratch ws_collapse;
    // wall-clock budget of a render's device work (pgpu_set_timeout; 0: none)
    // and whether work of a call that ran out of it may still be running
    int timeout_ms = 0;
    bool in_flight = false;
    // tree of the wide traversals of later uploads (pgpu_set_traversal_tree)
    int traversal = PGPU_TRAVERSAL_UPLOADED;
    std::vector<pgpu_bvh_node> ws_trav;
    std::vector<int> ws_leaf_of_prim;
};

namespace {

int fail(pgpu_ctx* c, int code, const char* fmt, ...) {
    if (c) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        std::vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        c->err = buf;
    }
    return code;
}

int cuda_fail(pgpu_ctx* c, cudaError_t e, const char* what) {
    return fail(c, PGPU_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// Waits for the device work recorded by c->ev1 when the context has a time
// budget: polls the event against the wall clock and, once the budget is
// spent, returns PGPU_ERR_TIMEOUT without waiting further (nothing has been
// copied to the caller's host buffers yet). The kernels themselves always
// end -- no kernel waits on a flag -- and the context's next call waits for
// them first (drain). Without a budget the caller's synchronize waits.
int wait_render(pgpu_ctx* c) {
    if (c->timeout_ms <= 0) return PGPU_OK;
    const auto t0 = std::chrono::steady_clock::now();
    while (true) {
        const cudaError_t e = cudaEventQuery(c->ev1);
        if (e == cudaSuccess) return PGPU_OK;
        if (e != cudaErrorNotReady) return cuda_fail(c, e, "waiting for the render");
        const double ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                .count();
        if (ms >= c->timeout_ms) {
            c->in_flight = true;
            return fail(c, PGPU_ERR_TIMEOUT,
                        "device work did not finish within the %d ms budget (pgpu_set_timeout)",
                        c->timeout_ms);
        }
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

// The first thing a call that uses the context's stream does: wait for work
// left running by a call that ran out of its time budget.
int drain(pgpu_ctx* c) {
    if (!c->in_flight) return PGPU_OK;
    c->in_flight = false;
    const cudaError_t e = cudaStreamSynchronize(c->stream);
    return e == cudaSuccess ? PGPU_OK : cuda_fail(c, e, "waiting for earlier device work");
}
#define PGPU_DRAIN(c)                          \
    do {                                       \
        if (int drc_ = drain(c)) return drc_;  \
    } while (0)

// f(begin, end) over [0, n) on the host worker threads (one when n is small).
template <class F>
void parallel_for(int n, F f) {
    constexpr int kGrain = 16384;
    const int T = std::min(host_threads(), (n + kGrain - 1) / kGrain);
    if (T <= 1) { f(0, n); return; }
    const int chunk = (n + T - 1) / T;
    host_run(T, [&](int t) {
        const int b = t * chunk, e = std::min(n, b + chunk);
        if (b < e) f(b, e);
    });
}

// Smallest index in [0, n) for which bad(k) holds, or -1 (threads).
template <class P>
int first_bad(int n, P bad) {
    std::atomic<int> first{n};
    parallel_for(n, [&](int b, int e) {
        for (int k = b; k < e && k < first.load(std::memory_order_relaxed); ++k)
            if (bad(k)) {
                int cur = first.load();
                while (k < cur && !first.compare_exchange_weak(cur, k)) {}
                break;
            }
    });
    return first.load() < n ? first.load() : -1;
}

// The context's stream-ordered memory pool (created on first use): scene
// arenas and device BVH builds allocate from it.
cudaError_t ensure_pool(pgpu_ctx* c) {
    if (!c->pool) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = c->device;
        cudaError_t e = cudaMemPoolCreate(&c->pool, &props);
        if (e != cudaSuccess) { c->pool = nullptr; return e; }
        // keep freed arenas for the next upload (released with the context)
        unsigned long long keep = ~0ull;
        cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    return cudaSuccess;
}

// Scene arena from the context's memory pool.
cudaError_t arena_alloc(pgpu_ctx* c, size_t bytes, void** out) {
    cudaError_t e = ensure_pool(c);
    if (e != cudaSuccess) return e;
    return cudaMallocFromPoolAsync(out, bytes, c->pool, c->stream);
}

#define PGPU_CUDA(ctx, call)                                          \
    do {                                                              \
        cudaError_t e_ = (call);                                      \
        if (e_ != cudaSuccess) return cuda_fail((ctx), e_, #call);    \
    } while (0)

template <typename T>
int ensure(pgpu_ctx* c, T*& ptr, size_t& cap, size_t need) {
    if (cap >= need && ptr) return PGPU_OK;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&ptr), std::max<size_t>(need, 256));
    if (e != cudaSuccess) {
        ptr = nullptr;
        return fail(c, PGPU_ERR_OUT_OF_MEMORY, "cudaMalloc(%zu): %s", need, cudaGetErrorString(e));
    }
    cap = std::max<size_t>(need, 256);
    return PGPU_OK;
}

DeviceScene* find_scene(pgpu_ctx* c, int id) {
    auto it = c->scenes.find(id);
    return it == c->scenes.end() ? nullptr : it->second.get();
}

// Validate Pencil's DFS node table against the unified primitive count:
// node 0 is the root, an interior node's left child is the next node and its
// right child comes later, every primitive is the leaf of exactly one node.
// A caller's material as the device reads it (area_emitter is set apart,
// from the scene's quad lights).
DevMaterial dev_material(const pgpu_material& m) {
    DevMaterial d{};
    std::memcpy(d.albedo, m.albedo, 12);
    d.kind = m.kind;
    std::memcpy(d.emission, m.emission, 12);
    d.reflectivity = m.reflectivity;
    d.ior = m.ior;
    d.specular = m.specular;
    d.shininess = m.shininess;
    std::memcpy(d.specular_color, m.specular_color, 12);
    return d;
}

int check_tree(pgpu_ctx* c, const pgpu_bvh_node* nodes, int n_nodes, int n_prims, int& depth) {
    depth = 0;
    if (n_prims == 0) {
        if (n_nodes != 0) return fail(c, PGPU_ERR_BVH_INVALID, "nodes given for an empty scene");
        return PGPU_OK;
    }
    if (n_nodes != 2 * n_prims - 1)
        return fail(c, PGPU_ERR_BVH_INVALID, "%d nodes for %d primitives (need 2n-1)", n_nodes,
                    n_prims);
    {
        const int bad = first_bad(n_nodes, [&](int k) {
            return !finite3(nodes[k].bmin) || !finite3(nodes[k].bmax);
        });
        if (bad >= 0) return fail(c, PGPU_ERR_BVH_INVALID, "node %d has a non-finite box", bad);
    }
    // DFS pre-order (the order Pencil's recursive build emits): an interior
    // node k has its left subtree at k + 1 and its right subtree right after
    // the left one. Subtree sizes, from the back, check exactly that; the
    // same sweep takes subtree heights (the root's is the depth), checks
    // that every primitive is in exactly one leaf and numbers the interior
    // nodes and the leaves in DFS order (c->ws_idx; counted from the back,
    // as a valid table has n_prims leaves and n_prims - 1 interior nodes).
    std::vector<int2>& sh = c->ws_size_height;     // (subtree size, height)
    sh.resize(n_nodes);
    std::vector<int>& idx = c->ws_idx;
    idx.resize(n_nodes);
    std::vector<char>& seen = c->ws_seen;
    seen.assign(n_prims, 0);
    int next_leaf = n_prims - 1, next_int = n_prims - 2;
    for (int k = n_nodes - 1; k >= 0; --k) {
        const pgpu_bvh_node& nd = nodes[k];
        if (nd.left < 0) {
            if (nd.right < 0 || nd.right >= n_prims)
                return fail(c, PGPU_ERR_BVH_INVALID, "leaf %d references primitive %d", k, nd.right);
            if (seen[nd.right]++)
                return fail(c, PGPU_ERR_BVH_INVALID, "primitive %d is in two leaves", nd.right);
            sh[k] = make_int2(1, 1);
            idx[k] = next_leaf--;
            continue;
        }
        idx[k] = next_int--;
        if (nd.left != k + 1 || nd.right <= nd.left || nd.right >= n_nodes ||
            nd.right != nd.left + sh[nd.left].x)
            return fail(c, PGPU_ERR_BVH_INVALID, "node %d is not in DFS pre-order", k);
        sh[k] = make_int2(1 + sh[nd.left].x + sh[nd.right].x,
                          1 + std::max(sh[nd.left].y, sh[nd.right].y));
    }
    if (sh[0].x != n_nodes) return fail(c, PGPU_ERR_BVH_INVALID, "unreachable nodes in table");
    depth = sh[0].y;
    if (depth > kMaxDepth)
        return fail(c, PGPU_ERR_UNSUPPORTED, "BVH depth %d exceeds %d", depth, kMaxDepth);
    return PGPU_OK;
}

int check_prim(pgpu_ctx* c, const pgpu_prim& p, int k, int n_mat) {
    if (p.type < PGPU_PRIM_SPHERE || p.type > PGPU_PRIM_CONE)
        return fail(c, PGPU_ERR_UNSUPPORTED, "primitive %d has unsupported type %d", k, p.type);
    if (p.material < 0 || p.material >= n_mat)
        return fail(c, PGPU_ERR_INVALID_ARG, "primitive %d uses material %d of %d", k, p.material, n_mat);
    for (int q = 0; q < 14; ++q)
        if (!std::isfinite(p.p[q]))
            return fail(c, PGPU_ERR_INVALID_ARG, "primitive %d has a non-finite parameter", k);
    return PGPU_OK;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

extern "C" {

int32_t pgpu_abi_version(void) { return PGPU_ABI_VERSION; }

int32_t pgpu_create(int32_t device, pgpu_ctx** out) {
    if (!out) return PGPU_ERR_INVALID_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return PGPU_ERR_CUDA;
    if (device < 0 || device >= n) return PGPU_ERR_INVALID_ARG;
    auto* c = new pgpu_ctx();
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
        cudaMalloc(reinterpret_cast<void**>(&c->d_cnt), CNT_N * sizeof(unsigned long long)) !=
            cudaSuccess ||
        cudaMallocHost(reinterpret_cast<void**>(&c->h_status), 16) != cudaSuccess) {
        pgpu_destroy(c);
        return PGPU_ERR_CUDA;
    }
    c->stream = c->own;
    c->wf = wavefront_new();
    *out = c;
    return PGPU_OK;
}

void pgpu_destroy(pgpu_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto& kv : c->scenes) {
        cudaFreeAsync(kv.second->arena, c->stream);
        if (kv.second->arena_wide) cudaFreeAsync(kv.second->arena_wide, c->stream);
    }
    c->scenes.clear();
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->pool) cudaMemPoolDestroy(c->pool);
    cudaFree(c->d_out);
    cudaFree(c->d_m2);
    cudaFree(c->d_cnt);
    cudaFree(c->d_query);
    cudaFree(c->d_adj);
    cudaFree(c->d_rgb8);
    cudaFree(c->d_thr);
    wavefront_delete(c->wf);
    if (c->h_status) cudaFreeHost(c->h_status);
    if (c->h_stage) cudaFreeHost(c->h_stage);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->own) cudaStreamDestroy(c->own);
    delete c;
}

const char* pgpu_last_error(const pgpu_ctx* c) { return c ? c->err.c_str() : "null context"; }

int32_t pgpu_set_stream(pgpu_ctx* c, void* stream) {
    if (!c) return PGPU_ERR_INVALID_ARG;
    PGPU_DRAIN(c);
    c->stream = stream ? static_cast<cudaStream_t>(stream) : c->own;
    return PGPU_OK;
}

void* pgpu_get_stream(pgpu_ctx* c) { return c ? static_cast<void*>(c->stream) : nullptr; }

int32_t pgpu_set_timeout(pgpu_ctx* c, int32_t ms) {
    if (!c) return PGPU_ERR_INVALID_ARG;
    if (ms < 0) return fail(c, PGPU_ERR_INVALID_ARG, "negative timeout %d ms", ms);
    c->timeout_ms = ms;
    return PGPU_OK;
}

int32_t pgpu_set_traversal_tree(pgpu_ctx* c, int32_t mode) {
    if (!c) return PGPU_ERR_INVALID_ARG;
    if (mode != PGPU_TRAVERSAL_UPLOADED && mode != PGPU_TRAVERSAL_LBVH &&
        mode != PGPU_TRAVERSAL_SAH)
        return fail(c, PGPU_ERR_INVALID_ARG, "unknown traversal tree %d", mode);
    c->traversal = mode;
    return PGPU_OK;
}

int32_t pgpu_make_prim(int32_t type, int32_t material, const float* a, const float* b,
                       const float* cc, float s0, float s1, pgpu_prim* out) {
    if (!out) return PGPU_ERR_INVALID_ARG;
    return make_prim(type, material, a, b, cc, s0, s1, out);
}

int32_t pgpu_build_bvh(const pgpu_scene* s, pgpu_bvh_node* out_nodes, int32_t* out_n_nodes,
                       int32_t* out_depth) {
    if (!s || !out_n_nodes || (s->n_prims > 0 && !s->prims) || s->n_prims < 0 ||
        s->n_mesh_triangles < 0 ||
        (s->n_mesh_triangles > 0 && (!s->mesh_indices || !s->mesh_vertices)))
        return PGPU_ERR_INVALID_ARG;
    for (int k = 0; k < 3 * s->n_mesh_triangles; ++k)
        if (s->mesh_indices[k] < 0 || s->mesh_indices[k] >= s->n_mesh_vertices)
            return PGPU_ERR_INVALID_ARG;
    std::vector<pgpu_prim> prims;
    unified_prims(*s, prims);
    std::vector<pgpu_bvh_node> nodes;
    int depth = 0;
    build_bvh(prims, nodes, depth);
    if (out_nodes) std::memcpy(out_nodes, nodes.data(), nodes.size() * sizeof(pgpu_bvh_node));
    *out_n_nodes = (int32_t)nodes.size();
    if (out_depth) *out_depth = depth;
    return PGPU_OK;
}

}  // extern "C"

// The traversal tree of an upload (PGPU_TRAVERSAL_LBVH / _SAH): built on the
// device over the scene's primitives, checked to be a DFS table over every
// primitive once, then given the uploaded tree's leaf boxes -- the builder's
// boxes are the same primitive boxes; where one differs in a bit, the
// uploaded one is taken and the interior boxes are refit as unions, so
// every box still contains its subtree's. leaf_of[p] receives the uploaded
// tree's leaf of primitive p.
static int traversal_tree(pgpu_ctx* c, const pgpu_scene& s, const pgpu_bvh_node* nodes,
                          int n_nodes, int nU, int mode, std::vector<int>& leaf_of,
                          std::vector<pgpu_bvh_node>& T) {
    leaf_of.assign(nU, -1);
    parallel_for(n_nodes, [&](int b, int e) {
        for (int k = b; k < e; ++k)
            if (nodes[k].left < 0) leaf_of[nodes[k].right] = k;
    });
    T.resize(n_nodes);
    int depth = 0;
    const cudaError_t e = mode == PGPU_TRAVERSAL_SAH
                              ? device_sah(s, nU, T.data(), depth, c->stream, c->pool, true)
                              : device_lbvh(s, nU, T.data(), depth, c->stream, c->pool);
    if (e != cudaSuccess) return cuda_fail(c, e, "traversal tree build");
    std::vector<char>& seen = c->ws_seen;
    seen.assign(nU, 0);
    std::atomic<int> bad{0}, differ{0};
    parallel_for(n_nodes, [&](int b, int e2) {
        for (int k = b; k < e2; ++k) {
            const pgpu_bvh_node& t = T[k];
            if (t.left >= 0) {
                if (t.left != k + 1 || t.right <= k + 1 || t.right >= n_nodes) bad = 1;
                continue;
            }
            if (t.right < 0 || t.right >= nU || leaf_of[t.right] < 0) { bad = 1; continue; }
            // one leaf per primitive: a primitive's flag is set by one leaf only
            if (__atomic_exchange_n(&seen[t.right], (char)1, __ATOMIC_RELAXED)) { bad = 1; continue; }
            const pgpu_bvh_node& u = nodes[leaf_of[t.right]];
            if (std::memcmp(t.bmin, u.bmin, 12) || std::memcmp(t.bmax, u.bmax, 12)) differ = 1;
        }
    });
    if (bad) return fail(c, PGPU_ERR_BVH_INVALID, "device traversal tree is not a DFS table");
    if (differ) {
        for (int k = n_nodes - 1; k >= 0; --k) {
            pgpu_bvh_node& t = T[k];
            if (t.left < 0) {
                const pgpu_bvh_node& u = nodes[leaf_of[t.right]];
                std::memcpy(t.bmin, u.bmin, 12);
                std::memcpy(t.bmax, u.bmax, 12);
                continue;
            }
            const pgpu_bvh_node &l = T[t.left], &r = T[t.right];
            for (int a = 0; a < 3; ++a) {
                t.bmin[a] = std::fmin(l.bmin[a], r.bmin[a]);
                t.bmax[a] = std::fmax(l.bmax[a], r.bmax[a]);
            }
        }
    }
    return PGPU_OK;
}

// pgpu_build_bvh_device / _sah: `sah` selects Pencil's binned SAH, else the LBVH.
static int32_t build_bvh_device(pgpu_ctx* c, const pgpu_scene* s, pgpu_bvh_node* out_nodes,
                                int32_t* out_n_nodes, int32_t* out_depth, bool sah) {
    if (!c) return PGPU_ERR_INVALID_ARG;
    PGPU_DRAIN(c);
    if (!s || !out_n_nodes || (s->n_prims > 0 && !s->prims) || s->n_prims < 0 ||
        s->n_mesh_triangles < 0 || s->n_mesh_vertices < 0 ||
        (s->n_mesh_triangles > 0 && (!s->mesh_indices || !s->mesh_vertices)))
        return fail(c, PGPU_ERR_INVALID_ARG, "bad scene arrays");
    const long long n_unified = (long long)s->n_prims + s->n_mesh_triangles;
    if (n_unified >= kMaxLeaves) return fail(c, PGPU_ERR_UNSUPPORTED, "too many primitives");
    {
        const int bad = first_bad(3 * s->n_mesh_triangles, [&](int k) {
            return s->mesh_indices[k] < 0 || s->mesh_indices[k] >= s->n_mesh_vertices;
        });
        if (bad >= 0) return fail(c, PGPU_ERR_INVALID_ARG, "mesh index %d out of range", bad);
    }
    const int n = (int)n_unified;
    *out_n_nodes = n ? 2 * n - 1 : 0;
    if (!out_nodes) return PGPU_OK;           // size query
    if (n <= 1) {                             // nothing to build: the host does it
        std::vector<pgpu_prim> prims;
        unified_prims(*s, prims);
        std::vector<pgpu_bvh_node> nodes;
        int depth = 0;
        build_bvh(prims, nodes, depth);
        std::memcpy(out_nodes, nodes.data(), nodes.size() * sizeof(pgpu_bvh_node));
        if (out_depth) *out_depth = depth;
        return PGPU_OK;
    }
    PGPU_CUDA(c, cudaSetDevice(c->device));
    PGPU_CUDA(c, ensure_pool(c));
    int depth = 0;
    cudaError_t e = sah ? device_sah(*s, n, out_nodes, depth, c->stream, c->pool, false)
                        : device_lbvh(*s, n, out_nodes, depth, c->stream, c->pool);
    if (e != cudaSuccess) return cuda_fail(c, e, "device BVH build");
    if (out_depth) *out_depth = depth;
    return PGPU_OK;
}

extern "C" {

int32_t pgpu_build_bvh_device(pgpu_ctx* c, const pgpu_scene* s, pgpu_bvh_node* out_nodes,
                              int32_t* out_n_nodes, int32_t* out_depth) {
    return build_bvh_device(c, s, out_nodes, out_n_nodes, out_depth, false);
}

int32_t pgpu_build_bvh_device_sah(pgpu_ctx* c, const pgpu_scene* s, pgpu_bvh_node* out_nodes,
                                  int32_t* out_n_nodes, int32_t* out_depth) {
    return build_bvh_device(c, s, out_nodes, out_n_nodes, out_depth, true);
}

int32_t pgpu_upload_scene(pgpu_ctx* c, const pgpu_scene* s, int32_t* out_id) {
    if (!c) return PGPU_ERR_INVALID_ARG;
    PGPU_DRAIN(c);
    if (!s || !out_id) return fail(c, PGPU_ERR_INVALID_ARG, "null scene or id pointer");
    if (s->n_prims < 0 || s->n_mesh_triangles < 0 || s->n_materials < 0 || s->n_lights < 0 ||
        s->n_nodes < 0 || s->n_mesh_vertices < 0)
        return fail(c, PGPU_ERR_INVALID_ARG, "negative count");
    if ((s->n_prims && !s->prims) || (s->n_materials && !s->materials) ||
        (s->n_lights && !s->lights) ||
        (s->n_mesh_triangles && (!s->mesh_indices || !s->mesh_vertices || !s->mesh_materials)))
        return fail(c, PGPU_ERR_INVALID_ARG, "null array with a nonzero count");
    if (s->camera.aperture != 0.0f)
        return fail(c, PGPU_ERR_UNSUPPORTED, "camera aperture (depth of field) is not supported");
    const long long n_unified = (long long)s->n_prims + s->n_mesh_triangles;
    if (n_unified >= kMaxLeaves) return fail(c, PGPU_ERR_UNSUPPORTED, "too many primitives");
    const int nU = (int)n_unified;
    {
        const int bad = first_bad(s->n_prims, [&](int k) {
            const pgpu_prim& p = s->prims[k];
            if (p.type < PGPU_PRIM_SPHERE || p.type > PGPU_PRIM_CONE) return true;
            if (p.material < 0 || p.material >= s->n_materials) return true;
            for (int q = 0; q < 14; ++q)
                if (!std::isfinite(p.p[q])) return true;
            return false;
        });
        if (bad >= 0) return check_prim(c, s->prims[bad], bad, s->n_materials);
    }
    {
        const int bad = first_bad(s->n_mesh_triangles, [&](int k) {
            for (int v = 0; v < 3; ++v) {
                const int idx = s->mesh_indices[3 * k + v];
                if (idx < 0 || idx >= s->n_mesh_vertices) return true;
            }
            return s->mesh_materials[k] < 0 || s->mesh_materials[k] >= s->n_materials;
        });
        if (bad >= 0) {
            for (int v = 0; v < 3; ++v) {
                const int idx = s->mesh_indices[3 * bad + v];
                if (idx < 0 || idx >= s->n_mesh_vertices)
                    return fail(c, PGPU_ERR_INVALID_ARG, "mesh triangle %d vertex %d out of range",
                                bad, idx);
            }
            return fail(c, PGPU_ERR_INVALID_ARG, "mesh triangle %d material out of range", bad);
        }
    }
    {
        const int bad = first_bad(s->n_mesh_vertices,
                                  [&](int k) { return !finite3(s->mesh_vertices + 3 * k); });
        if (bad >= 0) return fail(c, PGPU_ERR_INVALID_ARG, "mesh vertex %d is not finite", bad);
    }
    {
        const int bad = first_bad(s->n_materials, [&](int k) {
            const pgpu_material& m = s->materials[k];
            return m.kind < PGPU_MAT_DIFFUSE || m.kind > PGPU_MAT_DIELECTRIC || m.flags != 0;
        });
        if (bad >= 0) {
            const pgpu_material& m = s->materials[bad];
            if (m.flags != 0) return fail(c, PGPU_ERR_UNSUPPORTED, "material %d has flags set", bad);
            return fail(c, PGPU_ERR_UNSUPPORTED, "material %d has unsupported kind %d", bad, m.kind);
        }
    }
    std::vector<DevLight> lights(s->n_lights);
    std::vector<int> quad_mats;
    int has_quad = 0;
    for (int k = 0; k < s->n_lights; ++k) {
        const pgpu_light& l = s->lights[k];
        if (l.kind < PGPU_LIGHT_POINT || l.kind > PGPU_LIGHT_QUAD)
            return fail(c, PGPU_ERR_UNSUPPORTED, "light %d has unsupported kind %d", k, l.kind);
        DevLight d{};
        d.kind = l.kind;
        std::memcpy(d.pos, l.pos, 12);
        std::memcpy(d.intensity, l.intensity, 12);
        d.radius = l.radius;
        d.is_emissive = l.is_emissive;
        std::memcpy(d.edge_u, l.edge_u, 12);
        std::memcpy(d.edge_v, l.edge_v, 12);
        if (l.kind == PGPU_LIGHT_QUAD) {
            if (l.material < 0 || l.material >= s->n_materials)
                return fail(c, PGPU_ERR_INVALID_ARG, "quad light %d material out of range", k);
            HV cr = hcross(hv(l.edge_u), hv(l.edge_v));
            d.area = std::sqrt(cr.x * cr.x + cr.y * cr.y + cr.z * cr.z);
            const HV nq = hnorm(cr);     // the device's normalized(), same operations
            d.normal[0] = nq.x;
            d.normal[1] = nq.y;
            d.normal[2] = nq.z;
            if (!(d.area > 0.0f)) return fail(c, PGPU_ERR_INVALID_ARG, "quad light %d has no area", k);
            quad_mats.push_back(l.material);
            has_quad = 1;
        }
        lights[k] = d;
    }

    // BVH: caller's table (Pencil's tree) or the same tree built here
    std::vector<pgpu_bvh_node> built;
    const pgpu_bvh_node* nodes = s->nodes;
    int n_nodes = s->n_nodes;
    int depth = 0;
    if (!nodes) {
        std::vector<pgpu_prim> prims;
        unified_prims(*s, prims);
        build_bvh(prims, built, depth);
        nodes = built.data();
        n_nodes = (int)built.size();
    }
    int rc = check_tree(c, nodes, n_nodes, nU, depth);
    if (rc) return rc;

    // DFS order numbering of interior nodes and leaf slots (check_tree)
    const std::vector<int>& idx = c->ws_idx;
    const int n_leaf = nU, n_int = nU > 0 ? nU - 1 : 0;
    // triangles keep their first vertex and both edges (v1 - v0, v2 - v0, the
    // reference's first two operations, rounded alike here) in their leaf
    // slot (geo_a, geo_b, geo_c): a triangle test then loads them directly,
    // not via indices, and subtracts nothing; the w words hold the face
    // normal a hit record needs
    const bool has_tri = s->n_mesh_triangles > 0 || first_bad(s->n_prims, [&](int k) {
        return s->prims[k].type == PGPU_PRIM_TRIANGLE;
    }) >= 0;

    auto ref_of = [&](int k) -> int {
        if (nodes[k].left >= 0) return idx[k];
        int prim = nodes[k].right;
        int type = prim < s->n_prims ? s->prims[prim].type : PGPU_PRIM_TRIANGLE;
        return ~((type << kLeafTypeShift) | idx[k]);
    };

    // Staging: the main arena's bytes, then room for one wide node per
    // binary interior node (the most the collapse can make). The main part
    // is copied to the device while the wide nodes are being built.
    size_t off_nodes = 0;
    size_t off_ga = align256(off_nodes + (size_t)n_int * 64);
    size_t off_gb = align256(off_ga + (size_t)n_leaf * 16);
    size_t off_gc = align256(off_gb + (size_t)n_leaf * 16);
    const size_t gc_bytes = has_tri ? (size_t)n_leaf * 16 : 0;
    size_t off_lm = align256(off_gc + gc_bytes);
    size_t off_lp = align256(off_lm + (size_t)n_leaf * 4);
    size_t off_mt = align256(off_lp + (size_t)n_leaf * 4);
    size_t off_lt = align256(off_mt + (size_t)s->n_materials * sizeof(DevMaterial));
    size_t total = align256(off_lt + lights.size() * sizeof(DevLight));
    const size_t wide_cap = (size_t)n_int * kWideNodeFloat4 * 16;
    if (c->stage_cap < total + wide_cap) {
        if (c->h_stage) cudaFreeHost(c->h_stage);
        c->h_stage = nullptr;
        c->stage_cap = 0;
        if (cudaMallocHost(reinterpret_cast<void**>(&c->h_stage), total + wide_cap) != cudaSuccess) {
            c->h_stage = nullptr;
            return fail(c, PGPU_ERR_OUT_OF_MEMORY, "pinned staging of %zu bytes", total + wide_cap);
        }
        c->stage_cap = total + wide_cap;
    }
    unsigned char* host = c->h_stage;
    // every byte is written below except the alignment gaps; those are
    // zeroed so that uploads are deterministic
    {
        const size_t ends[][2] = {{off_nodes + (size_t)n_int * 64, off_ga},
                                  {off_ga + (size_t)n_leaf * 16, off_gb},
                                  {off_gb + (size_t)n_leaf * 16, off_gc},
                                  {off_gc + gc_bytes, off_lm},
                                  {off_lm + (size_t)n_leaf * 4, off_lp},
                                  {off_lp + (size_t)n_leaf * 4, off_mt},
                                  {off_mt + (size_t)s->n_materials * sizeof(DevMaterial), off_lt},
                                  {off_lt + lights.size() * sizeof(DevLight), total}};
        for (const auto& g : ends)
            if (g[1] > g[0]) std::memset(host + g[0], 0, g[1] - g[0]);
    }
    float4* h_nodes = reinterpret_cast<float4*>(host + off_nodes);
    float4* h_ga = reinterpret_cast<float4*>(host + off_ga);
    float4* h_gb = reinterpret_cast<float4*>(host + off_gb);
    float4* h_gc = has_tri ? reinterpret_cast<float4*>(host + off_gc) : nullptr;
    int* h_lm = reinterpret_cast<int*>(host + off_lm);
    int* h_lp = reinterpret_cast<int*>(host + off_lp);
    DevMaterial* h_mt = reinterpret_cast<DevMaterial*>(host + off_mt);
    parallel_for(s->n_materials, [&](int b, int e) {
        for (int k = b; k < e; ++k) h_mt[k] = dev_material(s->materials[k]);
    });
    for (int m : quad_mats) h_mt[m].area_emitter = 1;
    if (!lights.empty()) std::memcpy(host + off_lt, lights.data(), lights.size() * sizeof(DevLight));
    const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    auto vertex = [&](int i) {
        const float* v = s->mesh_vertices + 3 * (size_t)i;
        return make_float4(v[0], v[1], v[2], 0.0f);
    };
    // Triangle::hit's edge1 / edge2 (src/primitives.hpp:147-148): v - v0
    auto edge = [](const float4& v0, const float4& v) {
        return make_float4(v.x - v0.x, v.y - v0.y, v.z - v0.z, 0.0f);
    };
    // the triangle's face normal, normalized(edge1 x edge2) with Vec3's
    // operations in their order (src/vec3.hpp:56-68), in the w words of its
    // three slot entries
    auto put_normal = [](float4& a, float4& e1, float4& e2) {
        const float nx = e1.y * e2.z - e1.z * e2.y;
        const float ny = e1.z * e2.x - e1.x * e2.z;
        const float nz = e1.x * e2.y - e1.y * e2.x;
        const float len = std::sqrt(nx * nx + ny * ny + nz * nz);
        const bool ok = len > 1e-12f;
        a.w = ok ? nx / len : 0.0f;
        e1.w = ok ? ny / len : 0.0f;
        e2.w = ok ? nz / len : 0.0f;
    };
    auto convert = [&](int kb, int ke) {
    for (int k = kb; k < ke; ++k) {
        const pgpu_bvh_node& nd = nodes[k];
        if (nd.left >= 0) {
            const pgpu_bvh_node& L = nodes[nd.left];
            const pgpu_bvh_node& R = nodes[nd.right];
            float4* q = h_nodes + 4 * (size_t)idx[k];
            q[0] = make_float4(L.bmin[0], L.bmin[1], L.bmin[2], L.bmax[0]);
            q[1] = make_float4(L.bmax[1], L.bmax[2], R.bmin[0], R.bmin[1]);
            q[2] = make_float4(R.bmin[2], R.bmax[0], R.bmax[1], R.bmax[2]);
            int4 refs = make_int4(ref_of(nd.left), ref_of(nd.right), 0, 0);
            std::memcpy(&q[3], &refs, 16);
            continue;
        }
        const int slot = idx[k];
        const int prim = nd.right;
        h_lp[slot] = prim;
        float4 a = zero, b = zero, c = zero;
        if (prim >= s->n_prims) {
            const int t = prim - s->n_prims;
            h_lm[slot] = s->mesh_materials[t];
            a = vertex(s->mesh_indices[3 * t]);
            b = edge(a, vertex(s->mesh_indices[3 * t + 1]));
            c = edge(a, vertex(s->mesh_indices[3 * t + 2]));
            put_normal(a, b, c);
        } else {
            const pgpu_prim& p = s->prims[prim];
            const float* q = p.p;
            h_lm[slot] = p.material;
            switch (p.type) {
                case PGPU_PRIM_SPHERE:
                case PGPU_PRIM_CUBE:
                    a = make_float4(q[0], q[1], q[2], q[3]);
                    break;
                case PGPU_PRIM_TRIANGLE:
                    a = make_float4(q[0], q[1], q[2], 0.0f);
                    b = edge(a, make_float4(q[3], q[4], q[5], 0.0f));
                    c = edge(a, make_float4(q[6], q[7], q[8], 0.0f));
                    put_normal(a, b, c);
                    break;
                case PGPU_PRIM_PLANE:
                    a = make_float4(q[0], q[1], q[2], 0.0f);
                    b = make_float4(q[3], q[4], q[5], 0.0f);
                    break;
                case PGPU_PRIM_CYLINDER:
                case PGPU_PRIM_CONE:
                    a = make_float4(q[0], q[1], q[2], q[6]);
                    b = make_float4(q[3], q[4], q[5], q[7]);
                    break;
            }
        }
        h_ga[slot] = a;
        h_gb[slot] = b;
        if (h_gc) h_gc[slot] = c;
    }
    };
    parallel_for(n_nodes, convert);

    PGPU_CUDA(c, cudaSetDevice(c->device));
    auto ds = std::make_unique<DeviceScene>();
    // frees what was allocated when the upload fails from here on (stream
    // ordered: after the copies already queued)
    auto release = [&] {
        if (ds->arena) cudaFreeAsync(ds->arena, c->stream);
        if (ds->arena_wide) cudaFreeAsync(ds->arena_wide, c->stream);
        cudaStreamSynchronize(c->stream);
    };
    cudaError_t e = arena_alloc(c, total, &ds->arena);
    if (e != cudaSuccess) {
        ds->arena = nullptr;
        return fail(c, PGPU_ERR_OUT_OF_MEMORY, "scene arena of %zu bytes: %s", total,
                    cudaGetErrorString(e));
    }
    e = cudaMemcpyAsync(ds->arena, host, total, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) {
        release();
        return cuda_fail(c, e, "scene upload");
    }

    // The tree the wide traversals walk: the uploaded one, or one built on
    // the device over its leaves (pgpu_set_traversal_tree). Its leaves keep
    // the uploaded tree's leaf boxes and slots.
    const pgpu_bvh_node* tnodes = nodes;
    std::vector<int>& leaf_of = c->ws_leaf_of_prim;    // primitive -> its leaf in `nodes`
    const bool own_tree = c->traversal != PGPU_TRAVERSAL_UPLOADED && nU >= 2;
    if (own_tree) {
        rc = traversal_tree(c, *s, nodes, n_nodes, nU, c->traversal, leaf_of, c->ws_trav);
        if (rc) { release(); return rc; }
        tnodes = c->ws_trav.data();
    }
    // 4-wide nodes, built while the main part is in flight
    std::vector<int>& leaf_ref = c->ws_leaf_ref;
    leaf_ref.resize(n_nodes);
    parallel_for(n_nodes, [&](int b, int e2) {
        for (int k = b; k < e2; ++k)
            leaf_ref[k] = tnodes[k].left >= 0 ? 0
                          : ref_of(own_tree ? leaf_of[tnodes[k].right] : k);
    });
    int wide_stack = 0;
    float4* h_wide = reinterpret_cast<float4*>(host + total);
    const int n_wide = collapse_wide(tnodes, n_nodes, leaf_ref, kMaxDepth, h_wide,
                                     c->ws_collapse, wide_stack);
    if (wide_stack > kMaxDepth) {
        release();
        return fail(c, PGPU_ERR_UNSUPPORTED, "BVH needs %d stack entries, more than %d",
                    wide_stack, kMaxDepth);
    }
    const size_t wide_bytes = (size_t)n_wide * kWideNodeFloat4 * 16;
    if (n_wide) {
        e = arena_alloc(c, wide_bytes, &ds->arena_wide);
        if (e != cudaSuccess) {
            ds->arena_wide = nullptr;
            release();
            return fail(c, PGPU_ERR_OUT_OF_MEMORY, "wide-node arena of %zu bytes: %s", wide_bytes,
                        cudaGetErrorString(e));
        }
        e = cudaMemcpyAsync(ds->arena_wide, h_wide, wide_bytes, cudaMemcpyHostToDevice, c->stream);
        if (e != cudaSuccess) {
            release();
            return cuda_fail(c, e, "scene upload");
        }
    }
    // the glass flag while the copies run
    const bool has_glass = first_bad(s->n_materials, [&](int k) {
        return s->materials[k].kind == PGPU_MAT_DIELECTRIC;
    }) >= 0;
    e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        release();
        return cuda_fail(c, e, "scene upload");
    }
    ds->bytes = total + wide_bytes;
    unsigned char* base = static_cast<unsigned char*>(ds->arena);
    SceneView& v = ds->view;
    v.nodes = reinterpret_cast<const float4*>(base + off_nodes);
    v.wide = n_wide ? static_cast<const float4*>(ds->arena_wide) : nullptr;
    v.geo_a = reinterpret_cast<const float4*>(base + off_ga);
    v.geo_b = reinterpret_cast<const float4*>(base + off_gb);
    v.geo_c = has_tri ? reinterpret_cast<const float4*>(base + off_gc) : nullptr;
    v.leaf_mat = reinterpret_cast<const int*>(base + off_lm);
    v.leaf_prim = reinterpret_cast<const int*>(base + off_lp);
    v.mats = reinterpret_cast<const DevMaterial*>(base + off_mt);
    v.lights = reinterpret_cast<const DevLight*>(base + off_lt);
    v.n_lights = s->n_lights;
    v.n_leaves = n_leaf;
    v.has_quad_lights = has_quad;
    if (n_nodes == 0) {
        v.root_ref = kEmptyRoot;
    } else {
        v.root_ref = ref_of(0);
        std::memcpy(v.root_min, nodes[0].bmin, 12);
        std::memcpy(v.root_max, nodes[0].bmax, 12);
    }
    camera_basis(s->camera, v.cam);
    std::memcpy(v.bg, s->background, 12);
    std::memcpy(v.amb, s->ambient, 12);
    ds->n_unified = nU;
    ds->n_leaves = n_leaf;
    ds->n_interior = n_int;
    ds->n_wide = n_wide;
    ds->wide_stack = wide_stack;
    ds->depth = depth;
    ds->n_materials = s->n_materials;
    ds->has_glass = has_glass;
    ds->lights = std::move(lights);
    ds->quad_mats = std::move(quad_mats);
    ds->d_mats = reinterpret_cast<DevMaterial*>(base + off_mt);
    int id = c->next_id++;
    c->scenes[id] = std::move(ds);
    *out_id = id;
    return PGPU_OK;
}

int32_t pgpu_free_scene(pgpu_ctx* c, int32_t id) {
    if (!c) return PGPU_ERR_INVALID_ARG;
    PGPU_DRAIN(c);
    DeviceScene* ds = find_scene(c, id);
    if (!ds) return fail(c, PGPU_ERR_NO_SCENE, "unknown scene id %d", id);
    // work on the context stream that reads the scene finishes first; the
    // arena then returns to the pool
    cudaStreamSynchronize(c->stream);
    cudaFreeAsync(ds->arena, c->stream);
    if (ds->arena_wide) cudaFreeAsync(ds->arena_wide, c->stream);
    c->scenes.erase(id);
    return PGPU_OK;
}

int32_t pgpu_get_scene_info(pgpu_ctx* c, int32_t id, pgpu_scene_info* out) {
    if (!c) return PGPU_ERR_INVALID_ARG;
    PGPU_DRAIN(c);
    if (!out) return fail(c, PGPU_ERR_INVALID_ARG, "null info pointer");
    DeviceScene* ds = find_scene(c, id);
    if (!ds) return fail(c, PGPU_ERR_NO_SCENE, "unknown scene id %d", id);
    pgpu_scene_info info{};
    info.device_bytes = (int64_t)ds->bytes;
    info.n_leaves = ds->n_leaves;
    info.n_interior = ds->n_interior;
    info.n_wide = ds->n_wide;
    info.bvh_depth = ds->depth;
    info.wide_stack = ds->wide_stack;
    info.wide_width = kWideWidth;
    *out = info;
    return PGPU_OK;
}

int32_t pgpu_tonemap(pgpu_ctx* c, const float* hdr, int32_t n_pixels, int32_t tonemap,
                     float exposure, int32_t flags, uint8_t* out_rgb8) {
    if (!c) return PGPU_ERR_INVALID_ARG;
    PGPU_DRAIN(c);
    if (!hdr || !out_rgb8 || n_pixels < 0)
        return fail(c, PGPU_ERR_INVALID_ARG, "null buffer or negative pixel count");
    if (tonemap < 0 || tonemap > 2)
        return fail(c, PGPU_ERR_UNSUPPORTED, "tone map %d (0 none, 1 ACES, 2 Reinhard)", tonemap);
    if (!std::isfinite(exposure)) return fail(c, PGPU_ERR_INVALID_ARG, "exposure is not finite");
    if (n_pixels == 0) return PGPU_OK;
    PGPU_CUDA(c, cudaSetDevice(c->device));
    const size_t n3 = (size_t)n_pixels * 3;
    const float* d_in = hdr;
    if (!(flags & PGPU_TONEMAP_DEVICE_INPUT)) {
        int rc = ensure(c, c->d_out, c->out_cap, n3 * 4);
        if (rc) return rc;
        PGPU_CUDA(c, cudaMemcpyAsync(c->d_out, hdr, n3 * 4, cudaMemcpyHostToDevice, c->stream));
        d_in = c->d_out;
    }
    uint8_t* d_dst = out_rgb8;
    if (!(flags & PGPU_TONEMAP_DEVICE_OUTPUT)) {
        int rc = ensure(c, c->d_rgb8, c->rgb8_cap, n3);
        if (rc) return rc;
        d_dst = c->d_rgb8;
    }
    if (!c->d_thr) {
        int rc = ensure(c, c->d_thr, c->thr_cap, 256 * sizeof(float));
        if (rc) return rc;
        PGPU_CUDA(c, cudaMemcpy(c->d_thr, gamma_thresholds_host(), 256 * sizeof(float),
                                cudaMemcpyHostToDevice));
    }
    PGPU_CUDA(c, launch_tonemap(d_in, n_pixels, tonemap, exposure, d_dst, c->d_thr, c->stream));
    if (!(flags & PGPU_TONEMAP_DEVICE_OUTPUT))
        PGPU_CUDA(c, cudaMemcpyAsync(out_rgb8, d_dst, n3, cudaMemcpyDeviceToHost, c->stream));
    PGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    return PGPU_OK;
}

int32_t pgpu_update_materials(pgpu_ctx* c, int32_t id, const pgpu_material* m, int32_t n) {
    if (!c) return PGPU_ERR_INVALID_ARG;
    PGPU_DRAIN(c);
    DeviceScene* ds = find_scene(c, id);
    if (!ds) return fail(c, PGPU_ERR_NO_SCENE, "unknown scene id %d", id);
    if (!m || n != ds->n_materials)
        return fail(c, PGPU_ERR_INVALID_ARG, "material count %d, scene has %d", n, ds->n_materials);
    std::vector<DevMaterial> mats(n);
    bool has_glass = false;
    for (int k = 0; k < n; ++k) {
        if (m[k].kind < PGPU_MAT_DIFFUSE || m[k].kind > PGPU_MAT_DIELECTRIC || m[k].flags != 0)
            return fail(c, PGPU_ERR_UNSUPPORTED, "material %d unsupported", k);
        mats[k] = dev_material(m[k]);
        has_glass = has_glass || m[k].kind == PGPU_MAT_DIELECTRIC;
    }
    for (int q : ds->quad_mats) mats[q].area_emitter = 1;
    PGPU_CUDA(c, cudaMemcpyAsync(ds->d_mats, mats.data(), mats.size() * sizeof(DevMaterial),
                                 cudaMemcpyHostToDevice, c->stream));
    PGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    ds->has_glass = has_glass;
    return PGPU_OK;
}

}  // extern "C"

namespace pgpu {

// Validate render parameters; fills cfg.
int make_cfg(pgpu_ctx* c, const DeviceScene* ds, const pgpu_render_params* p, RenderCfg& cfg) {
    if (!p) return fail(c, PGPU_ERR_INVALID_ARG, "null render params");
    if (p->width <= 0 || p->height <= 0 || p->samples <= 0 || p->depth < 0)
        return fail(c, PGPU_ERR_INVALID_ARG, "bad size %dx%d, samples %d, depth %d", p->width,
                    p->height, p->samples, p->depth);
    if ((long long)p->width * p->height > (1LL << 28) || p->samples > 64)
        return fail(c, PGPU_ERR_INVALID_ARG, "image of %dx%d with n=%d is too large", p->width,
                    p->height, p->samples);
    if (p->mode != PGPU_MODE_PATHTRACE && p->mode != PGPU_MODE_WHITTED)
        return fail(c, PGPU_ERR_INVALID_ARG, "unknown mode %d", p->mode);
    if (p->engine != PGPU_ENGINE_WAVEFRONT && p->engine != PGPU_ENGINE_MEGAKERNEL)
        return fail(c, PGPU_ERR_INVALID_ARG, "unknown engine %d", p->engine);
    if (p->rng != PGPU_RNG_COUNTER && p->rng != PGPU_RNG_PIXEL_SEQUENTIAL)
        return fail(c, PGPU_ERR_INVALID_ARG, "unknown rng %d", p->rng);
    if (p->glass != PGPU_GLASS_FRESNEL_SPLIT && p->glass != PGPU_GLASS_BOTH_BRANCHES)
        return fail(c, PGPU_ERR_INVALID_ARG, "unknown glass mode %d", p->glass);
    if (!(p->shadow_bias >= 0.0f) || p->soft_shadow_samples <= 0 || p->sample_offset < 0)
        return fail(c, PGPU_ERR_INVALID_ARG, "bad shadow bias, soft-shadow samples or offset");
    if (p->engine == PGPU_ENGINE_WAVEFRONT &&
        (p->rng != PGPU_RNG_COUNTER || p->glass != PGPU_GLASS_FRESNEL_SPLIT))
        return fail(c, PGPU_ERR_UNSUPPORTED,
                    "the wavefront engine needs the counter RNG and Fresnel-split glass");
    if (p->glass == PGPU_GLASS_BOTH_BRANCHES && p->depth > kMaxTreeFrames)
        return fail(c, PGPU_ERR_UNSUPPORTED, "two-branch glass supports depth <= %d", kMaxTreeFrames);
    cfg.W = p->width;
    cfg.H = p->height;
    cfg.n = p->samples;
    cfg.spp = p->samples * p->samples;
    cfg.depth = p->depth;
    cfg.mode = p->mode;
    cfg.engine = p->engine;
    cfg.rng = p->rng;
    cfg.glass = p->glass;
    cfg.soft = p->soft_shadow_samples;
    cfg.bias = p->shadow_bias;
    cfg.salt = p->seed;
    cfg.sample_offset = p->sample_offset;
    cfg.count = (p->flags & (PGPU_FLAG_COUNT_RAYS | PGPU_FLAG_COUNT_NODES)) != 0;
    if (p->refill_below < 0 || p->refill_below > 31)
        return fail(c, PGPU_ERR_INVALID_ARG, "refill_below must be 0..31");
    cfg.refill = p->refill_below;
    if (p->queue_capacity < 0 || p->queue_capacity > (1 << 28))
        return fail(c, PGPU_ERR_INVALID_ARG, "queue_capacity must be 0..2^28 paths");
    cfg.queue_capacity = p->queue_capacity;
    if (p->sort_key < 0 || p->sort_key > 3)
        return fail(c, PGPU_ERR_INVALID_ARG, "sort_key must be 0..3");
    cfg.sort_key = p->sort_key;
    cfg.profile = (p->flags & PGPU_FLAG_PROFILE_KERNELS) != 0;
    cfg.packets = (p->flags & PGPU_FLAG_NO_PACKETS) == 0;
    cfg.mis = (p->flags & PGPU_FLAG_MIS) != 0;
    cfg.binary_tree = (p->flags & PGPU_FLAG_BINARY_TREE) != 0;
    if (p->block_size != 0 && p->block_size != 64 && p->block_size != 128 && p->block_size != 256)
        return fail(c, PGPU_ERR_INVALID_ARG, "block_size must be 0, 64, 128 or 256");
    cfg.block = p->block_size;
    cfg.win[0] = cfg.win[1] = cfg.win[2] = cfg.win[3] = 0;
    cfg.worker = false;
    (void)ds;
    return PGPU_OK;
}

// Run jobs through the wavefront engine; checks the device status word.
int run_wavefront(pgpu_ctx* c, const std::vector<DeviceScene*>& scenes,
                  const std::vector<RenderCfg>& cfgs, const std::vector<float*>& outs,
                  const std::vector<float*>& m2s, bool use_graph, int* launches,
                  double* kernel_ms) {
    std::vector<SceneView> views;
    std::vector<std::vector<DevLight>> lights;
    std::vector<int> job_view;
    std::map<const DeviceScene*, int> vidx;
    for (auto* ds : scenes) {
        auto it = vidx.find(ds);
        if (it == vidx.end()) {
            int k = (int)views.size();
            vidx[ds] = k;
            views.push_back(ds->view);
            lights.push_back(ds->lights);
            job_view.push_back(k);
        } else {
            job_view.push_back(it->second);
        }
    }
    *c->h_status = 0;
    cudaError_t e = wavefront_render(*c->wf, views, lights, job_view, cfgs, outs, m2s, c->d_cnt,
                                     c->stream, use_graph, launches, c->h_status, kernel_ms);
    if (e != cudaSuccess) return cuda_fail(c, e, "wavefront launch");
    return PGPU_OK;
}

// pgpu_render and pgpu_render_window: the image, or the window `win` of it.
static int32_t render_impl(pgpu_ctx* c, int32_t id, const pgpu_render_params* p,
                           const int32_t* win, float* out_rgb, float* out_m2, pgpu_stats* stats) {
    auto t0 = std::chrono::steady_clock::now();
    if (!c) return PGPU_ERR_INVALID_ARG;
    PGPU_DRAIN(c);
    DeviceScene* ds = find_scene(c, id);
    if (!ds) return fail(c, PGPU_ERR_NO_SCENE, "unknown scene id %d", id);
    if (!out_rgb) return fail(c, PGPU_ERR_INVALID_ARG, "null output");
    RenderCfg cfg;
    int rc = make_cfg(c, ds, p, cfg);
    if (rc) return rc;
    if (win) {
        if (win[2] <= 0 || win[3] <= 0 || win[0] < 0 || win[1] < 0 || win[0] + win[2] > cfg.W ||
            win[1] + win[3] > cfg.H)
            return fail(c, PGPU_ERR_INVALID_ARG, "window %d,%d %dx%d outside the %dx%d image",
                        win[0], win[1], win[2], win[3], cfg.W, cfg.H);
        for (int k = 0; k < 4; ++k) cfg.win[k] = win[k];
    }
    PGPU_CUDA(c, cudaSetDevice(c->device));
    const bool dev_out = (p->flags & PGPU_FLAG_DEVICE_OUTPUT) != 0;
    const size_t n3 = (size_t)cfg.pixels() * 3;
    float* d_out = dev_out ? out_rgb : nullptr;
    float* d_m2 = dev_out ? out_m2 : nullptr;
    if (!dev_out) {
        if ((rc = ensure(c, c->d_out, c->out_cap, n3 * 4))) return rc;
        d_out = c->d_out;
        if (out_m2) {
            if ((rc = ensure(c, c->d_m2, c->m2_cap, n3 * 4))) return rc;
            d_m2 = c->d_m2;
        }
    }
    if (cfg.count)
        PGPU_CUDA(c, cudaMemsetAsync(c->d_cnt, 0, CNT_N * sizeof(unsigned long long), c->stream));
    int launches = 1;
    double kms[KC_N] = {0};
    PGPU_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    cudaError_t e;
    if (cfg.engine == PGPU_ENGINE_MEGAKERNEL) {
        e = launch_megakernel(ds->view, cfg, d_out, d_m2, c->d_cnt, c->stream);
        if (e != cudaSuccess) return cuda_fail(c, e, "megakernel launch");
    } else {
        *c->h_status = 0;
        rc = run_wavefront(c, {ds}, {cfg}, {d_out}, {d_m2}, (p->flags & PGPU_FLAG_NO_GRAPH) == 0,
                           &launches, cfg.profile ? kms : nullptr);
        if (rc) return rc;
    }
    PGPU_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    if ((rc = wait_render(c))) return rc;
    if (!dev_out) {
        PGPU_CUDA(c, cudaMemcpyAsync(out_rgb, d_out, n3 * 4, cudaMemcpyDeviceToHost, c->stream));
        if (out_m2)
            PGPU_CUDA(c, cudaMemcpyAsync(out_m2, d_m2, n3 * 4, cudaMemcpyDeviceToHost, c->stream));
    }
    unsigned long long cnt[CNT_N] = {0};
    if (cfg.count)
        PGPU_CUDA(c, cudaMemcpyAsync(cnt, c->d_cnt, sizeof(cnt), cudaMemcpyDeviceToHost, c->stream));
    PGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    if (cfg.engine == PGPU_ENGINE_WAVEFRONT && *c->h_status != 0)
        return fail(c, PGPU_ERR_QUEUE_OVERFLOW, "shadow record queue overflow");
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        stats->device_ms = ms;
        stats->paths = (uint64_t)cfg.pixels() * cfg.spp;
        stats->extension_rays = cnt[CNT_EXT];
        stats->shadow_rays = cnt[CNT_SHADOW];
        stats->reference_rays = cnt[CNT_REF];
        stats->node_visits = cnt[CNT_NODES];
        stats->prim_tests = cnt[CNT_PRIMS];
        stats->ext_node_visits = cnt[CNT_NODES_EXT];
        stats->ext_leaf_bytes = cnt[CNT_LEAF_EXT];
        stats->shadow_node_visits = cnt[CNT_NODES_SH];
        stats->shadow_leaf_bytes = cnt[CNT_LEAF_SH];
        if (cfg.engine == PGPU_ENGINE_MEGAKERNEL && cfg.profile) kms[KC_MEGAKERNEL] = ms;
        for (int k = 0; k < KC_N; ++k) stats->kernel_ms[k] = kms[k];
        stats->kernel_launches = launches;
        stats->total_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return PGPU_OK;
}

}  // namespace pgpu

extern "C" {

int32_t pgpu_render(pgpu_ctx* c, int32_t id, const pgpu_render_params* p, float* out_rgb,
                    float* out_m2, pgpu_stats* stats) {
    return render_impl(c, id, p, nullptr, out_rgb, out_m2, stats);
}

int32_t pgpu_render_window(pgpu_ctx* c, int32_t id, const pgpu_render_params* p, int32_t x,
                           int32_t y, int32_t w, int32_t h, float* out_rgb, float* out_m2,
                           pgpu_stats* stats) {
    const int32_t win[4] = {x, y, w, h};
    return render_impl(c, id, p, win, out_rgb, out_m2, stats);
}

int32_t pgpu_render_tile(pgpu_ctx* c, int32_t id, const pgpu_render_params* p, int32_t tile_x,
                         int32_t tile_y, int32_t tile_w, int32_t tile_h, float* out_rgb) {
    if (!c) return PGPU_ERR_INVALID_ARG;
    PGPU_DRAIN(c);
    DeviceScene* ds = find_scene(c, id);
    if (!ds) return fail(c, PGPU_ERR_NO_SCENE, "unknown scene id %d", id);
    if (!out_rgb) return fail(c, PGPU_ERR_INVALID_ARG, "null output");
    pgpu_render_params q = *p;
    q.engine = PGPU_ENGINE_MEGAKERNEL;     // tiles run on the megakernel
    RenderCfg cfg;
    int rc = make_cfg(c, ds, &q, cfg);
    if (rc) return rc;
    if (tile_w <= 0 || tile_h <= 0 || tile_x < 0 || tile_y < 0 || tile_x + tile_w > cfg.W ||
        tile_y + tile_h > cfg.H)
        return fail(c, PGPU_ERR_INVALID_ARG, "tile %d,%d %dx%d outside the %dx%d image", tile_x,
                    tile_y, tile_w, tile_h, cfg.W, cfg.H);
    cfg.count = false;
    PGPU_CUDA(c, cudaSetDevice(c->device));
    const bool dev_out = (p->flags & PGPU_FLAG_DEVICE_OUTPUT) != 0;
    const size_t n3 = (size_t)tile_w * tile_h * 3;
    float* d_out = out_rgb;
    if (!dev_out) {
        if ((rc = ensure(c, c->d_out, c->out_cap, n3 * 4))) return rc;
        d_out = c->d_out;
    }
    cfg.win[0] = tile_x;
    cfg.win[1] = tile_y;
    cfg.win[2] = tile_w;
    cfg.win[3] = tile_h;
    cfg.worker = true;
    cudaError_t e = launch_megakernel(ds->view, cfg, d_out, nullptr, c->d_cnt, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "megakernel launch");
    if (!dev_out)
        PGPU_CUDA(c, cudaMemcpyAsync(out_rgb, d_out, n3 * 4, cudaMemcpyDeviceToHost, c->stream));
    PGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    return PGPU_OK;
}

int32_t pgpu_render_batch(pgpu_ctx* c, int32_t n_jobs, const int32_t* ids,
                          const pgpu_render_params* params, float* const* outs, pgpu_stats* stats) {
    auto t0 = std::chrono::steady_clock::now();
    if (!c) return PGPU_ERR_INVALID_ARG;
    PGPU_DRAIN(c);
    if (n_jobs <= 0 || !ids || !params || !outs)
        return fail(c, PGPU_ERR_INVALID_ARG, "bad batch arguments");
    std::vector<DeviceScene*> scenes(n_jobs);
    std::vector<RenderCfg> cfgs(n_jobs);
    size_t total = 0;
    bool dev_out = (params[0].flags & PGPU_FLAG_DEVICE_OUTPUT) != 0;
    for (int k = 0; k < n_jobs; ++k) {
        scenes[k] = find_scene(c, ids[k]);
        if (!scenes[k]) return fail(c, PGPU_ERR_NO_SCENE, "job %d: unknown scene id %d", k, ids[k]);
        int rc = make_cfg(c, scenes[k], &params[k], cfgs[k]);
        if (rc) return rc;
        if (cfgs[k].engine != PGPU_ENGINE_WAVEFRONT)
            return fail(c, PGPU_ERR_UNSUPPORTED, "job %d: batches run on the wavefront engine", k);
        if (((params[k].flags & PGPU_FLAG_DEVICE_OUTPUT) != 0) != dev_out)
            return fail(c, PGPU_ERR_INVALID_ARG, "jobs mix host and device outputs");
        if (!outs[k]) return fail(c, PGPU_ERR_INVALID_ARG, "job %d: null output", k);
        total += (size_t)cfgs[k].W * cfgs[k].H * 3;
    }
    PGPU_CUDA(c, cudaSetDevice(c->device));
    std::vector<float*> d_outs(n_jobs), d_m2s(n_jobs, nullptr);
    if (dev_out) {
        for (int k = 0; k < n_jobs; ++k) d_outs[k] = outs[k];
    } else {
        int rc = ensure(c, c->d_out, c->out_cap, total * 4);
        if (rc) return rc;
        size_t off = 0;
        for (int k = 0; k < n_jobs; ++k) {
            d_outs[k] = c->d_out + off;
            off += (size_t)cfgs[k].W * cfgs[k].H * 3;
        }
    }
    bool count = false;
    for (auto& cf : cfgs) count = count || cf.count;
    if (count) PGPU_CUDA(c, cudaMemsetAsync(c->d_cnt, 0, CNT_N * sizeof(unsigned long long), c->stream));
    int launches = 0;
    PGPU_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    double kms[KC_N] = {0};
    const bool prof = (params[0].flags & PGPU_FLAG_PROFILE_KERNELS) != 0;
    int rc = run_wavefront(c, scenes, cfgs, d_outs, d_m2s, (params[0].flags & PGPU_FLAG_NO_GRAPH) == 0,
                           &launches, prof ? kms : nullptr);
    if (rc) return rc;
    PGPU_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    if ((rc = wait_render(c))) return rc;
    if (!dev_out)
        for (int k = 0; k < n_jobs; ++k)
            PGPU_CUDA(c, cudaMemcpyAsync(outs[k], d_outs[k], (size_t)cfgs[k].W * cfgs[k].H * 12,
                                         cudaMemcpyDeviceToHost, c->stream));
    unsigned long long cnt[CNT_N] = {0};
    if (count)
        PGPU_CUDA(c, cudaMemcpyAsync(cnt, c->d_cnt, sizeof(cnt), cudaMemcpyDeviceToHost, c->stream));
    PGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    if (*c->h_status != 0) return fail(c, PGPU_ERR_QUEUE_OVERFLOW, "shadow record queue overflow");
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        stats->device_ms = ms;
        for (auto& cf : cfgs) stats->paths += (uint64_t)cf.W * cf.H * cf.spp;
        stats->extension_rays = cnt[CNT_EXT];
        stats->shadow_rays = cnt[CNT_SHADOW];
        stats->reference_rays = cnt[CNT_REF];
        stats->node_visits = cnt[CNT_NODES];
        stats->prim_tests = cnt[CNT_PRIMS];
        stats->ext_node_visits = cnt[CNT_NODES_EXT];
        stats->ext_leaf_bytes = cnt[CNT_LEAF_EXT];
        stats->shadow_node_visits = cnt[CNT_NODES_SH];
        stats->shadow_leaf_bytes = cnt[CNT_LEAF_SH];
        for (int k = 0; k < KC_N; ++k) stats->kernel_ms[k] = kms[k];
        stats->kernel_launches = launches;
        stats->total_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return PGPU_OK;
}

int32_t pgpu_adjoint(pgpu_ctx* c, int32_t id, const pgpu_render_params* p, const float* dl,
                     double* d_albedo, double* d_emission, double* d_light, float* out_rgb,
                     pgpu_stats* stats) {
    auto t0 = std::chrono::steady_clock::now();
    if (!c) return PGPU_ERR_INVALID_ARG;
    PGPU_DRAIN(c);
    DeviceScene* ds = find_scene(c, id);
    if (!ds) return fail(c, PGPU_ERR_NO_SCENE, "unknown scene id %d", id);
    if (!dl || !d_albedo || !d_emission || (!d_light && !ds->lights.empty()))
        return fail(c, PGPU_ERR_INVALID_ARG, "null adjoint buffer");
    RenderCfg cfg;
    int rc = make_cfg(c, ds, p, cfg);
    if (rc) return rc;
    if (cfg.rng != PGPU_RNG_COUNTER || cfg.glass != PGPU_GLASS_FRESNEL_SPLIT)
        return fail(c, PGPU_ERR_UNSUPPORTED, "the adjoint replays the counter-RNG, Fresnel-split estimator");
    if (cfg.depth > adjoint_max_depth())
        return fail(c, PGPU_ERR_UNSUPPORTED, "adjoint depth is limited to %d", adjoint_max_depth());
    if (cfg.mis)
        return fail(c, PGPU_ERR_UNSUPPORTED, "the adjoint replays trace_path's light weights, not MIS");
    if ((int)ds->lights.size() > adjoint_max_lights())
        return fail(c, PGPU_ERR_UNSUPPORTED, "adjoint supports at most %d lights", adjoint_max_lights());
    PGPU_CUDA(c, cudaSetDevice(c->device));
    const size_t n3 = (size_t)cfg.W * cfg.H * 3;
    const size_t nm = (size_t)ds->n_materials, nl = ds->lights.size();
    const size_t grad_b = (2 * nm + nl) * 3 * sizeof(double);
    const size_t need = align256(n3 * 4) + align256(n3 * 4) + align256(grad_b);
    if ((rc = ensure(c, c->d_adj, c->adj_cap, need))) return rc;
    float* d_dl = reinterpret_cast<float*>(c->d_adj);
    float* d_img = reinterpret_cast<float*>(c->d_adj + align256(n3 * 4));
    double* d_g = reinterpret_cast<double*>(c->d_adj + 2 * align256(n3 * 4));
    PGPU_CUDA(c, cudaMemcpyAsync(d_dl, dl, n3 * 4, cudaMemcpyHostToDevice, c->stream));
    PGPU_CUDA(c, cudaMemsetAsync(d_g, 0, grad_b, c->stream));
    if (cfg.count)
        PGPU_CUDA(c, cudaMemsetAsync(c->d_cnt, 0, CNT_N * sizeof(unsigned long long), c->stream));
    PGPU_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    cudaError_t e = launch_adjoint(ds->view, cfg, d_dl, d_g, d_g + 3 * nm, d_g + 6 * nm,
                                   out_rgb ? d_img : nullptr, c->d_cnt, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "adjoint launch");
    PGPU_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    if ((rc = wait_render(c))) return rc;
    PGPU_CUDA(c, cudaMemcpyAsync(d_albedo, d_g, nm * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    PGPU_CUDA(c, cudaMemcpyAsync(d_emission, d_g + 3 * nm, nm * 3 * sizeof(double),
                                 cudaMemcpyDeviceToHost, c->stream));
    if (nl)
        PGPU_CUDA(c, cudaMemcpyAsync(d_light, d_g + 6 * nm, nl * 3 * sizeof(double),
                                     cudaMemcpyDeviceToHost, c->stream));
    if (out_rgb)
        PGPU_CUDA(c, cudaMemcpyAsync(out_rgb, d_img, n3 * 4, cudaMemcpyDeviceToHost, c->stream));
    unsigned long long cnt[CNT_N] = {0};
    if (cfg.count)
        PGPU_CUDA(c, cudaMemcpyAsync(cnt, c->d_cnt, sizeof(cnt), cudaMemcpyDeviceToHost, c->stream));
    PGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        stats->device_ms = ms;
        stats->paths = (uint64_t)cfg.W * cfg.H * cfg.spp;
        stats->extension_rays = cnt[CNT_EXT];
        stats->shadow_rays = cnt[CNT_SHADOW];
        stats->reference_rays = cnt[CNT_REF];
        stats->kernel_launches = 1;
        stats->total_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return PGPU_OK;
}

static int32_t run_query(pgpu_ctx* c, int32_t id, bool camera, const float* in, int32_t n,
                         int32_t* prim, float* t) {
    if (!c) return PGPU_ERR_INVALID_ARG;
    PGPU_DRAIN(c);
    DeviceScene* ds = find_scene(c, id);
    if (!ds) return fail(c, PGPU_ERR_NO_SCENE, "unknown scene id %d", id);
    if (n < 0 || (n > 0 && (!in || !prim || !t))) return fail(c, PGPU_ERR_INVALID_ARG, "bad query");
    if (n == 0) return PGPU_OK;
    PGPU_CUDA(c, cudaSetDevice(c->device));
    const size_t in_b = (size_t)n * (camera ? 2 : 6) * 4;
    const size_t need = align256(in_b) + 2 * align256((size_t)n * 4);
    int rc = ensure(c, reinterpret_cast<unsigned char*&>(c->d_query), c->query_cap, need);
    if (rc) return rc;
    unsigned char* b = static_cast<unsigned char*>(c->d_query);
    float* d_in = reinterpret_cast<float*>(b);
    int* d_prim = reinterpret_cast<int*>(b + align256(in_b));
    float* d_t = reinterpret_cast<float*>(b + align256(in_b) + align256((size_t)n * 4));
    PGPU_CUDA(c, cudaMemcpyAsync(d_in, in, in_b, cudaMemcpyHostToDevice, c->stream));
    cudaError_t e = launch_query(ds->view, camera, d_in, n, d_prim, d_t, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "query launch");
    PGPU_CUDA(c, cudaMemcpyAsync(prim, d_prim, (size_t)n * 4, cudaMemcpyDeviceToHost, c->stream));
    PGPU_CUDA(c, cudaMemcpyAsync(t, d_t, (size_t)n * 4, cudaMemcpyDeviceToHost, c->stream));
    PGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    return PGPU_OK;
}

int32_t pgpu_trace_rays(pgpu_ctx* c, int32_t id, const float* rays, int32_t n, int32_t* prim,
                        float* t) {
    return run_query(c, id, false, rays, n, prim, t);
}

int32_t pgpu_primary_hits(pgpu_ctx* c, int32_t id, const float* uv, int32_t n, int32_t* prim,
                          float* t) {
    return run_query(c, id, true, uv, n, prim, t);
}

}  // extern "C"

// ---- render without allocating ------------------------------------------------------
// For callers that must not allocate device memory while rendering (see
// pencil_gpu.h). The first call on a device looks up the static scratch's
// address and reserves the context's error-message buffer; after that no call
// allocates host or device memory.
extern "C" int32_t pgpu_render_noalloc(pgpu_ctx* c, int32_t id, const pgpu_render_params* p,
                                       float* out_rgb_device, float* out_m2_device) {
    if (!c) return PGPU_ERR_INVALID_ARG;
    PGPU_DRAIN(c);
    if (c->err.capacity() < 512) c->err.reserve(512);
    DeviceScene* ds = find_scene(c, id);
    if (!ds) return fail(c, PGPU_ERR_NO_SCENE, "unknown scene id %d", id);
    if (!out_rgb_device) return fail(c, PGPU_ERR_INVALID_ARG, "null output");
    RenderCfg cfg;
    int rc = make_cfg(c, ds, p, cfg);
    if (rc) return rc;
    if (cfg.engine != PGPU_ENGINE_WAVEFRONT)
        return fail(c, PGPU_ERR_UNSUPPORTED, "the no-allocation render is the wavefront engine");
    PGPU_CUDA(c, cudaSetDevice(c->device));
    // The call stages its scene view and job from host stack memory and
    // synchronizes its stream before it returns; neither survives a capture.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    PGPU_CUDA(c, cudaStreamIsCapturing(c->stream, &cap));
    if (cap != cudaStreamCaptureStatusNone)
        return fail(c, PGPU_ERR_INVALID_ARG,
                    "pgpu_render_noalloc was called while its stream is being captured");
    const char* why = nullptr;
    int launches = 0;
    const bool has_glass = ds->has_glass;
    *c->h_status = 0;
    cudaError_t e = wavefront_render_static(c->device, ds->view, ds->lights.data(),
                                            (int)ds->lights.size(), has_glass, cfg, out_rgb_device,
                                            out_m2_device, c->stream, c->h_status, &launches,
                                            &why);
    if (why) return fail(c, PGPU_ERR_INVALID_ARG, "%s", why);
    if (e != cudaSuccess) return cuda_fail(c, e, "no-allocation render");
    PGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    if (*c->h_status != 0) return fail(c, PGPU_ERR_QUEUE_OVERFLOW, "shadow record overflow");
    return PGPU_OK;
}
