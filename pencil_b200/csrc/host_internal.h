// host_internal.h - declarations shared by the host-side translation units
// of libpencil_gpu.so.
#pragma once

#include <cstdint>
#include <functional>
#include <vector>

#include "../../include/pencil_gpu.h"
#include "scene_layout.h"

namespace pgpu {

// bvh_build.cpp
void unified_prims(const pgpu_scene& s, std::vector<pgpu_prim>& out);
void build_bvh(const std::vector<pgpu_prim>& prims, std::vector<pgpu_bvh_node>& nodes,
               int& depth);
int make_prim(int type, int material, const float* a, const float* b, const float* c, float s0,
              float s1, pgpu_prim* out);

// host_pool.cpp: task(0 .. n-1) on the process's host worker threads and the
// calling thread (up to 16 in all, started once); returns when every task
// has run. Tasks must not call host_run themselves.
int host_threads();
void host_run(int n, const std::function<void(int)>& task);

// Scratch memory of collapse_wide, kept by the caller between calls so that
// repeated uploads reuse it instead of faulting in fresh pages.
struct WideScratch {
    std::vector<std::vector<float4>> local;   // one block per subtree task
};

// bvh_wide.cpp: 4-wide nodes (kWideNodeFloat4 float4 each) collapsed from a
// validated binary tree in DFS pre-order, written to the front of `out`,
// which must hold one wide node per binary interior node (there are never
// more). leaf_ref[k] is the leaf ref of binary leaf k. Returns the number of
// wide nodes (0 when the root is a leaf); stack_need receives the most stack
// entries a traversal holds, which is at most max_stack unless the binary
// tree itself needs more.
int collapse_wide(const pgpu_bvh_node* nodes, int n_nodes, const std::vector<int>& leaf_ref,
                  int max_stack, float4* out, WideScratch& scratch, int& stack_need);

// Render configuration after validation.
struct RenderCfg {
    int W, H, n, spp, depth, mode, engine, rng, glass, soft;
    float bias;
    uint32_t salt;
    int sample_offset;
    bool count;
    int refill;
    int queue_capacity;
    int sort_key;
    bool profile;
    bool packets;     // wavefront: camera rays of a one-scene frame as warp packets
    bool mis;         // trace_path_mis's light weights
    bool binary_tree; // megakernel: Pencil's binary tree instead of the 4-wide tree
    int block;        // wavefront threads per block (0: the default)
    int win[4];       // window x, y, w, h of the image (w = 0: the whole image)
    bool worker;      // the distributed worker's jitter (render_tile)
    long long pixels() const { return win[2] > 0 ? (long long)win[2] * win[3] : (long long)W * H; }
};

// Device counters written by the kernels (atomic adds).
enum DevCounter {
    CNT_EXT = 0,
    CNT_SHADOW = 1,
    CNT_REF = 2,
    CNT_NODES = 3,
    CNT_LEAF_BYTES = 4,
    CNT_PRIMS = 5,
    CNT_NODES_EXT = 6,
    CNT_LEAF_EXT = 7,
    CNT_NODES_SH = 8,
    CNT_LEAF_SH = 9,
    CNT_N = 16
};

// Kernel classes of pgpu_stats.kernel_ms.
enum KernelClass { KC_GENERATE = 0, KC_EXTEND, KC_SHADE, KC_SHADOW, KC_ACCUMULATE, KC_MEGAKERNEL, KC_N };

}  // namespace pgpu
