// bvh_device.cu - a BVH built on the GPU, in Pencil's table format.
//
// Pencil builds a binned-SAH tree on the host (src/bvh.hpp:54-192); for
// scenes that change every frame, or many scenes at once, that build can
// cost more than the render. This builds a linear BVH instead: primitive
// boxes (Primitive::aabb, src/primitives.hpp), 30-bit Morton codes of the box
// centres over the scene's centre bounds, a radix sort of (code, index), the
// binary radix tree over the sorted codes (Karras 2012: each internal node
// finds its key range from the longest common prefixes of its neighbours),
// boxes and subtree sizes bottom-up (the second child to arrive at a node
// merges, so no thread waits), then every node's DFS pre-order index from
// the sizes on its path to the root. The result is a pgpu_bvh_node table in
// DFS pre-order with one primitive per leaf -- the format of Pencil's tree and
// of pgpu_build_bvh -- that pgpu_upload_scene takes as it is. It is a
// different tree from Pencil's: a ray reaches the same primitives, so hits
// agree except where two surfaces tie within rounding.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_segmented_radix_sort.cuh>

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cstdint>
#include <vector>

#include "host_internal.h"

namespace pgpu {

namespace {

struct DBox {
    float mn[3], mx[3];
};

// Primitive::aabb of every kind (as bvh_build.cpp's prim_box).
__device__ DBox prim_box_dev(const pgpu_prim& p) {
    DBox b;
    const float* q = p.p;
    for (int k = 0; k < 3; ++k) { b.mn[k] = 1e30f; b.mx[k] = -1e30f; }
    switch (p.type) {
        case PGPU_PRIM_SPHERE:
        case PGPU_PRIM_CUBE:
            for (int k = 0; k < 3; ++k) { b.mn[k] = q[k] - q[3]; b.mx[k] = q[k] + q[3]; }
            break;
        case PGPU_PRIM_TRIANGLE:
            for (int k = 0; k < 3; ++k) {
                b.mn[k] = fminf(fminf(q[k], q[3 + k]), q[6 + k]);
                b.mx[k] = fmaxf(fmaxf(q[k], q[3 + k]), q[6 + k]);
            }
            break;
        case PGPU_PRIM_PLANE:
            for (int k = 0; k < 3; ++k) { b.mn[k] = -1e6f; b.mx[k] = 1e6f; }
            break;
        case PGPU_PRIM_CYLINDER: {
            const float r = q[6], hh = q[7];
            for (int k = 0; k < 3; ++k) {
                const float ext = fabsf(q[3 + k] * hh) + r;
                b.mn[k] = q[k] - ext;
                b.mx[k] = q[k] + ext;
            }
            break;
        }
        case PGPU_PRIM_CONE: {
            const float r = q[6], h = q[7];
            for (int k = 0; k < 3; ++k) {
                const float base = q[k] - q[3 + k] * h;
                b.mn[k] = fminf(q[k], base) - r;
                b.mx[k] = fmaxf(q[k], base) + r;
            }
            break;
        }
        default:
            break;
    }
    return b;
}

// Boxes of the unified primitives: prims first, then mesh triangles.
__global__ void lb_boxes(const pgpu_prim* prims, int n_prims, const float* verts,
                         const int* idx, int n_tri, DBox* boxes) {
    const int n = n_prims + n_tri;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        if (k < n_prims) {
            boxes[k] = prim_box_dev(prims[k]);
        } else {
            const int t = k - n_prims;
            DBox b;
            for (int a = 0; a < 3; ++a) {
                const float x0 = verts[3 * idx[3 * t] + a], x1 = verts[3 * idx[3 * t + 1] + a],
                            x2 = verts[3 * idx[3 * t + 2] + a];
                b.mn[a] = fminf(fminf(x0, x1), x2);
                b.mx[a] = fmaxf(fmaxf(x0, x1), x2);
            }
            boxes[k] = b;
        }
    }
}

// Order-preserving int image of a float (for atomic min/max).
__device__ __forceinline__ int ord(float f) {
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float unord(int i) {
    return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff);
}

// Bounds of the box centres (bounds[0..2] min, [3..5] max, as ord ints).
__global__ void lb_centre_bounds(const DBox* boxes, int n, int* bounds) {
    int mn[3] = {INT_MAX, INT_MAX, INT_MAX}, mx[3] = {INT_MIN, INT_MIN, INT_MIN};
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        for (int a = 0; a < 3; ++a) {
            const int c = ord(0.5f * (boxes[k].mn[a] + boxes[k].mx[a]));
            mn[a] = min(mn[a], c);
            mx[a] = max(mx[a], c);
        }
    }
    for (int a = 0; a < 3; ++a) {
        for (int off = 16; off > 0; off >>= 1) {
            mn[a] = min(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], off));
            mx[a] = max(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], off));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(bounds + a, mn[a]);
            atomicMax(bounds + 3 + a, mx[a]);
        }
    }
}

__device__ __forceinline__ uint32_t spread10(uint32_t x) {
    x &= 0x3ffu;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

// key = Morton code of the box centre << 32 | primitive index (unique keys).
__global__ void lb_keys(const DBox* boxes, int n, const int* bounds, unsigned long long* keys) {
    float lo[3], scale[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = unord(bounds[a]);
        const float ext = unord(bounds[3 + a]) - lo[a];
        scale[a] = ext > 0.0f ? 1024.0f / ext : 0.0f;
    }
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        uint32_t c[3];
        for (int a = 0; a < 3; ++a) {
            const float f = (0.5f * (boxes[k].mn[a] + boxes[k].mx[a]) - lo[a]) * scale[a];
            const int q = f > 0.0f ? (int)f : 0;
            c[a] = (uint32_t)min(q, 1023);
        }
        const uint32_t m = spread10(c[0]) | (spread10(c[1]) << 1) | (spread10(c[2]) << 2);
        keys[k] = ((unsigned long long)m << 32) | (unsigned long long)(uint32_t)k;
    }
}

// Length of the common prefix of sorted keys i and j (-1 outside [0, n)).
__device__ __forceinline__ int delta(const unsigned long long* keys, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    return __clzll(keys[i] ^ keys[j]);   // keys are unique, so i != j gives < 64
}

// Internal nodes 0..n-2 (node 0 the root), leaves n-1..2n-2 (leaf of sorted
// position s is node n-1+s). Sets both children and their parents.
__global__ void lb_tree(const unsigned long long* keys, int n, int* left, int* right,
                        int* parent) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n - 1; i += gridDim.x * blockDim.x) {
        const int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
        const int dmin = delta(keys, n, i, i - d);
        int lmax = 2;
        // ends once i + lmax * d leaves [0, n) (delta -1 there)
        while (lmax < (1 << 29) && delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
        int l = 0;
        for (int t = lmax >> 1; t >= 1; t >>= 1)
            if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
        const int j = i + l * d;
        const int dnode = delta(keys, n, i, j);
        int s = 0;
        for (int t = l, k = 0; k < 32; ++k) {   // t = ceil(l/2), ceil(l/4), ..., 1
            t = (t + 1) >> 1;
            if (s + t < l && delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
            if (t <= 1) break;
        }
        const int g = i + s * d + min(d, 0);
        const int lo = min(i, j), hi = max(i, j);
        const int lc = (lo == g) ? (n - 1 + g) : g;
        const int rc = (hi == g + 1) ? (n - 1 + g + 1) : g + 1;
        left[i] = lc;
        right[i] = rc;
        parent[lc] = i;
        parent[rc] = i;
    }
}

// Boxes and subtree sizes from the leaves up: the second child to arrive at
// a node merges the two and continues; the first stops.
__global__ void lb_refit(const DBox* boxes, const unsigned long long* keys, int n,
                         const int* left, const int* right, const int* parent, DBox* nbox,
                         int* size, int* arrivals) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        int node = n - 1 + s;
        nbox[node] = boxes[(int)(keys[s] & 0xffffffffull)];
        size[node] = 1;
        // at most n - 1 steps up (a guard only: the tree has no cycles)
        for (int step = 0; node != 0 && step < n; ++step) {
            __threadfence();
            const int p = parent[node];
            if (p < 0 || p >= n - 1) break;
            if (atomicAdd(arrivals + p, 1) == 0) break;   // the sibling is not done yet
            __threadfence();
            const int l = left[p], r = right[p];
            // the sibling was written on another SM: read through L2
            const float* fa = reinterpret_cast<const float*>(nbox + l);
            const float* fb = reinterpret_cast<const float*>(nbox + r);
            DBox m;
            for (int k = 0; k < 3; ++k) {
                m.mn[k] = fminf(__ldcg(fa + k), __ldcg(fb + k));
                m.mx[k] = fmaxf(__ldcg(fa + 3 + k), __ldcg(fb + 3 + k));
            }
            nbox[p] = m;
            size[p] = 1 + __ldcg(size + l) + __ldcg(size + r);
            node = p;
        }
    }
}

// DFS pre-order index and level of every node from the sizes on its path to
// the root; then the table row.
__global__ void lb_emit(const unsigned long long* keys, int n, const int* left,
                        const int* right, const int* parent, const DBox* nbox, const int* size,
                        int* pre, int* level, int* max_level) {
    const int total = 2 * n - 1;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < total; v += gridDim.x * blockDim.x) {
        int idx = 0, lvl = 1, x = v;
        // at most n steps (a guard only: the tree has no cycles)
        for (int step = 0; x != 0 && step < n; ++step) {
            const int p = parent[x];
            if (p < 0 || p >= n - 1) break;
            idx += (left[p] == x) ? 1 : 1 + size[left[p]];
            ++lvl;
            x = p;
        }
        pre[v] = idx;
        level[v] = lvl;
        atomicMax(max_level, lvl);
    }
}

__global__ void lb_write(const unsigned long long* keys, int n, const int* left, const int* right,
                         const DBox* nbox, const int* pre, pgpu_bvh_node* out) {
    const int total = 2 * n - 1;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < total; v += gridDim.x * blockDim.x) {
        pgpu_bvh_node r;
        for (int k = 0; k < 3; ++k) { r.bmin[k] = nbox[v].mn[k]; r.bmax[k] = nbox[v].mx[k]; }
        if (v < n - 1) {
            r.left = pre[left[v]];
            r.right = pre[right[v]];
        } else {
            r.left = -1;
            r.right = (int)(keys[v - (n - 1)] & 0xffffffffull);
        }
        const int at = pre[v];
        if (at >= 0 && at < total) out[at] = r;
    }
}

// Build memory from the context's stream-ordered pool, returned to it on
// the build's stream when the build ends (no device-wide synchronisation,
// and a repeated build reuses the pool's memory).
struct DevBuf {
    void* p = nullptr;
    cudaStream_t st = nullptr;
    cudaError_t alloc(size_t bytes, cudaMemPool_t pool, cudaStream_t s) {
        st = s;
        return cudaMallocFromPoolAsync(&p, bytes, pool, s);
    }
    ~DevBuf() { if (p) cudaFreeAsync(p, st); }
};

// ---- binned SAH on the device ------------------------------------------------------
// Pencil's own build (BVH::build_range / sah_split / median_split,
// src/bvh.hpp:74-192; bvh_build.cpp restates it on the host), top down, one
// level of the tree at a time, every node of the level at once:
//   bin        the primitives of every node with more than 4 into 12 buckets
//              along its longest axis by box centre (bins in shared memory,
//              then one atomic per bin field and block)
//   choose     per node the bucket boundary of least cost
//              1 + (nL SA_L + nR SA_R) / SA_P from prefix and suffix merges of
//              the bins, with the reference's operations in its order
//   partition  stable, by bucket (Pencil's std::partition is not stable: the
//              two orders differ only inside each side, which decides nothing
//              but ties of a later median split)
//   children   the two ranges, their boxes (the prefix / suffix merges, equal
//              to the merge of their primitives' boxes) and their DFS
//              pre-order indices (a subtree over c primitives has 2c - 1 nodes)
// Nodes of 2 to 4 primitives finish in one thread each with Pencil's median
// split (sort by centroid sum, split at the middle) down to the leaves; a
// larger node whose axis has no extent, or whose primitives all fall in one
// bucket, takes the median split over its whole range (a segmented sort).
constexpr int kSahBuckets = 12;
constexpr int kSahChunk = 1024;    // primitives per block of the bin / partition passes
constexpr int kSahBlock = 256;
// The quality variant (traversal trees, not Pencil's tree): buckets over the
// node's centroid bounds rather than its box, on all three axes.
constexpr int kQualBuckets = 16;
template <bool Q> constexpr int kBinsPerTask = Q ? 3 * kQualBuckets : kSahBuckets;

struct SahTask {                   // a node with more than 4 primitives
    int start, count;              // its range of the permutation
    int node, level;               // DFS pre-order index, level (root 1)
    float mn[3], mx[3];            // its box
};
struct SahSmall {                  // a node with 2 to 4 primitives
    int start, count, node, level;
};
struct SahBin {
    int count;
    int mn[3], mx[3];              // ord() images
};
struct SahChoice {
    int mode;                      // 0 bucket split, 1 median split
    int axis, best, nl;
    float lmn[3], lmx[3], rmn[3], rmx[3];
};

__device__ __forceinline__ int sah_axis(const float* mn, const float* mx) {
    const float ex = mx[0] - mn[0], ey = mx[1] - mn[1], ez = mx[2] - mn[2];
    if (ex >= ey && ex >= ez) return 0;
    if (ey >= ez) return 1;
    return 2;
}
__device__ __forceinline__ float sah_area(const float* mn, const float* mx) {
    const float ex = mx[0] - mn[0], ey = mx[1] - mn[1], ez = mx[2] - mn[2];
    return 2.0f * (ex * ey + ey * ez + ex * ez);
}
__device__ __forceinline__ int sah_bucket(const DBox& b, int axis, float lo, float hi) {
    const float center = (b.mn[axis] + b.mx[axis]) * 0.5f;
    int k = (int)((center - lo) / (hi - lo) * kSahBuckets);
    if (k < 0) k = 0;
    if (k >= kSahBuckets) k = kSahBuckets - 1;
    return k;
}
// Quality variant: bucket of a box centre over the node's centroid bounds
// cb (ord() images: min x y z, max x y z) along `axis`.
__device__ __forceinline__ int qual_bucket(const DBox& b, int axis, const int* cb) {
    const float lo = unord(cb[axis]), hi = unord(cb[3 + axis]);
    const float center = (b.mn[axis] + b.mx[axis]) * 0.5f;
    int k = (int)((center - lo) / (hi - lo) * kQualBuckets);
    if (k < 0) k = 0;
    if (k >= kQualBuckets) k = kQualBuckets - 1;
    return k;
}
// The bucket a primitive of task t falls in along the chosen axis.
template <bool Q>
__device__ __forceinline__ int task_bucket(const DBox& b, int axis, const SahTask& tk,
                                           const int* cb_task) {
    if constexpr (Q) return qual_bucket(b, axis, cb_task);
    else return sah_bucket(b, axis, tk.mn[axis], tk.mx[axis]);
}
__device__ __forceinline__ float sah_key2(const DBox& b, int axis) {
    return b.mn[axis] + b.mx[axis];
}

// Task of a work item (items are the tasks' chunks, task after task).
__device__ __forceinline__ int item_task(const int* item_off, int T, int item) {
    int lo = 0, hi = T - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (item_off[mid] <= item) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void sah_chunks(const SahTask* tasks, int T, int* nchunk) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x)
        nchunk[t] = (tasks[t].count + kSahChunk - 1) / kSahChunk;
}

__global__ void sah_bins_init(SahBin* bins, int n) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        SahBin b;
        b.count = 0;
        for (int a = 0; a < 3; ++a) { b.mn[a] = ord(1e30f); b.mx[a] = ord(-1e30f); }
        bins[k] = b;
    }
}

// Quality variant: the centroid bounds of every task (ord() images), one
// block per item, one atomic per bound and block.
__global__ void sah_cb_init(int* cb, int n) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        cb[k] = (k % 6) < 3 ? ord(1e30f) : ord(-1e30f);
}
__global__ void __launch_bounds__(kSahBlock)
sah_cbounds(const SahTask* tasks, int T, const int* item_off, const int* nchunk, const int* perm,
            const DBox* boxes, int* cb) {
    const int items = item_off[T - 1] + nchunk[T - 1];
    if ((int)blockIdx.x >= items) return;
    const int t = item_task(item_off, T, blockIdx.x);
    const SahTask tk = tasks[t];
    const int begin = tk.start + (blockIdx.x - item_off[t]) * kSahChunk;
    const int end = min(begin + kSahChunk, tk.start + tk.count);
    int mn[3] = {INT_MAX, INT_MAX, INT_MAX}, mx[3] = {INT_MIN, INT_MIN, INT_MIN};
    for (int p = begin + threadIdx.x; p < end; p += blockDim.x) {
        const DBox b = boxes[perm[p]];
        for (int a = 0; a < 3; ++a) {
            const int c = ord((b.mn[a] + b.mx[a]) * 0.5f);
            mn[a] = min(mn[a], c);
            mx[a] = max(mx[a], c);
        }
    }
    for (int a = 0; a < 3; ++a) {
        for (int off = 16; off > 0; off >>= 1) {
            mn[a] = min(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], off));
            mx[a] = max(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], off));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(cb + 6 * t + a, mn[a]);
            atomicMax(cb + 6 * t + 3 + a, mx[a]);
        }
    }
}

// One block per item: the chunk's primitives into the task's bins -- 12
// along the longest axis of its box (Pencil), or 16 per axis over its
// centroid bounds on each axis where they have an extent (quality).
template <bool Q>
__global__ void __launch_bounds__(kSahBlock)
sah_bin(const SahTask* tasks, int T, const int* item_off, const int* nchunk, const int* perm,
        const DBox* boxes, const int* cb, SahBin* bins) {
    constexpr int NB = kBinsPerTask<Q>;
    __shared__ int s_cnt[NB], s_mn[NB][3], s_mx[NB][3];
    const int items = item_off[T - 1] + nchunk[T - 1];
    if ((int)blockIdx.x >= items) return;
    const int t = item_task(item_off, T, blockIdx.x);
    const SahTask tk = tasks[t];
    const int axis = sah_axis(tk.mn, tk.mx);
    bool on_axis[3] = {false, false, false};
    if constexpr (Q) {
        for (int a = 0; a < 3; ++a) on_axis[a] = unord(cb[6 * t + 3 + a]) > unord(cb[6 * t + a]);
        if (!on_axis[0] && !on_axis[1] && !on_axis[2]) return;   // median split: no bins
    } else {
        if (!(tk.mx[axis] > tk.mn[axis])) return;                 // median split: no bins
    }
    for (int k = threadIdx.x; k < NB; k += blockDim.x) {
        s_cnt[k] = 0;
        for (int a = 0; a < 3; ++a) {
            s_mn[k][a] = ord(1e30f);
            s_mx[k][a] = ord(-1e30f);
        }
    }
    __syncthreads();
    const int begin = tk.start + (blockIdx.x - item_off[t]) * kSahChunk;
    const int end = min(begin + kSahChunk, tk.start + tk.count);
    for (int p = begin + threadIdx.x; p < end; p += blockDim.x) {
        const DBox b = boxes[perm[p]];
        auto put = [&](int k) {
            atomicAdd(&s_cnt[k], 1);
            for (int a = 0; a < 3; ++a) {
                atomicMin(&s_mn[k][a], ord(b.mn[a]));
                atomicMax(&s_mx[k][a], ord(b.mx[a]));
            }
        };
        if constexpr (Q) {
            for (int ax = 0; ax < 3; ++ax)
                if (on_axis[ax]) put(ax * kQualBuckets + qual_bucket(b, ax, cb + 6 * t));
        } else {
            put(sah_bucket(b, axis, tk.mn[axis], tk.mx[axis]));
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < NB; k += blockDim.x) {
        if (s_cnt[k] == 0) continue;
        SahBin* g = bins + (size_t)t * NB + k;
        atomicAdd(&g->count, s_cnt[k]);
        for (int a = 0; a < 3; ++a) {
            atomicMin(&g->mn[a], s_mn[k][a]);
            atomicMax(&g->mx[a], s_mx[k][a]);
        }
    }
}

// The cheapest boundary among `nb` bins (prefix / suffix merges, cost
// 1 + (nL SA_L + nR SA_R) / SA_P with the reference's operations in its
// order); updates c and best_cost when a boundary beats best_cost.
__device__ __forceinline__ void sah_best_boundary(const SahBin* b, int nb, int axis,
                                                  float sa_parent, SahChoice& c,
                                                  float& best_cost) {
    float pmn[kQualBuckets + 1][3], pmx[kQualBuckets + 1][3];
    float smn[kQualBuckets + 1][3], smx[kQualBuckets + 1][3];
    int pc[kQualBuckets + 1], sc[kQualBuckets + 1];
    for (int a = 0; a < 3; ++a) {
        pmn[0][a] = smn[nb][a] = 1e30f;
        pmx[0][a] = smx[nb][a] = -1e30f;
    }
    pc[0] = sc[nb] = 0;
    for (int i = 0; i < nb; ++i) {
        for (int a = 0; a < 3; ++a) {
            pmn[i + 1][a] = fminf(pmn[i][a], unord(b[i].mn[a]));
            pmx[i + 1][a] = fmaxf(pmx[i][a], unord(b[i].mx[a]));
        }
        pc[i + 1] = pc[i] + b[i].count;
    }
    for (int i = nb - 1; i >= 0; --i) {
        for (int a = 0; a < 3; ++a) {
            smn[i][a] = fminf(smn[i + 1][a], unord(b[i].mn[a]));
            smx[i][a] = fmaxf(smx[i + 1][a], unord(b[i].mx[a]));
        }
        sc[i] = sc[i + 1] + b[i].count;
    }
    for (int i = 1; i < nb; ++i) {
        const int nL = pc[i], nR = sc[i];
        if (nL == 0 || nR == 0) continue;
        const float sa_l = sah_area(pmn[i], pmx[i]);
        const float sa_r = sah_area(smn[i], smx[i]);
        const float cost =
            1.0f + ((float)nL * sa_l + (float)nR * sa_r) / (sa_parent > 0 ? sa_parent : 1.0f);
        if (cost < best_cost) {
            best_cost = cost;
            c.mode = 0;
            c.axis = axis;
            c.best = i;
            c.nl = nL;
            for (int a = 0; a < 3; ++a) {
                c.lmn[a] = pmn[i][a];
                c.lmx[a] = pmx[i][a];
                c.rmn[a] = smn[i][a];
                c.rmx[a] = smx[i][a];
            }
        }
    }
}

// One thread per task: sah_split's choice (src/bvh.hpp:119-192) -- or, in
// the quality variant, the best boundary over the three axes' bins -- or the
// median split along the box's longest axis when no boundary separates.
template <bool Q>
__global__ void sah_choose(const SahTask* tasks, int T, const SahBin* bins, const int* cb,
                           SahChoice* ch, int* fb_list, int* n_fb) {
    constexpr int NB = kBinsPerTask<Q>;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x) {
        const SahTask tk = tasks[t];
        SahChoice c;
        c.axis = sah_axis(tk.mn, tk.mx);
        c.mode = 1;
        c.best = -1;
        c.nl = tk.count / 2;
        float best_cost = FLT_MAX;
        const float sa_parent = sah_area(tk.mn, tk.mx);
        const SahBin* b = bins + (size_t)t * NB;
        if constexpr (Q) {
            for (int ax = 0; ax < 3; ++ax)
                if (unord(cb[6 * t + 3 + ax]) > unord(cb[6 * t + ax]))
                    sah_best_boundary(b + ax * kQualBuckets, kQualBuckets, ax, sa_parent, c,
                                      best_cost);
            if (c.mode == 1) c.axis = sah_axis(tk.mn, tk.mx);
        } else {
            if (tk.mx[c.axis] > tk.mn[c.axis])
                sah_best_boundary(b, kSahBuckets, c.axis, sa_parent, c, best_cost);
        }
        ch[t] = c;
        if (c.mode == 1) fb_list[atomicAdd(n_fb, 1)] = t;
    }
}

// Stable partition of bucket-split tasks, pass 1: left-side count of each item.
template <bool Q>
__global__ void __launch_bounds__(kSahBlock)
sah_part_count(const SahTask* tasks, int T, const int* item_off, const int* nchunk,
               const SahChoice* ch, const int* perm, const DBox* boxes, const int* cb,
               int* left_cnt) {
    __shared__ int s_sum[kSahBlock / 32];
    const int items = item_off[T - 1] + nchunk[T - 1];
    if ((int)blockIdx.x >= items) return;
    const int t = item_task(item_off, T, blockIdx.x);
    const SahTask tk = tasks[t];
    const SahChoice c = ch[t];
    int cnt = 0;
    if (c.mode == 0) {
        const int begin = tk.start + (blockIdx.x - item_off[t]) * kSahChunk;
        const int end = min(begin + kSahChunk, tk.start + tk.count);
        for (int p = begin + threadIdx.x; p < end; p += blockDim.x)
            cnt += task_bucket<Q>(boxes[perm[p]], c.axis, tk, cb + 6 * t) < c.best ? 1 : 0;
    }
    for (int off = 16; off > 0; off >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, off);
    if ((threadIdx.x & 31) == 0) s_sum[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        int sum = 0;
        for (int w = 0; w < kSahBlock / 32; ++w) sum += s_sum[w];
        left_cnt[blockIdx.x] = sum;
    }
}

// Pass 2: every primitive of a bucket-split task to its place in `out`, the
// left side first, each side in the order of `perm`.
template <bool Q>
__global__ void __launch_bounds__(kSahBlock)
sah_part_write(const SahTask* tasks, int T, const int* item_off, const int* nchunk,
               const SahChoice* ch, const int* perm, const DBox* boxes, const int* cb,
               const int* left_off, int* out) {
    __shared__ int s_warp[kSahBlock / 32];
    const int items = item_off[T - 1] + nchunk[T - 1];
    if ((int)blockIdx.x >= items) return;
    const int t = item_task(item_off, T, blockIdx.x);
    const SahTask tk = tasks[t];
    const SahChoice c = ch[t];
    if (c.mode != 0) return;
    const int first_item = item_off[t];
    const int chunk0 = tk.start + (blockIdx.x - first_item) * kSahChunk;
    const int end = min(chunk0 + kSahChunk, tk.start + tk.count);
    // lefts before this item within the task, and rights likewise
    int lbase = left_off[blockIdx.x] - left_off[first_item];
    int rbase = (chunk0 - tk.start) - lbase;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int p0 = chunk0; p0 < end; p0 += blockDim.x) {
        const int p = p0 + threadIdx.x;
        const bool on = p < end;
        const int prim = on ? perm[p] : 0;
        const bool left = on && task_bucket<Q>(boxes[prim], c.axis, tk, cb + 6 * t) < c.best;
        const unsigned m = __ballot_sync(0xffffffffu, left);
        if (lane == 0) s_warp[warp] = __popc(m);
        __syncthreads();
        int before = 0, total = 0;
        for (int w = 0; w < kSahBlock / 32; ++w) {
            if (w < warp) before += s_warp[w];
            total += s_warp[w];
        }
        const int lrank = before + __popc(m & ((1u << lane) - 1u));
        const int nvalid = min((int)blockDim.x, end - p0);
        // (the bins counted the same buckets, so every place lies in the task's
        // range; the bound is checked all the same)
        const int at = left ? tk.start + lbase + lrank : tk.start + c.nl + rbase + (threadIdx.x - lrank);
        if (on && at >= tk.start && at < tk.start + tk.count) out[at] = prim;
        lbase += total;
        rbase += nvalid - total;
        __syncthreads();
    }
}

// Pass 3: the partitioned ranges back into `perm`.
__global__ void sah_part_copy(const SahTask* tasks, int T, const int* item_off,
                              const int* nchunk, const SahChoice* ch, const int* src, int* dst) {
    const int items = item_off[T - 1] + nchunk[T - 1];
    if ((int)blockIdx.x >= items) return;
    const int t = item_task(item_off, T, blockIdx.x);
    if (ch[t].mode != 0) return;
    const SahTask tk = tasks[t];
    const int begin = tk.start + (blockIdx.x - item_off[t]) * kSahChunk;
    const int end = min(begin + kSahChunk, tk.start + tk.count);
    for (int p = begin + threadIdx.x; p < end; p += blockDim.x) dst[p] = src[p];
}

// Median-split tasks: sizes, then the (centroid sum, primitive) pairs of
// their ranges side by side for a segmented sort.
__global__ void sah_fb_sizes(const SahTask* tasks, const int* fb, int n_fb, int* sizes) {
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < n_fb; f += gridDim.x * blockDim.x)
        sizes[f] = tasks[fb[f]].count;
}
__global__ void sah_fb_gather(const SahTask* tasks, const SahChoice* ch, const int* fb,
                              const int* fb_off, const int* perm, const DBox* boxes,
                              float* keys, int* vals) {
    const int f = blockIdx.x;
    const SahTask tk = tasks[fb[f]];
    const int axis = ch[fb[f]].axis;
    for (int i = threadIdx.x; i < tk.count; i += blockDim.x) {
        const int prim = perm[tk.start + i];
        keys[fb_off[f] + i] = sah_key2(boxes[prim], axis);
        vals[fb_off[f] + i] = prim;
    }
}
// The sorted ranges back into `perm`, and the boxes of their two halves.
__global__ void sah_fb_scatter(const SahTask* tasks, SahChoice* ch, const int* fb,
                               const int* fb_off, const int* vals, int* perm, const DBox* boxes) {
    __shared__ int s_box[2][6];
    const int f = blockIdx.x;
    const int t = fb[f];
    const SahTask tk = tasks[t];
    const int half = tk.count / 2;
    if (threadIdx.x < 2) {
        for (int a = 0; a < 3; ++a) {
            s_box[threadIdx.x][a] = ord(1e30f);
            s_box[threadIdx.x][3 + a] = ord(-1e30f);
        }
    }
    __syncthreads();
    int mn[2][3], mx[2][3];
    for (int h = 0; h < 2; ++h)
        for (int a = 0; a < 3; ++a) { mn[h][a] = ord(1e30f); mx[h][a] = ord(-1e30f); }
    for (int i = threadIdx.x; i < tk.count; i += blockDim.x) {
        const int prim = vals[fb_off[f] + i];
        perm[tk.start + i] = prim;
        const int h = i < half ? 0 : 1;
        for (int a = 0; a < 3; ++a) {
            mn[h][a] = min(mn[h][a], ord(boxes[prim].mn[a]));
            mx[h][a] = max(mx[h][a], ord(boxes[prim].mx[a]));
        }
    }
    for (int h = 0; h < 2; ++h)
        for (int a = 0; a < 3; ++a) {
            atomicMin(&s_box[h][a], mn[h][a]);
            atomicMax(&s_box[h][3 + a], mx[h][a]);
        }
    __syncthreads();
    if (threadIdx.x == 0) {
        SahChoice c = ch[t];
        c.nl = half;
        for (int a = 0; a < 3; ++a) {
            c.lmn[a] = unord(s_box[0][a]);
            c.lmx[a] = unord(s_box[0][3 + a]);
            c.rmn[a] = unord(s_box[1][a]);
            c.rmx[a] = unord(s_box[1][3 + a]);
        }
        ch[t] = c;
    }
}

__device__ __forceinline__ void sah_write(pgpu_bvh_node* nodes, int total, int at,
                                          const float* mn, const float* mx, int left, int right) {
    if (at < 0 || at >= total) return;         // a guard only: the indices stay in the table
    pgpu_bvh_node r;
    for (int a = 0; a < 3; ++a) { r.bmin[a] = mn[a]; r.bmax[a] = mx[a]; }
    r.left = left;
    r.right = right;
    nodes[at] = r;
}

// One thread per task: the node's row, and its two children -- a leaf, a
// small task (2 to 4 primitives) or a task of the next level.
__global__ void sah_children(const SahTask* tasks, int T, const SahChoice* ch, const int* perm,
                             SahTask* next, int* n_next, SahSmall* small, int* n_small,
                             pgpu_bvh_node* nodes, int total, int* max_level) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x) {
        const SahTask tk = tasks[t];
        const SahChoice c = ch[t];
        const int nl = c.nl, nr = tk.count - c.nl;
        const int lnode = tk.node + 1, rnode = tk.node + 2 * nl;
        sah_write(nodes, total, tk.node, tk.mn, tk.mx, lnode, rnode);
        for (int side = 0; side < 2; ++side) {
            const int cnt = side ? nr : nl;
            const int start = side ? tk.start + nl : tk.start;
            const int node = side ? rnode : lnode;
            const float* mn = side ? c.rmn : c.lmn;
            const float* mx = side ? c.rmx : c.lmx;
            if (cnt == 1) {
                sah_write(nodes, total, node, mn, mx, -1, perm[start]);
                atomicMax(max_level, tk.level + 1);
            } else if (cnt <= 4) {
                small[atomicAdd(n_small, 1)] = SahSmall{start, cnt, node, tk.level + 1};
            } else {
                SahTask nt;
                nt.start = start;
                nt.count = cnt;
                nt.node = node;
                nt.level = tk.level + 1;
                for (int a = 0; a < 3; ++a) { nt.mn[a] = mn[a]; nt.mx[a] = mx[a]; }
                next[atomicAdd(n_next, 1)] = nt;
            }
        }
    }
}

// One thread per small task: build_range for 2 to 4 primitives (box, longest
// axis, median split by centroid sum -- insertion order kept among equal
// keys -- down to the leaves).
__global__ void sah_small(const SahSmall* small, int n_small, int* perm, const DBox* boxes,
                          pgpu_bvh_node* nodes, int total, int* max_level) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n_small; k += gridDim.x * blockDim.x) {
        SahSmall stack[8];
        int sp = 0;
        stack[sp++] = small[k];
        while (sp > 0) {
            const SahSmall s = stack[--sp];
            float mn[3] = {1e30f, 1e30f, 1e30f}, mx[3] = {-1e30f, -1e30f, -1e30f};
            for (int i = 0; i < s.count; ++i) {
                const DBox& b = boxes[perm[s.start + i]];
                for (int a = 0; a < 3; ++a) {
                    mn[a] = fminf(mn[a], b.mn[a]);
                    mx[a] = fmaxf(mx[a], b.mx[a]);
                }
            }
            atomicMax(max_level, s.level);
            if (s.count == 1) {
                sah_write(nodes, total, s.node, mn, mx, -1, perm[s.start]);
                continue;
            }
            const int axis = sah_axis(mn, mx);
            for (int i = 1; i < s.count; ++i) {          // insertion sort (stable)
                const int v = perm[s.start + i];
                const float kv = sah_key2(boxes[v], axis);
                int j = i - 1;
                while (j >= 0 && sah_key2(boxes[perm[s.start + j]], axis) > kv) {
                    perm[s.start + j + 1] = perm[s.start + j];
                    --j;
                }
                perm[s.start + j + 1] = v;
            }
            const int half = s.count / 2;
            sah_write(nodes, total, s.node, mn, mx, s.node + 1, s.node + 2 * half);
            stack[sp++] = SahSmall{s.start + half, s.count - half, s.node + 2 * half, s.level + 1};
            stack[sp++] = SahSmall{s.start, half, s.node + 1, s.level + 1};
        }
    }
}

// The root: its box (a reduction over every primitive's box), its task.
__global__ void sah_root_box(const DBox* boxes, int n, int* bounds) {
    int mn[3] = {INT_MAX, INT_MAX, INT_MAX}, mx[3] = {INT_MIN, INT_MIN, INT_MIN};
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        for (int a = 0; a < 3; ++a) {
            mn[a] = min(mn[a], ord(boxes[k].mn[a]));
            mx[a] = max(mx[a], ord(boxes[k].mx[a]));
        }
    for (int a = 0; a < 3; ++a) {
        for (int off = 16; off > 0; off >>= 1) {
            mn[a] = min(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], off));
            mx[a] = max(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], off));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(bounds + a, mn[a]);
            atomicMax(bounds + 3 + a, mx[a]);
        }
    }
}
__global__ void sah_root(const int* bounds, int n, SahTask* tasks, SahSmall* small,
                         int* perm) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        perm[k] = k;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        SahTask t;
        t.start = 0;
        t.count = n;
        t.node = 0;
        t.level = 1;
        for (int a = 0; a < 3; ++a) { t.mn[a] = unord(bounds[a]); t.mx[a] = unord(bounds[3 + a]); }
        if (n > 4) tasks[0] = t;
        else small[0] = SahSmall{0, n, 0, 1};
    }
}

}  // namespace

// Builds the table on the current device; n_unified >= 2. Device memory for
// the build is allocated here and freed before returning.
cudaError_t device_lbvh(const pgpu_scene& s, int n_unified, pgpu_bvh_node* out, int& depth,
                        cudaStream_t st, cudaMemPool_t pool) {
    const int n = n_unified;
    const size_t np = (size_t)s.n_prims, nv = (size_t)s.n_mesh_vertices,
                 nt = (size_t)s.n_mesh_triangles;
    const size_t total = 2 * (size_t)n - 1;
    // one block of device memory for the inputs and every stage
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    size_t bytes = al(np * sizeof(pgpu_prim)) + al(nv * 12) + al(nt * 12) +
                   al((size_t)n * sizeof(DBox)) + al(6 * 4) + 2 * al((size_t)n * 8) +
                   3 * al(total * 4) + al(total * sizeof(DBox)) + 3 * al(total * 4) +
                   al((size_t)n * 4) + al(4) + al(total * sizeof(pgpu_bvh_node));
    size_t sort_bytes = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, sort_bytes, (unsigned long long*)nullptr,
                                   (unsigned long long*)nullptr, n, 0, 64, st);
    bytes += al(sort_bytes);
    DevBuf mem;
    cudaError_t e = mem.alloc(bytes, pool, st);
    if (e != cudaSuccess) return e;
    unsigned char* p = static_cast<unsigned char*>(mem.p);
    auto take = [&](size_t b) { unsigned char* r = p; p += al(b); return r; };
    auto* d_prims = reinterpret_cast<pgpu_prim*>(take(np * sizeof(pgpu_prim)));
    auto* d_verts = reinterpret_cast<float*>(take(nv * 12));
    auto* d_idx = reinterpret_cast<int*>(take(nt * 12));
    auto* d_boxes = reinterpret_cast<DBox*>(take((size_t)n * sizeof(DBox)));
    auto* d_bounds = reinterpret_cast<int*>(take(6 * 4));
    auto* d_keys = reinterpret_cast<unsigned long long*>(take((size_t)n * 8));
    auto* d_sorted = reinterpret_cast<unsigned long long*>(take((size_t)n * 8));
    auto* d_left = reinterpret_cast<int*>(take(total * 4));
    auto* d_right = reinterpret_cast<int*>(take(total * 4));
    auto* d_parent = reinterpret_cast<int*>(take(total * 4));
    auto* d_nbox = reinterpret_cast<DBox*>(take(total * sizeof(DBox)));
    auto* d_size = reinterpret_cast<int*>(take(total * 4));
    auto* d_pre = reinterpret_cast<int*>(take(total * 4));
    auto* d_level = reinterpret_cast<int*>(take(total * 4));
    auto* d_arrive = reinterpret_cast<int*>(take((size_t)n * 4));
    auto* d_maxlvl = reinterpret_cast<int*>(take(4));
    auto* d_out = reinterpret_cast<pgpu_bvh_node*>(take(total * sizeof(pgpu_bvh_node)));
    void* d_sort_tmp = take(sort_bytes);

    if (np) e = cudaMemcpyAsync(d_prims, s.prims, np * sizeof(pgpu_prim), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && nv)
        e = cudaMemcpyAsync(d_verts, s.mesh_vertices, nv * 12, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && nt)
        e = cudaMemcpyAsync(d_idx, s.mesh_indices, nt * 12, cudaMemcpyHostToDevice, st);
    const int init[6] = {INT_MAX, INT_MAX, INT_MAX, INT_MIN, INT_MIN, INT_MIN};
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_bounds, init, sizeof(init), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_arrive, 0, (size_t)n * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_maxlvl, 0, 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_parent, 0xff, total * 4, st);
    if (e != cudaSuccess) return e;
    const int B = 256;
    auto grid = [&](size_t work) { return (int)std::min<size_t>((work + B - 1) / B, 148 * 32); };
    lb_boxes<<<grid(n), B, 0, st>>>(d_prims, (int)np, d_verts, d_idx, (int)nt, d_boxes);
    lb_centre_bounds<<<grid(n), B, 0, st>>>(d_boxes, n, d_bounds);
    lb_keys<<<grid(n), B, 0, st>>>(d_boxes, n, d_bounds, d_keys);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    e = cub::DeviceRadixSort::SortKeys(d_sort_tmp, sort_bytes, d_keys, d_sorted, n, 0, 64, st);
    if (e != cudaSuccess) return e;
    lb_tree<<<grid(n - 1), B, 0, st>>>(d_sorted, n, d_left, d_right, d_parent);
    lb_refit<<<grid(n), B, 0, st>>>(d_boxes, d_sorted, n, d_left, d_right, d_parent, d_nbox,
                                    d_size, d_arrive);
    lb_emit<<<grid(total), B, 0, st>>>(d_sorted, n, d_left, d_right, d_parent, d_nbox, d_size,
                                       d_pre, d_level, d_maxlvl);
    lb_write<<<grid(total), B, 0, st>>>(d_sorted, n, d_left, d_right, d_nbox, d_pre, d_out);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(out, d_out, total * sizeof(pgpu_bvh_node),
                             cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return e;
    if ((e = cudaMemcpyAsync(&depth, d_maxlvl, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return e;
    return cudaStreamSynchronize(st);
}

// Pencil's binned SAH tree, built on the current device; n_unified >= 2.
// Device memory for the build is allocated here and freed before returning.
template <bool Q>
static cudaError_t device_sah_impl(const pgpu_scene& s, int n_unified, pgpu_bvh_node* out,
                                   int& depth, cudaStream_t st, cudaMemPool_t pool) {
    constexpr int NB = kBinsPerTask<Q>;
    const int n = n_unified;
    const size_t np = (size_t)s.n_prims, nv = (size_t)s.n_mesh_vertices,
                 nt = (size_t)s.n_mesh_triangles;
    const size_t total = 2 * (size_t)n - 1;
    const int t_max = n / 5 + 1;                          // tasks of > 4 primitives per level
    const int item_max = t_max + n / kSahChunk + 1;       // their chunks
    const int small_max = n / 2 + 1;                      // tasks of 2 to 4 primitives, in all
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    size_t scan_bytes = 0, seg_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (int*)nullptr, (int*)nullptr,
                                  std::max(item_max, t_max), st);
    cub::DeviceSegmentedRadixSort::SortPairs(nullptr, seg_bytes, (const float*)nullptr,
                                             (float*)nullptr, (const int*)nullptr, (int*)nullptr,
                                             n, t_max, (const int*)nullptr, (const int*)nullptr,
                                             0, 32, st);
    size_t bytes = al(np * sizeof(pgpu_prim)) + al(nv * 12) + al(nt * 12) +
                   al((size_t)n * sizeof(DBox)) + 2 * al((size_t)n * 4) + al(8 * 4) +
                   2 * al((size_t)t_max * sizeof(SahTask)) + al((size_t)small_max * sizeof(SahSmall)) +
                   al((size_t)t_max * NB * sizeof(SahBin)) + al((size_t)t_max * 6 * 4) +
                   al((size_t)t_max * sizeof(SahChoice)) + 2 * al((size_t)t_max * 4) +
                   2 * al((size_t)item_max * 4) + 3 * al((size_t)t_max * 4) +
                   2 * al((size_t)n * 4) + 2 * al((size_t)n * 4) +
                   al(total * sizeof(pgpu_bvh_node)) + al(scan_bytes) + al(seg_bytes) + al(2 * 4);
    DevBuf mem;
    cudaError_t e = mem.alloc(bytes, pool, st);
    if (e != cudaSuccess) return e;
    unsigned char* p = static_cast<unsigned char*>(mem.p);
    auto take = [&](size_t b) { unsigned char* r = p; p += al(b); return r; };
    auto* d_prims = reinterpret_cast<pgpu_prim*>(take(np * sizeof(pgpu_prim)));
    auto* d_verts = reinterpret_cast<float*>(take(nv * 12));
    auto* d_idx = reinterpret_cast<int*>(take(nt * 12));
    auto* d_boxes = reinterpret_cast<DBox*>(take((size_t)n * sizeof(DBox)));
    auto* d_perm = reinterpret_cast<int*>(take((size_t)n * 4));
    auto* d_tmp = reinterpret_cast<int*>(take((size_t)n * 4));
    auto* d_ctr = reinterpret_cast<int*>(take(8 * 4));   // bounds[6], n_next, n_fb
    SahTask* d_task[2] = {reinterpret_cast<SahTask*>(take((size_t)t_max * sizeof(SahTask))),
                          reinterpret_cast<SahTask*>(take((size_t)t_max * sizeof(SahTask)))};
    auto* d_small = reinterpret_cast<SahSmall*>(take((size_t)small_max * sizeof(SahSmall)));
    auto* d_bins = reinterpret_cast<SahBin*>(take((size_t)t_max * NB * sizeof(SahBin)));
    auto* d_cb = reinterpret_cast<int*>(take((size_t)t_max * 6 * 4));   // quality: centroid bounds
    auto* d_ch = reinterpret_cast<SahChoice*>(take((size_t)t_max * sizeof(SahChoice)));
    auto* d_nchunk = reinterpret_cast<int*>(take((size_t)t_max * 4));
    auto* d_item_off = reinterpret_cast<int*>(take((size_t)t_max * 4));
    auto* d_left_cnt = reinterpret_cast<int*>(take((size_t)item_max * 4));
    auto* d_left_off = reinterpret_cast<int*>(take((size_t)item_max * 4));
    auto* d_fb = reinterpret_cast<int*>(take((size_t)t_max * 4));
    auto* d_fb_size = reinterpret_cast<int*>(take((size_t)t_max * 4));
    auto* d_fb_off = reinterpret_cast<int*>(take((size_t)t_max * 4));
    auto* d_keys = reinterpret_cast<float*>(take((size_t)n * 4));
    auto* d_keys2 = reinterpret_cast<float*>(take((size_t)n * 4));
    auto* d_vals = reinterpret_cast<int*>(take((size_t)n * 4));
    auto* d_vals2 = reinterpret_cast<int*>(take((size_t)n * 4));
    auto* d_out = reinterpret_cast<pgpu_bvh_node*>(take(total * sizeof(pgpu_bvh_node)));
    void* d_scan_tmp = take(scan_bytes);
    void* d_seg_tmp = take(seg_bytes);
    int* d_misc = reinterpret_cast<int*>(take(2 * 4));   // small tasks, deepest level

    if (np) e = cudaMemcpyAsync(d_prims, s.prims, np * sizeof(pgpu_prim), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && nv)
        e = cudaMemcpyAsync(d_verts, s.mesh_vertices, nv * 12, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && nt)
        e = cudaMemcpyAsync(d_idx, s.mesh_indices, nt * 12, cudaMemcpyHostToDevice, st);
    const int init[8] = {INT_MAX, INT_MAX, INT_MAX, INT_MIN, INT_MIN, INT_MIN, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_ctr, init, sizeof(init), cudaMemcpyHostToDevice, st);
    const int misc_init[2] = {n > 4 ? 0 : 1, 0};   // a root of 2 to 4 primitives is small
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_misc, misc_init, sizeof(misc_init), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    const int B = kSahBlock;
    auto grid = [&](size_t work) {
        return (int)std::max<size_t>(1, std::min<size_t>((work + B - 1) / B, 148 * 32));
    };
    lb_boxes<<<grid(n), B, 0, st>>>(d_prims, (int)np, d_verts, d_idx, (int)nt, d_boxes);
    sah_root_box<<<grid(n), B, 0, st>>>(d_boxes, n, d_ctr);
    sah_root<<<grid(n), B, 0, st>>>(d_ctr, n, d_task[0], d_small, d_perm);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    int T = n > 4 ? 1 : 0;
    int cur = 0;
    int host_ctr[2];
    // every level holds at least one node more than the previous: at most n levels
    for (int lvl = 0; T > 0 && lvl < n; ++lvl) {
        SahTask* tasks = d_task[cur];
        sah_chunks<<<grid(T), B, 0, st>>>(tasks, T, d_nchunk);
        if ((e = cub::DeviceScan::ExclusiveSum(d_scan_tmp, scan_bytes, d_nchunk, d_item_off, T,
                                               st)) != cudaSuccess)
            return e;
        const int grid_items = std::min(item_max, T + n / kSahChunk + 1);
        if constexpr (Q) {
            sah_cb_init<<<grid(T * 6), B, 0, st>>>(d_cb, T * 6);
            sah_cbounds<<<grid_items, B, 0, st>>>(tasks, T, d_item_off, d_nchunk, d_perm,
                                                  d_boxes, d_cb);
        }
        sah_bins_init<<<grid(T * NB), B, 0, st>>>(d_bins, T * NB);
        sah_bin<Q><<<grid_items, B, 0, st>>>(tasks, T, d_item_off, d_nchunk, d_perm, d_boxes,
                                             d_cb, d_bins);
        if ((e = cudaMemsetAsync(d_ctr + 6, 0, 2 * 4, st)) != cudaSuccess) return e;
        sah_choose<Q><<<grid(T), B, 0, st>>>(tasks, T, d_bins, d_cb, d_ch, d_fb, d_ctr + 7);
        if ((e = cudaMemsetAsync(d_left_cnt, 0, (size_t)grid_items * 4, st)) != cudaSuccess)
            return e;
        sah_part_count<Q><<<grid_items, B, 0, st>>>(tasks, T, d_item_off, d_nchunk, d_ch, d_perm,
                                                    d_boxes, d_cb, d_left_cnt);
        if ((e = cub::DeviceScan::ExclusiveSum(d_scan_tmp, scan_bytes, d_left_cnt, d_left_off,
                                               grid_items, st)) != cudaSuccess)
            return e;
        sah_part_write<Q><<<grid_items, B, 0, st>>>(tasks, T, d_item_off, d_nchunk, d_ch, d_perm,
                                                    d_boxes, d_cb, d_left_off, d_tmp);
        sah_part_copy<<<grid_items, B, 0, st>>>(tasks, T, d_item_off, d_nchunk, d_ch, d_tmp,
                                                d_perm);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        // median splits of this level
        if ((e = cudaMemcpyAsync(host_ctr, d_ctr + 6, 2 * 4, cudaMemcpyDeviceToHost, st)) !=
                cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess)
            return e;
        const int n_fb = host_ctr[1];
        if (n_fb > 0) {
            sah_fb_sizes<<<grid(n_fb), B, 0, st>>>(tasks, d_fb, n_fb, d_fb_size);
            if ((e = cub::DeviceScan::ExclusiveSum(d_scan_tmp, scan_bytes, d_fb_size, d_fb_off,
                                                   n_fb, st)) != cudaSuccess)
                return e;
            sah_fb_gather<<<n_fb, B, 0, st>>>(tasks, d_ch, d_fb, d_fb_off, d_perm, d_boxes,
                                              d_keys, d_vals);
            // the segments' end offsets are the next segments' begin offsets;
            // the last one ends at the sum of the sizes
            int last_off = 0, last_size = 0;
            if ((e = cudaMemcpyAsync(&last_off, d_fb_off + n_fb - 1, 4, cudaMemcpyDeviceToHost,
                                     st)) != cudaSuccess ||
                (e = cudaMemcpyAsync(&last_size, d_fb_size + n_fb - 1, 4, cudaMemcpyDeviceToHost,
                                     st)) != cudaSuccess ||
                (e = cudaStreamSynchronize(st)) != cudaSuccess)
                return e;
            const int fb_total = last_off + last_size;
            if ((e = cudaMemcpyAsync(d_fb_off + n_fb, &fb_total, 4, cudaMemcpyHostToDevice, st)) !=
                cudaSuccess)
                return e;
            if ((e = cub::DeviceSegmentedRadixSort::SortPairs(
                     d_seg_tmp, seg_bytes, d_keys, d_keys2, d_vals, d_vals2, fb_total, n_fb,
                     d_fb_off, d_fb_off + 1, 0, 32, st)) != cudaSuccess)
                return e;
            sah_fb_scatter<<<n_fb, B, 0, st>>>(tasks, d_ch, d_fb, d_fb_off, d_vals2, d_perm,
                                               d_boxes);
        }
        sah_children<<<grid(T), B, 0, st>>>(tasks, T, d_ch, d_perm, d_task[cur ^ 1], d_ctr + 6,
                                            d_small, d_misc, d_out, (int)total, d_misc + 1);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if ((e = cudaMemcpyAsync(host_ctr, d_ctr + 6, 4, cudaMemcpyDeviceToHost, st)) !=
                cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess)
            return e;
        T = host_ctr[0];
        cur ^= 1;
    }
    if ((e = cudaMemcpyAsync(host_ctr, d_misc, 2 * 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return e;
    if (host_ctr[0] > 0)
        sah_small<<<grid(host_ctr[0]), B, 0, st>>>(d_small, host_ctr[0], d_perm, d_boxes, d_out,
                                                  (int)total, d_misc + 1);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(out, d_out, total * sizeof(pgpu_bvh_node),
                             cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return e;
    if ((e = cudaMemcpyAsync(&depth, d_misc + 1, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return e;
    return cudaStreamSynchronize(st);
}

cudaError_t device_sah(const pgpu_scene& s, int n_unified, pgpu_bvh_node* out, int& depth,
                       cudaStream_t st, cudaMemPool_t pool, bool quality) {
    return quality ? device_sah_impl<true>(s, n_unified, out, depth, st, pool)
                   : device_sah_impl<false>(s, n_unified, out, depth, st, pool);
}

}  // namespace pgpu
