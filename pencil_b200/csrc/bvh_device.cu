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

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
};

}  // namespace

// Builds the table on the current device; n_unified >= 2. Device memory for
// the build is allocated here and freed before returning.
cudaError_t device_lbvh(const pgpu_scene& s, int n_unified, std::vector<pgpu_bvh_node>& out,
                        int& depth, cudaStream_t st) {
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
    cudaError_t e = cudaMalloc(&mem.p, bytes);
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
    out.resize(total);
    if ((e = cudaMemcpyAsync(out.data(), d_out, total * sizeof(pgpu_bvh_node),
                             cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return e;
    if ((e = cudaMemcpyAsync(&depth, d_maxlvl, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return e;
    return cudaStreamSynchronize(st);
}

}  // namespace pgpu
