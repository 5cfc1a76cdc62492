// wavefront.cu - the wavefront path tracer.
//
// Paths of one or many render jobs (scenes of uneven size) form one path
// space: job after job, pixel after pixel, sample after sample. The space is
// processed in chunks of whole pixels that fit the queue capacity Q. For each
// chunk the kernels run
//
//   generate                          camera rays of every path in the chunk
//   depth x { extend, shade, shadow } closest hit / shade_vertex / any hit
//   accumulate                        per-pixel sums in the megakernel's order
//
// extend, shade and shadow are persistent: a grid sized to fill the GPU whose
// warps fetch 32 queue entries at a time from an atomic cursor. Path state
// lives in SoA arrays indexed by the path's slot in the chunk (float4 fields,
// so every access is one coalesced 128-bit load); queues hold slots. shade
// compacts surviving paths into the next queue with one atomic per warp
// (ballot + popc), optionally binned by the octant of the new ray direction
// (sort key 1) so that warps traverse with matching near/far child order.
// Sort key 2 instead orders each iteration's shadow work by where its first
// shadow ray starts (a counting sort over Morton cells and octants).
// Next-event shadow rays are stored per slot and resolved by shadow in the
// order shade made them, with the same NeeAccum as the megakernel, so each
// path's radiance is bit-identical to the megakernel's. The whole frame is
// one CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "host_internal.h"
#include "path.cuh"

namespace pgpu {

constexpr int kWfShared = 16;
// Threads per block of the wavefront kernels: kWfBlock unless the render
// asks for 64 or 256 (an autotuned launch shape); the kernels are compiled
// for blocks of up to kWfMaxBlock threads.
constexpr int kWfBlock = 128;
constexpr int kWfMaxBlock = 256;
constexpr int kOctants = 8;
constexpr int kDefaultRefill = 20;   // lanes still busy when a warp refetches
// Sort key 2: each iteration's shadow work ordered by the Morton code of the
// first shadow ray's origin (6 bits per axis of the scene's root box) and its
// direction octant, so that a warp's shadow rays start close together and
// traverse alike (2^21 bins; a counting sort per iteration).
constexpr int kMortonBits = 6;
constexpr int kSortBins = 1 << (3 * kMortonBits + 3);
// Sort key 3 also orders each iteration's extension rays, by the same kind of
// key at kMortonBitsE bits per axis (2^18 bins: coarser cells sort the
// extension rays as well for a cheaper histogram and scan).
constexpr int kMortonBitsE = 5;
constexpr int kSortBinsE = 1 << (3 * kMortonBitsE + 3);

// One render job of the path space.
struct WfJob {
    PathParams P;
    int view;                 // index into the SceneView table
    long long path_off;       // first path of the job in the path space
    long long pix_off;        // first pixel of the job in the pixel space
    int G;                    // accumulation lanes (as the megakernel's)
    float* out;               // device image
    float* m2;                // device second moments (or null)
};

// Device buffers of the wavefront (capacity Q slots, S shadow records each).
struct WfArgs {
    const SceneView* views;
    const WfJob* jobs;
    int n_jobs;
    int Q;
    int maxS;
    float4* ray_o;
    float4* ray_d;
    float4* T;
    float4* L;
    uint4* st;                // rng, depth, flags, job
    float4* hit;              // t, best ref, leaf slot, found
    float4* pb;               // Whitted vertex: pending base.xyz, scale s
    float4* pw;               // Whitted vertex: pending weight.xyz
    // Shadow record k of a slot: one 64-byte block, [(k * Q + slot) * 4 + f],
    //   f = 0 origin.xyz, tmin; 1 direction.xyz, tmax;
    //       2 contribution.xyz, test | group_end << 1;
    //       3 (block k = 0 only) the vertex's pending tail.xyz, kind | records << 2.
    // The shadow kernel visits slots in sorted, not slot, order: a record it
    // reads is two whole sectors, the pending word sharing the second.
    float4* rec;
    int* q[2];                // queues: kOctants bins of Q entries each
    int* counts;              // [iteration * kOctants + bin]
    unsigned int* work;       // [iteration * 3 + kernel] fetch cursors
    int* status;              // 1: shadow record overflow
    unsigned long long* counters;
    int sort_key;
    int packets;              // 1: the first bounce of a one-scene frame as warp packets
    int refill_below;         // extend/shadow: a warp refetches rays once at most
                              // this many of its lanes are still traversing
    // sort keys 2/3 (counting sort by sort_key_of of each iteration's shadow
    // work, and with key 3 of its next extension rays):
    int* key_s;               // [e] key of tmp_s[e]'s first shadow ray
    int* tmp_s;               // unsorted slots with shadow work
    int* qs;                  // the same slots sorted by key
    int* hist_s;              // kSortBins counters, then local bin offsets
    int* chunk_off;           // kSortBins / 1024 chunk totals, then chunk offsets
    int* tcnt;                // [iteration * 2 + 1] slots with shadow work
    int* key_e;               // [e] key of the next queue's entry e
    int* qe;                  // the next queue sorted by key (shade keeps the
                              // unsorted one: it reads path state by slot)
    int* hist_e;
    int* chunk_off_e;
    // A one-scene frame's scene and job, read from the kernel parameters
    // (constant bank) by the ONE instantiations: a lane then finds its node
    // and geometry pointers without a dependent global load per step.
    SceneView view0;
    WfJob job0;
};

// The scene / job of job index `jb`: the parameter copies in a one-scene
// frame, the device tables otherwise.
template <bool ONE>
__device__ __forceinline__ const SceneView& view_of(const WfArgs& A, int jb) {
    if constexpr (ONE) return A.view0;
    else return A.views[A.jobs[jb].view];
}
template <bool ONE>
__device__ __forceinline__ const WfJob& job_of(const WfArgs& A, int jb) {
    if constexpr (ONE) return A.job0;
    else return A.jobs[jb];
}

// Sort key of a ray: Morton code of its origin in the scene's root box
// (kMortonBits per axis), then the octant of its direction.
__device__ __forceinline__ uint32_t spread_bits3(uint32_t x) {
    x &= 0x3ffu;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}
template <int BITS = kMortonBits>
__device__ __forceinline__ int sort_key_of(const SceneView& S, V3 o, V3 d) {
    const float cells = (float)(1 << BITS);
    uint32_t c[3];
    const float oo[3] = {o.x, o.y, o.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float ext = S.root_max[a] - S.root_min[a];
        const float f = ext > 0.0f ? (oo[a] - S.root_min[a]) * (cells / ext) : 0.0f;
        const int q = f > 0.0f ? (int)f : 0;   // NaN and below the box: cell 0
        c[a] = (uint32_t)min(q, (1 << BITS) - 1);
    }
    const uint32_t m = spread_bits3(c[0]) | (spread_bits3(c[1]) << 1) | (spread_bits3(c[2]) << 2);
    const uint32_t oct = (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
    return (int)((m << 3) | oct);
}

__device__ __forceinline__ int find_job(const WfJob* jobs, int n, long long path) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].path_off <= path) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int find_job_pix(const WfJob* jobs, int n, long long pix) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].pix_off <= pix) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Add this thread's counters to the device totals (one atomic per warp and
// counter). cls 1: traversal by extend, 2: by shadow (split node counters).
template <bool COUNT>
__device__ __forceinline__ void flush_counts(const WfArgs& A, const RayCount& rc, int cls = 0) {
    if (!COUNT) return;
    unsigned long long v[6] = {rc.ext, rc.shadow, rc.ref, rc.tc.nodes, rc.tc.leaf_bytes,
                               rc.tc.prims};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        unsigned long long x = v[k];
        for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
        if ((threadIdx.x & 31) == 0 && x) {
            atomicAdd(A.counters + k, x);
            if (cls == 1 && k == 3) atomicAdd(A.counters + CNT_NODES_EXT, x);
            if (cls == 1 && k == 4) atomicAdd(A.counters + CNT_LEAF_EXT, x);
            if (cls == 2 && k == 3) atomicAdd(A.counters + CNT_NODES_SH, x);
            if (cls == 2 && k == 4) atomicAdd(A.counters + CNT_LEAF_SH, x);
        }
    }
}

// Number of entries in iteration `it`'s queue and the queue entry -> slot map
// across octant bins. The bin counts are staged in shared memory, once per
// block, so that the persistent loops hold no registers for them.
struct QView {
    const int* q;
    const int* cnt;   // shared: kOctants bin counts
    int Q;
    int total;
    __device__ __forceinline__ int slot(int e) const {
        int b = 0;
#pragma unroll 1
        for (; b < kOctants - 1; ++b) {
            const int c = cnt[b];
            if (e < c) break;
            e -= c;
        }
        return q[(size_t)b * Q + e];
    }
};
// Every thread of the block calls this (it synchronises the block once).
__device__ __forceinline__ QView qview(const WfArgs& A, int it) {
    __shared__ int s_cnt[kOctants];
    if (threadIdx.x < kOctants) s_cnt[threadIdx.x] = A.counts[it * kOctants + threadIdx.x];
    __syncthreads();
    QView v;
    v.q = A.q[it & 1];
    v.cnt = s_cnt;
    v.Q = A.Q;
    v.total = 0;
#pragma unroll
    for (int k = 0; k < kOctants; ++k) v.total += s_cnt[k];
    return v;
}

// Warp-cooperative fetch of 32 queue entries; returns the base (>= total: done).
__device__ __forceinline__ int fetch32(unsigned int* cursor) {
    int base = 0;
    if ((threadIdx.x & 31) == 0) base = (int)atomicAdd(cursor, 32u);
    return __shfl_sync(0xffffffffu, base, 0);
}

// ---- generate -----------------------------------------------------------------
template <bool COUNT, bool ONE>
__global__ void __launch_bounds__(kWfMaxBlock)
wf_generate(WfArgs A, long long path_begin, int n_slots) {
    RayCount rc = {};
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    bool live = false;
    if (slot < n_slots) {
        long long path = path_begin + slot;
        const int jb = ONE ? 0 : find_job(A.jobs, A.n_jobs, path);
        const WfJob& J = job_of<ONE>(A, jb);
        const PathParams& P = J.P;
        const SceneView& S = view_of<ONE>(A, jb);
        long long local = path - J.path_off;
        int pix = (int)(local / P.spp);
        int s = (int)(local % P.spp);
        // pixel of the image (of the job's window when it has one)
        const int ww = P.tile_w > 0 ? P.tile_w : P.W;
        int i = pix % ww + P.tile_x, j = pix / ww + P.tile_y;
        Rng rng{path_seed(i, j, s + P.sample_offset, P.salt)};
        float u, v;
        sample_uv(i, j, s % P.n, s / P.n, P.W, P.H, P.n, rng, u, v);
        Ray r = camera_ray(S.cam, u, v);
        A.ray_o[slot] = make_float4(r.o.x, r.o.y, r.o.z, 0.0f);
        A.ray_d[slot] = make_float4(r.d.x, r.d.y, r.d.z, 0.0f);
        // a path's first shade (iteration 0) starts from T = 1, L = 0 without
        // loading them; only a path that is never shaded needs its L here
        if (P.depth <= 0) A.L[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        A.rec[(size_t)slot * 4 + 3] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(0));  // nothing pending
        uint32_t flags = P.mode == kModeWhitted ? kFlagWhitted : 0u;
        A.st[slot] = make_uint4(rng.s, (unsigned)P.depth, flags, (unsigned)jb);
        if (COUNT) rc.ref++;
        live = P.depth > 0;
    }
    if constexpr (ONE) {
        // one job: either every path of the chunk is live or none is, so the
        // first queue is the slot order itself (no append atomics)
        if (live) A.q[0][slot] = slot;
        if (slot == 0 && A.job0.P.depth > 0) A.counts[0] = n_slots;
    } else {
        unsigned m = __ballot_sync(0xffffffffu, live);
        if (m) {
            int first = 0;
            if (lane == __ffs(m) - 1) first = atomicAdd(A.counts, __popc(m));
            first = __shfl_sync(0xffffffffu, first, __ffs(m) - 1);
            if (live) A.q[0][first + __popc(m & ((1u << lane) - 1u))] = slot;
        }
    }
    flush_counts<COUNT>(A, rc);
}

// ---- extend -------------------------------------------------------------------
// Persistent closest-hit traversal. A lane keeps its ray's traversal state
// between node steps; when few lanes of the warp are still busy, the idle
// lanes take new rays from the queue (one atomic per warp), so warps keep
// traversing instead of waiting for their slowest ray.
template <bool COUNT, bool ONE>
__global__ void __launch_bounds__(kWfMaxBlock)
wf_extend(WfArgs A, int it) {
    extern __shared__ int smem[];
    TravStack<kWfShared> stk;
    stk.sref = smem + threadIdx.x;
    stk.st = reinterpret_cast<float*>(smem + kWfShared * blockDim.x) + threadIdx.x;
    stk.stride = blockDim.x;
    RayCount rc = {};
    const QView qv = qview(A, it);
    const bool sorted_e = A.sort_key == 3 && it > 0;   // shade sorted this queue too
    unsigned int* cursor = A.work + it * 3 + 0;
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    ClosestTrav4<kWfShared, COUNT> tr;
    const SceneView* S = nullptr;       // the lane's scene (unused when ONE)
    auto scene = [&]() -> const SceneView& {
        if constexpr (ONE) return A.view0;
        else return *S;
    };
    int slot = -1;
    bool active = false;
    bool exhausted = false;
    while (true) {
        unsigned act = __ballot_sync(0xffffffffu, active);
        if (!exhausted && __popc(act) <= A.refill_below) {
            const unsigned idle = ~act;
            int base = 0;
            if (lane == 0) base = (int)atomicAdd(cursor, (unsigned)__popc(idle));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base + __popc(idle) >= qv.total) exhausted = true;
            if (!active) {
                const int e = base + __popc(idle & below);
                if (e < qv.total) {
                    slot = sorted_e ? A.qe[e] : qv.slot(e);
                    if constexpr (!ONE) S = &A.views[A.jobs[A.st[slot].w].view];
                    const float4 o = A.ray_o[slot], d = A.ray_d[slot];
                    if (COUNT) rc.ext++;
                    if (tr.init(scene(), Ray{v3(o.x, o.y, o.z), v3(d.x, d.y, d.z)}, 1e-4f, 1e9f,
                                &rc.tc))
                        A.hit[slot] = make_float4(tr.t_best, __int_as_float(tr.best_ref),
                                                  __int_as_float(tr.best), 0.0f);
                    else
                        active = true;
                }
            }
            act = __ballot_sync(0xffffffffu, active);
        }
        if (act == 0) {
            if (exhausted) break;
            continue;
        }
        if (active && tr.step(scene(), stk, &rc.tc)) {
            A.hit[slot] = make_float4(tr.t_best, __int_as_float(tr.best_ref),
                                      __int_as_float(tr.best), 0.0f);
            active = false;
        }
    }
    flush_counts<COUNT>(A, rc, 1);
}

// Warp-aggregated append of `slot` where `take`: one atomic per warp; with
// `keys`, `key` is stored at the same position.
__device__ __forceinline__ void warp_append(bool take, int slot, int* counter, int* list,
                                            int lane, int* keys = nullptr, int key = 0) {
    const unsigned m = __ballot_sync(0xffffffffu, take);
    if (!m) return;
    int first = 0;
    if (lane == __ffs(m) - 1) first = atomicAdd(counter, __popc(m));
    first = __shfl_sync(0xffffffffu, first, __ffs(m) - 1);
    if (take) {
        const int pos = first + __popc(m & ((1u << lane) - 1u));
        list[pos] = slot;
        if (keys) keys[pos] = key;
    }
}

// ---- extend, camera rays: warp packets --------------------------------------------
// The first bounce's queue holds the camera rays in slot order, so a warp's
// 32 rays are the samples of neighbouring pixels of one scene: nearly the same
// ray (a batch's first queue is appended a generate warp at a time, so its
// warps are mostly such groups too; a warp whose rays belong to different
// scenes traces them one by one).
// The warp traverses the wide tree once for all of them: every lane tests
// every node the packet enters against its own ray and its own t_best, the
// packet enters a child that any lane still reaches (nearest first by the
// lanes' smallest entry distance), and one shared stack serves the warp.
// Node loads are broadcasts and all lanes stay busy. A lane still tests a
// leaf only when its own slab test reaches it, so its result is the closest
// hit among the same leaves as its own traversal would test.
template <bool COUNT, bool ONE>
__global__ void __launch_bounds__(kWfMaxBlock) wf_extend_packet(WfArgs A) {
    __shared__ int s_ref[kWfMaxBlock / 32][kMaxStack];
    __shared__ float s_key[kWfMaxBlock / 32][kMaxStack];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int* sref = s_ref[warp];
    float* skey = s_key[warp];
    RayCount rc = {};
    const QView qv = qview(A, 0);
    unsigned int* cursor = A.work + 0;
    while (true) {
        const int base = fetch32(cursor);
        if (base >= qv.total) break;
        const int e = base + lane;
        const bool valid = e < qv.total;
        const int slot = valid ? qv.slot(e) : -1;
        int view = 0;
        if constexpr (!ONE) {
            view = valid ? A.jobs[A.st[slot].w].view : -1;
            const int view0 = __shfl_sync(0xffffffffu, view, 0);   // lane 0 has a ray
            if (!__all_sync(0xffffffffu, !valid || view == view0)) {
                if (valid) {
                    const SceneView& Sv = A.views[view];
                    const float4 o = A.ray_o[slot], d = A.ray_d[slot];
                    if (COUNT) rc.ext++;
                    ClosestTrav4<0, COUNT> t1;
                    TravStack<0> st1;
                    if (!t1.init(Sv, Ray{v3(o.x, o.y, o.z), v3(d.x, d.y, d.z)}, 1e-4f, 1e9f,
                                 &rc.tc))
                        while (!t1.step(Sv, st1, &rc.tc)) {
                        }
                    A.hit[slot] = make_float4(t1.t_best, __int_as_float(t1.best_ref),
                                              __int_as_float(t1.best), 0.0f);
                }
                continue;
            }
            view = view0;
        }
        const SceneView& S = ONE ? A.view0 : A.views[view];
        ClosestTrav4<kWfShared, COUNT> tr;
        bool active = false;
        if (valid) {
            const float4 o = A.ray_o[slot], d = A.ray_d[slot];
            if (COUNT) rc.ext++;
            active = !tr.init(S, Ray{v3(o.x, o.y, o.z), v3(d.x, d.y, d.z)}, 1e-4f, 1e9f, &rc.tc);
        }
        // lanes without a ray still load each node the packet enters: give
        // them the lo-first plane order
        if (!active) tr.rp.ox = tr.rp.oy = tr.rp.oz = 0;
        if (__any_sync(0xffffffffu, active)) {
            int node = 0, sp = 0;
            while (true) {
                const WideNode w = load_wide(S.wide, node, tr.rp);
                if (COUNT && active) rc.tc.nodes++;
                float ee[kWideWidth];
                unsigned m = active ? slab_wide(w, tr.rp, tr.tmin, tr.t_best, ee) : 0u;
                const unsigned lm = m & leaf_bits(w);
                m &= ~lm;
                unsigned ulm = __reduce_or_sync(0xffffffffu, lm);
                while (ulm) {
                    const int k = __ffs(ulm) - 1;
                    ulm &= ulm - 1;
                    if (((lm >> k) & 1u) && pick_e(ee, k) <= tr.t_best)
                        tr.test_leaf(S, pick_ref(w, k), &rc.tc);
                }
                // per child, the smallest entry distance of a lane that still
                // reaches it (entries are positive: their bits order as ints)
                float key[kWideWidth];
                int ref[kWideWidth];
                if constexpr (kWideWidth == 4) {
                    ref[0] = w.ref[0].x;
                    ref[1] = w.ref[0].y;
                    ref[2] = w.ref[0].z;
                    ref[3] = w.ref[0].w;
                } else {
#pragma unroll
                    for (int k = 0; k < kWideWidth; ++k) ref[k] = i4c(w.ref[k >> 2], k & 3);
                }
#pragma unroll
                for (int k = 0; k < kWideWidth; ++k) {
                    const bool reach = ((m >> k) & 1u) && ee[k] <= tr.t_best;
                    key[k] = __uint_as_float(__reduce_min_sync(
                        0xffffffffu, reach ? __float_as_uint(ee[k]) : 0x7f800000u));
                }
                // the nearest child next; the others stacked in child order
                // (a full sort of four keys cost more than it saved)
                int best = 0;
                float kb = key[0];
#pragma unroll
                for (int k = 1; k < kWideWidth; ++k)
                    if (key[k] < kb) { kb = key[k]; best = k; }
                if (kb != INFINITY) {
                    __syncwarp();
#pragma unroll
                    for (int k = kWideWidth - 1; k >= 0; --k)
                        if (k != best && key[k] != INFINITY) {
                            if (lane == 0) { sref[sp] = ref[k]; skey[sp] = key[k]; }
                            ++sp;
                        }
                    __syncwarp();
                    if constexpr (kWideWidth == 4) {
                        node = best == 0 ? ref[0] : best == 1 ? ref[1] : best == 2 ? ref[2] : ref[3];
                    } else {
                        node = ref[0];
#pragma unroll
                        for (int k = 1; k < kWideWidth; ++k) node = best == k ? ref[k] : node;
                    }
                    continue;
                }
                // pop the nearest entry some lane may still reach
                const float reach = __uint_as_float(__reduce_max_sync(
                    0xffffffffu, active ? __float_as_uint(tr.t_best) : 0u));
                bool found = false;
                while (sp > 0) {
                    --sp;
                    if (skey[sp] <= reach) { node = sref[sp]; found = true; break; }
                }
                if (!found) break;
            }
        }
        if (valid)
            A.hit[slot] = make_float4(tr.t_best, __int_as_float(tr.best_ref),
                                      __int_as_float(tr.best), 0.0f);
    }
    flush_counts<COUNT>(A, rc, 1);
}

// ---- shade --------------------------------------------------------------------
// Emitter that stores a vertex's shadow records and pending terms per slot.
struct StoreNee {
    const WfArgs& A;
    int slot;
    int n;
    int kind;
    V3 base, tail, w;
    float s;
    V3 o0, d0;                // first shadow ray (the sort key of the slot's shadow work)
    __device__ StoreNee(const WfArgs& a, int sl)
        : A(a), slot(sl), n(0), kind(0), base(v3(0, 0, 0)), tail(v3(0, 0, 0)), w(v3(0, 0, 0)),
          s(0.0f), o0(v3(0, 0, 0)), d0(v3(0, 0, 0)) {}
    __device__ __forceinline__ void begin_none() { kind = 0; }
    __device__ __forceinline__ void begin_pt() { kind = 1; }
    __device__ __forceinline__ void begin_whitted(V3 b) { kind = 2; base = b; }
    __device__ __forceinline__ void shadow(V3&, const Ray& r, float tmin, float tmax, bool test,
                                           V3 c, int group_end) {
        if (n >= A.maxS) {
            atomicOr(A.status, 1);
            return;
        }
        float4* b = A.rec + ((size_t)n * A.Q + slot) * 4;
        if (n == 0) { o0 = r.o; d0 = r.d; }
        b[0] = make_float4(r.o.x, r.o.y, r.o.z, tmin);
        b[1] = make_float4(r.d.x, r.d.y, r.d.z, tmax);
        b[2] = make_float4(c.x, c.y, c.z, __int_as_float((test ? 1 : 0) | (group_end << 1)));
        ++n;
    }
    __device__ __forceinline__ void pending(V3 tl, V3 ww, float ss) { tail = tl; w = ww; s = ss; }
    __device__ __forceinline__ void store() {
        // pt: tail and kind | records << 2; a Whitted vertex also needs its
        // base and scale (pb) and weight (pw)
        A.rec[(size_t)slot * 4 + 3] =
            make_float4(tail.x, tail.y, tail.z, __int_as_float(kind | (n << 2)));
        if (kind == 2) {
            A.pb[slot] = make_float4(base.x, base.y, base.z, s);
            A.pw[slot] = make_float4(w.x, w.y, w.z, 0.0f);
        }
    }
};

// At most 72 registers (28 warps per SM): the shading state machine is
// latency-bound, and the extra resident warps pay for a few spilled words.
template <bool COUNT, bool ONE>
__global__ void __maxnreg__(72)
wf_shade(WfArgs A, int it) {
    RayCount rc = {};
    QView qv = qview(A, it);
    unsigned int* cursor = A.work + it * 3 + 1;
    int* qout = A.q[(it + 1) & 1];
    int* cout = A.counts + (it + 1) * kOctants;
    const int lane = threadIdx.x & 31;
    while (true) {
        int base = fetch32(cursor);
        if (base >= qv.total) break;
        int e = base + lane;
        bool alive = false;
        bool shadow_work = false;
        int slot = -1;
        int bin = 0;
        int key = -1;
        int key_next = -1;
        if (e < qv.total) {
            slot = qv.slot(e);
            uint4 stv = A.st[slot];
            const WfJob& J = job_of<ONE>(A, stv.w);
            const SceneView& S = view_of<ONE>(A, stv.w);
            const float4 o = A.ray_o[slot], d = A.ray_d[slot];
            const float4 T = it == 0 ? make_float4(1.0f, 1.0f, 1.0f, 0.0f) : A.T[slot];
            const float4 L = it == 0 ? make_float4(0.0f, 0.0f, 0.0f, 0.0f) : A.L[slot];
            float4 hv = A.hit[slot];
            PathState ps;
            ps.ray = Ray{v3(o.x, o.y, o.z), v3(d.x, d.y, d.z)};
            ps.T = v3(T.x, T.y, T.z);
            ps.L = v3(L.x, L.y, L.z);
            ps.rng.s = stv.x;
            ps.depth = (int)stv.y;
            ps.flags = stv.z;
            int leaf = __float_as_int(hv.z);
            Hit h;
            bool found = leaf >= 0;
            if (found) make_hit(S, __float_as_int(hv.y), leaf, ps.ray, 1e-4f, hv.x, h);
            StoreNee E(A, slot);
            alive = shade_vertex(S, J.P, ps, found, h, E);
            E.store();
            shadow_work = E.kind != 0;
            if (A.sort_key >= 2 && shadow_work) key = sort_key_of(S, E.o0, E.d0);
            if (COUNT && alive && (ps.flags & kFlagWhitted)) rc.ref++;
            A.L[slot] = make_float4(ps.L.x, ps.L.y, ps.L.z, 0.0f);
            if (alive) {
                A.ray_o[slot] = make_float4(ps.ray.o.x, ps.ray.o.y, ps.ray.o.z, 0.0f);
                A.ray_d[slot] = make_float4(ps.ray.d.x, ps.ray.d.y, ps.ray.d.z, 0.0f);
                A.T[slot] = make_float4(ps.T.x, ps.T.y, ps.T.z, 0.0f);
                A.st[slot] = make_uint4(ps.rng.s, (unsigned)ps.depth, ps.flags, stv.w);
                if (A.sort_key == 1)
                    bin = (ps.ray.d.x < 0.0f ? 1 : 0) | (ps.ray.d.y < 0.0f ? 2 : 0) |
                          (ps.ray.d.z < 0.0f ? 4 : 0);
                if (A.sort_key == 3) key_next = sort_key_of<kMortonBitsE>(S, ps.ray.o, ps.ray.d);
            }
        }
        // sort key 2: the unsorted list of slots with shadow work and their
        // keys, ordered by wf_sort_scatter
        if (A.sort_key >= 2) {
            warp_append(shadow_work, slot, A.tcnt + 2 * it + 1, A.tmp_s, lane, A.key_s, key);
            // bin counts, one atomic per distinct key in the warp
            const unsigned same = __match_any_sync(0xffffffffu, key);
            if (shadow_work && lane == __ffs(same) - 1) atomicAdd(A.hist_s + key, __popc(same));
        }
        if (A.sort_key == 3) {
            const unsigned same = __match_any_sync(0xffffffffu, key_next);
            if (alive && lane == __ffs(same) - 1) atomicAdd(A.hist_e + key_next, __popc(same));
        }
        // warp-aggregated append, one atomic per (warp, bin)
        const int nbins = A.sort_key == 1 ? kOctants : 1;
#pragma unroll 1
        for (int b = 0; b < nbins; ++b) {
            unsigned m = __ballot_sync(0xffffffffu, alive && bin == b);
            if (!m) continue;
            int first = 0;
            if (lane == __ffs(m) - 1) first = atomicAdd(cout + b, __popc(m));
            first = __shfl_sync(0xffffffffu, first, __ffs(m) - 1);
            if (alive && bin == b) {
                const int pos = first + __popc(m & ((1u << lane) - 1u));
                qout[(size_t)b * A.Q + pos] = slot;
                if (A.sort_key == 3) A.key_e[pos] = key_next;   // one bin under key 3
            }
        }
    }
    flush_counts<COUNT>(A, rc);
}

// ---- sort key 2: counting sort of shade's shadow-work list ----------------------
// The bin counts are scanned in chunks of kSortChunk bins: wf_sort_scan turns
// each chunk into local exclusive offsets and its total into chunk_off;
// wf_sort_chunks scans the chunk totals. A slot's position is then
// chunk_off[key / kSortChunk] plus its bin's running local offset.
constexpr int kSortChunk = 1024;
constexpr int kSortChunks = kSortBins / kSortChunk;
constexpr int kSortChunksE = kSortBinsE / kSortChunk;
static_assert(kSortBins % kSortChunk == 0 && kSortBinsE % kSortChunk == 0,
              "the bin scan works on whole chunks");

// Exclusive scan of one value per thread of a 1024-thread block; returns the
// block total through *total.
__device__ __forceinline__ int block_scan_1024(int v, int* s_warp, int* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = s_warp[lane];
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, off);
            if (lane >= off) w += y;
        }
        s_warp[lane] = w;
    }
    __syncthreads();
    *total = s_warp[31];
    return x - v + (warp ? s_warp[warp - 1] : 0);
}

__global__ void __launch_bounds__(kSortChunk) wf_sort_scan(int* hist, int* chunk_off) {
    __shared__ int s_warp[32];
    int* h = hist + (size_t)blockIdx.x * kSortChunk;
    int total = 0;
    const int ex = block_scan_1024(h[threadIdx.x], s_warp, &total);
    h[threadIdx.x] = ex;
    if (threadIdx.x == 0) chunk_off[blockIdx.x] = total;
}

template <int CHUNKS>
__global__ void __launch_bounds__(kSortChunk) wf_sort_chunks(int* chunk_off) {
    __shared__ int s_warp[32];
    constexpr int per = (CHUNKS + kSortChunk - 1) / kSortChunk;
    int v[per];
    int sum = 0;
#pragma unroll
    for (int k = 0; k < per; ++k) {
        const int c = threadIdx.x * per + k;
        v[k] = c < CHUNKS ? chunk_off[c] : 0;
        sum += v[k];
    }
    int total = 0;
    int run = block_scan_1024(sum, s_warp, &total);
#pragma unroll
    for (int k = 0; k < per; ++k) {
        const int c = threadIdx.x * per + k;
        if (c < CHUNKS) chunk_off[c] = run;
        run += v[k];
    }
}

// Places every listed slot at its bin's next position (the order inside a
// bin is arbitrary; a path's result does not depend on its queue position).
// list[0, *count) -> out by keyof[e], the key stored beside list entry e.
__global__ void __launch_bounds__(kWfMaxBlock)
wf_sort_scatter(const int* list, const int* count, const int* keyof, int* hist,
                const int* chunk_off, int* out) {
    const int ns = *count;
    const int lane = threadIdx.x & 31;
    const int stride = gridDim.x * blockDim.x;
    // whole warps iterate together (the key match below needs every lane)
    for (int e0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31); e0 < ns; e0 += stride) {
        const int e = e0 + lane;
        const bool on = e < ns;
        const int slot = on ? list[e] : -1;
        const int key = on ? keyof[e] : -1;
        const unsigned same = __match_any_sync(0xffffffffu, key);
        const int leader = __ffs(same) - 1;
        int base = 0;
        if (on && lane == leader)
            base = chunk_off[key / kSortChunk] + atomicAdd(hist + key, __popc(same));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (on) out[base + __popc(same & ((1u << lane) - 1u))] = slot;
    }
}

// ---- shadow -------------------------------------------------------------------
// Persistent any-hit traversal of every slot's shadow records, with the same
// lane refill as extend. A lane owns one slot: it resolves the slot's records
// in the order shade made them, feeding each visibility into the same
// NeeAccum as the megakernel, then applies the pending terms to L.
// At most 80 registers (three blocks of 256 or six of 128 threads per SM):
// left free the kernel takes 105 (127 with 8-wide nodes), which leaves four
// blocks of 128 per SM -- too few warps to hide the latency of its loads.
constexpr int kShadowMinBlocks = 3;

template <bool COUNT, bool ONE>
__global__ void __launch_bounds__(kWfMaxBlock, kShadowMinBlocks)
wf_shadow(WfArgs A, int it) {
    extern __shared__ int smem[];
    TravStack<kWfShared> stk;
    stk.sref = smem + threadIdx.x;
    stk.st = reinterpret_cast<float*>(smem + kWfShared * blockDim.x) + threadIdx.x;
    stk.stride = blockDim.x;
    RayCount rc = {};
    const QView qv = qview(A, it);
    // sort key 2: the slots with shadow work, sorted by their first shadow ray
    const bool sorted = A.sort_key >= 2;
    const int total = sorted ? A.tcnt[2 * it + 1] : qv.total;
    unsigned int* cursor = A.work + it * 3 + 2;
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    AnyTrav4<kWfShared, COUNT> tr;
    const SceneView* S = nullptr;       // the lane's scene (unused when ONE)
    auto scene = [&]() -> const SceneView& {
        if constexpr (ONE) return A.view0;
        else return *S;
    };
    NeeAccum acc;
    V3 L = v3(0, 0, 0), c = v3(0, 0, 0);
    int slot = -1, k = 0, n = 0, group_end = 0;
    bool active = false;
    bool exhausted = false;

    // Resolve records k, k+1, ... of this lane's slot until one needs a
    // traversal (returns true) or all are done (pending terms applied).
    auto advance = [&]() -> bool {
        while (k < n) {
            const float4* b = A.rec + ((size_t)k * A.Q + slot) * 4;
            const float4 sc = b[2];
            const int bits = __float_as_int(sc.w);
            c = v3(sc.x, sc.y, sc.z);
            group_end = bits >> 1;
            if (bits & 1) {
                const float4 so = b[0], sd = b[1];
                if (COUNT) rc.shadow++;
                if (!tr.init(scene(), Ray{v3(so.x, so.y, so.z), v3(sd.x, sd.y, sd.z)}, so.w, sd.w,
                             &rc.tc))
                    return true;
                acc.add(L, c, group_end, !tr.hit);
            } else {
                acc.add(L, c, group_end, true);
            }
            ++k;
        }
        const float4 pt = A.rec[(size_t)slot * 4 + 3];
        V3 w = v3(0.0f, 0.0f, 0.0f);
        float sc = 0.0f;
        if (acc.kind == 2) {
            const float4 pw = A.pw[slot];
            w = v3(pw.x, pw.y, pw.z);
            sc = A.pb[slot].w;
        }
        acc.finish(L, v3(pt.x, pt.y, pt.z), w, sc);
        A.L[slot] = make_float4(L.x, L.y, L.z, 0.0f);
        return false;
    };

    while (true) {
        unsigned act = __ballot_sync(0xffffffffu, active);
        if (!exhausted && __popc(act) <= A.refill_below) {
            const unsigned idle = ~act;
            int base = 0;
            if (lane == 0) base = (int)atomicAdd(cursor, (unsigned)__popc(idle));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base + __popc(idle) >= total) exhausted = true;
            if (!active) {
                const int e = base + __popc(idle & below);
                if (e < total) {
                    slot = sorted ? A.qs[e] : qv.slot(e);
                    const int info = __float_as_int(A.rec[(size_t)slot * 4 + 3].w);
                    const int kind = info & 3;
                    if (kind != 0) {
                        if constexpr (!ONE) S = &A.views[A.jobs[A.st[slot].w].view];
                        const float4 L4 = A.L[slot];
                        if (kind == 1) {
                            acc.begin_pt();
                        } else {
                            const float4 pb = A.pb[slot];
                            acc.begin_whitted(v3(pb.x, pb.y, pb.z));
                        }
                        L = v3(L4.x, L4.y, L4.z);
                        n = info >> 2;
                        k = 0;
                        active = advance();
                    }
                }
            }
            act = __ballot_sync(0xffffffffu, active);
        }
        if (act == 0) {
            if (exhausted) break;
            continue;
        }
        if (active && tr.step(scene(), stk, &rc.tc)) {
            acc.add(L, c, group_end, !tr.hit);
            ++k;
            active = advance();
        }
    }
    flush_counts<COUNT>(A, rc, 2);
}

// ---- accumulate -----------------------------------------------------------------
// The sums of one pixel by its warp: lane g < G (the job's accumulation
// lanes) sums samples g, g+G, ... in order and the lanes are combined by the
// megakernel's halving tree, so the sums round exactly as the megakernel's;
// the warp's loads of the pixel's samples are contiguous.
__device__ __forceinline__ void accumulate_pixel(const WfArgs& A, long long pix,
                                                 long long path_begin, int g) {
    const int jb = find_job_pix(A.jobs, A.n_jobs, pix);
    const WfJob& J = A.jobs[jb];
    const int spp = J.P.spp, G = J.G;
    const long long lp = pix - J.pix_off;
    const long long first = J.path_off + lp * spp - path_begin;
    V3 acc = v3(0, 0, 0), acc2 = v3(0, 0, 0);
    if (g < G) {
        for (int s = g; s < spp; s += G) {
            const float4 l = A.L[first + s];
            const V3 c = v3(l.x, l.y, l.z);
            acc = acc + c;
            acc2 = acc2 + c * c;
        }
    }
    for (int off = G >> 1; off > 0; off >>= 1) {
        const V3 o = v3(__shfl_down_sync(0xffffffffu, acc.x, off),
                        __shfl_down_sync(0xffffffffu, acc.y, off),
                        __shfl_down_sync(0xffffffffu, acc.z, off));
        const V3 o2 = v3(__shfl_down_sync(0xffffffffu, acc2.x, off),
                         __shfl_down_sync(0xffffffffu, acc2.y, off),
                         __shfl_down_sync(0xffffffffu, acc2.z, off));
        if (g < off) {
            acc = acc + o;
            acc2 = acc2 + o2;
        }
    }
    if (g != 0) return;
    const float denom = (float)spp;
    float* o = J.out + 3 * lp;
    o[0] = acc.x / denom;
    o[1] = acc.y / denom;
    o[2] = acc.z / denom;
    if (J.m2) {
        float* q = J.m2 + 3 * lp;
        q[0] = acc2.x / denom;
        q[1] = acc2.y / denom;
        q[2] = acc2.z / denom;
    }
}

// A warp per pixel of the chunk, grid-stride over the pixels.
__global__ void __launch_bounds__(kWfMaxBlock)
wf_accumulate(WfArgs A, long long pix_begin, int n_pix, long long path_begin) {
    const int g = threadIdx.x & 31;
    const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long k = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; k < n_pix;
         k += warps)
        accumulate_pixel(A, pix_begin + k, path_begin, g);
}

// Blocks of wf_accumulate for `pixels` pixels: a warp each, at most `cap`.
static unsigned accumulate_blocks(long long pixels, int cap, int block = kWfBlock) {
    const long long b = (pixels * 32 + block - 1) / block;
    return (unsigned)(b < cap ? b : cap);
}

// ---- host side ------------------------------------------------------------------
struct WfPlanJob {
    const SceneView* view;
    RenderCfg cfg;
    float* out;
    float* m2;
};

static int lanes_for(int spp) {
    int lim = spp < 32 ? spp : 32, G = 1;
    while (G * 2 <= lim) G *= 2;
    return G;
}

// Scratch of the wavefront, owned by the context (grown on demand).
struct WfScratch {
    void* mem = nullptr;
    size_t bytes = 0;
    int Q = 0;
    int maxS = 0;
    int iters = 0;
    int jobs_cap = 0;
    int views_cap = 0;
    int block = kWfBlock;             // threads per block of this frame's kernels
    WfArgs args{};
    SceneView* d_views = nullptr;
    WfJob* d_jobs = nullptr;
    cudaGraphExec_t graph = nullptr;
    unsigned long long graph_key = 0;
    unsigned long long last_key = 0;  // the shape of the previous frame
    SceneView graph_view0{};          // the parameters a one-scene graph was captured with
    WfJob graph_job0{};
    // second stream of a frame: bounce k's shadow kernel runs beside bounce
    // k+1's extend kernel (created on first use, on the context's device)
    cudaStream_t side = nullptr;
    cudaEvent_t ev_shaded = nullptr;  // shade k and its sorts are done
    cudaEvent_t ev_shadow = nullptr;  // shadow k is done
};

static size_t al(size_t x) { return (x + 255) & ~size_t(255); }

static cudaError_t ensure_scratch(WfScratch& W, int Q, int maxS, int iters, int n_jobs,
                                  int n_views) {
    if (W.mem && W.Q >= Q && W.maxS >= maxS && W.iters >= iters && W.jobs_cap >= n_jobs &&
        W.views_cap >= n_views)
        return cudaSuccess;
    if (W.graph) { cudaGraphExecDestroy(W.graph); W.graph = nullptr; W.graph_key = 0; }
    if (W.mem) cudaFree(W.mem);
    W.mem = nullptr;
    Q = std::max(Q, W.Q);
    maxS = std::max(std::max(maxS, W.maxS), 1);
    iters = std::max(iters, W.iters);
    n_jobs = std::max(n_jobs, W.jobs_cap);
    n_views = std::max(n_views, W.views_cap);
    size_t per = al((size_t)Q * 16);
    size_t sz = 0;
    sz += 8 * per;                                   // ray_o ray_d T L st hit pb pw
    sz += 4 * (size_t)maxS * per;                    // shadow records (64 B each)
    sz += 2 * al((size_t)kOctants * Q * 4);          // queues
    sz += al((size_t)(iters + 2) * kOctants * 4);    // counts
    sz += al((size_t)(iters + 2) * 3 * 4);           // work cursors
    sz += al(4);                                     // status
    sz += 5 * al((size_t)Q * 4);                     // sort: keys, list, sorted queues
    sz += al((size_t)kSortBins * 4) + al((size_t)kSortBinsE * 4);        // sort: histograms
    sz += al((size_t)kSortChunks * 4) + al((size_t)kSortChunksE * 4);    // chunk offsets
    sz += al((size_t)(iters + 2) * 2 * 4);           // sort: list counts
    sz += al((size_t)n_views * sizeof(SceneView));
    sz += al((size_t)n_jobs * sizeof(WfJob));
    cudaError_t e = cudaMalloc(&W.mem, sz);
    if (e != cudaSuccess) { W.mem = nullptr; W.bytes = 0; W.Q = 0; return e; }
    W.bytes = sz;
    W.Q = Q;
    W.maxS = maxS;
    W.iters = iters;
    W.jobs_cap = n_jobs;
    W.views_cap = n_views;
    unsigned char* p = static_cast<unsigned char*>(W.mem);
    auto take = [&](size_t b) { unsigned char* r = p; p += al(b); return r; };
    WfArgs& A = W.args;
    A.Q = Q;
    A.maxS = maxS;
    A.ray_o = reinterpret_cast<float4*>(take((size_t)Q * 16));
    A.ray_d = reinterpret_cast<float4*>(take((size_t)Q * 16));
    A.T = reinterpret_cast<float4*>(take((size_t)Q * 16));
    A.L = reinterpret_cast<float4*>(take((size_t)Q * 16));
    A.st = reinterpret_cast<uint4*>(take((size_t)Q * 16));
    A.hit = reinterpret_cast<float4*>(take((size_t)Q * 16));
    A.pb = reinterpret_cast<float4*>(take((size_t)Q * 16));
    A.pw = reinterpret_cast<float4*>(take((size_t)Q * 16));
    A.rec = reinterpret_cast<float4*>(take((size_t)maxS * Q * 64));
    A.q[0] = reinterpret_cast<int*>(take((size_t)kOctants * Q * 4));
    A.q[1] = reinterpret_cast<int*>(take((size_t)kOctants * Q * 4));
    A.counts = reinterpret_cast<int*>(take((size_t)(iters + 2) * kOctants * 4));
    A.work = reinterpret_cast<unsigned int*>(take((size_t)(iters + 2) * 3 * 4));
    A.status = reinterpret_cast<int*>(take(4));
    A.key_s = reinterpret_cast<int*>(take((size_t)Q * 4));
    A.tmp_s = reinterpret_cast<int*>(take((size_t)Q * 4));
    A.qs = reinterpret_cast<int*>(take((size_t)Q * 4));
    A.hist_s = reinterpret_cast<int*>(take((size_t)kSortBins * 4));
    A.chunk_off = reinterpret_cast<int*>(take((size_t)kSortChunks * 4));
    A.key_e = reinterpret_cast<int*>(take((size_t)Q * 4));
    A.qe = reinterpret_cast<int*>(take((size_t)Q * 4));
    A.hist_e = reinterpret_cast<int*>(take((size_t)kSortBinsE * 4));
    A.chunk_off_e = reinterpret_cast<int*>(take((size_t)kSortChunksE * 4));
    A.tcnt = reinterpret_cast<int*>(take((size_t)(iters + 2) * 2 * 4));
    W.d_views = reinterpret_cast<SceneView*>(take((size_t)n_views * sizeof(SceneView)));
    W.d_jobs = reinterpret_cast<WfJob*>(take((size_t)n_jobs * sizeof(WfJob)));
    A.views = W.d_views;
    A.jobs = W.d_jobs;
    return cudaSuccess;
}

// Shadow records a vertex can make: path-trace (point/directional lights +
// quad lights) or Whitted (soft samples of every point/directional light).
static int max_shadow_records(const SceneView& v, const std::vector<DevLight>& lights, int soft) {
    int pt = 0, wh = 0;
    for (const auto& l : lights) {
        pt += 1;
        if (l.kind != 2) wh += l.radius > 0.0f ? soft : 1;
    }
    (void)v;
    return std::max(1, std::max(pt, wh));
}

struct WfOccupancy {
    int grid_extend = 0, grid_shade = 0, grid_shadow = 0, grid_scatter = 0, grid_packet = 0;
    int grid_accumulate = 0;
};

template <bool COUNT, bool ONE>
static cudaError_t occupancy(WfOccupancy& o, int blk = kWfBlock) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    size_t smem = (size_t)kWfShared * blk * 8;
    int b1 = 0, b2 = 0, b3 = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, wf_extend<COUNT, ONE>, blk, smem);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b2, wf_shade<COUNT, ONE>, blk, 0);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b3, wf_shadow<COUNT, ONE>, blk, smem);
    o.grid_extend = sms * std::max(b1, 1);
    o.grid_shade = sms * std::max(b2, 1);
    o.grid_shadow = sms * std::max(b3, 1);
    o.grid_scatter = sms * 8;
    o.grid_accumulate = sms * 16 * kWfBlock / blk;
    int b4 = 0;
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b4, wf_extend_packet<COUNT, ONE>, blk, 0);
    o.grid_packet = sms * std::max(b4, 1);
    return e;
}

// Enqueue the kernels of the whole path space on `st` (captured into a graph
// by the caller).
// Events around launches when a render is profiled (kernel class, start, end).
struct LaunchTimer {
    bool on = false;
    std::vector<int> cls;
    std::vector<cudaEvent_t> ev;
    void mark(int c, cudaStream_t st, bool start) {
        if (!on) return;
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, st);
        ev.push_back(e);
        if (start) cls.push_back(c);
    }
    // sum per class after the stream has finished; releases the events
    void collect(double* ms) {
        for (size_t k = 0; k < cls.size(); ++k) {
            float t = 0.0f;
            cudaEventElapsedTime(&t, ev[2 * k], ev[2 * k + 1]);
            ms[cls[k]] += t;
        }
        for (auto e : ev) cudaEventDestroy(e);
        ev.clear();
        cls.clear();
    }
};

// ONE: a one-scene frame (W.args.view0 / job0 hold its scene and job).
template <bool COUNT, bool ONE>
static cudaError_t enqueue_frame(const WfScratch& W, const std::vector<WfJob>& jobs, int iters,
                                 int Qeff, cudaStream_t st, int* launches, LaunchTimer& lt) {
    const int blk = W.block;
    WfOccupancy occ;
    cudaError_t e = occupancy<COUNT, ONE>(occ, blk);
    if (e != cudaSuccess) return e;
    const bool packet_first = W.args.packets != 0;
    // timed (profiled) frames stay on one stream so that kernel classes add
    // up; chunks of under 2^20 paths too, whose kernels are shorter than the
    // cross-stream waits would cost
    const bool overlap = W.side != nullptr && !lt.on && Qeff >= (1 << 20);
    const WfArgs& A = W.args;
    const size_t smem = (size_t)kWfShared * blk * 8;
    // walk the path space in chunks of whole pixels
    int ji = 0;
    long long pix_in_job = 0;
    const int n_jobs = (int)jobs.size();
    int n_launch = 0;
    while (ji < n_jobs) {
        long long path_begin = jobs[ji].path_off + pix_in_job * jobs[ji].P.spp;
        long long pix_begin = jobs[ji].pix_off + pix_in_job;
        long long slots = 0, pixels = 0;
        while (ji < n_jobs) {
            const WfJob& J = jobs[ji];
            long long npix = J.P.tile_w > 0 ? (long long)J.P.tile_w * J.P.tile_h
                                            : (long long)J.P.W * J.P.H;
            long long room = (Qeff - slots) / J.P.spp;
            long long take = std::min(room, npix - pix_in_job);
            if (take <= 0) break;
            slots += take * J.P.spp;
            pixels += take;
            pix_in_job += take;
            if (pix_in_job == npix) { ++ji; pix_in_job = 0; }
        }
        if (slots == 0) return cudaErrorInvalidValue;   // a pixel larger than Q
        size_t cnt_bytes = (size_t)(iters + 2) * kOctants * 4;
        if ((e = cudaMemsetAsync(A.counts, 0, cnt_bytes, st)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(A.work, 0, (size_t)(iters + 2) * 3 * 4, st)) != cudaSuccess) return e;
        if (A.sort_key >= 2 &&
            (e = cudaMemsetAsync(A.tcnt, 0, (size_t)(iters + 2) * 2 * 4, st)) != cudaSuccess)
            return e;
        int gblocks = (int)((slots + blk - 1) / blk);
        lt.mark(KC_GENERATE, st, true);
        wf_generate<COUNT, ONE><<<gblocks, blk, 0, st>>>(A, path_begin, (int)slots);
        lt.mark(KC_GENERATE, st, false);
        n_launch += 1;
        // With a side stream, shadow k runs on it beside extend k+1 (they
        // touch disjoint state: shadow k reads the shadow records and pending
        // terms and adds to L, extend k+1 reads rays and writes hits); shade
        // k+1 waits for both. Each kernel's tail then overlaps the other's.
        auto launch_extend = [&](int it) {
            lt.mark(KC_EXTEND, st, true);
            if (it == 0 && packet_first)
                wf_extend_packet<COUNT, ONE><<<occ.grid_packet, blk, 0, st>>>(A);
            else
                wf_extend<COUNT, ONE><<<occ.grid_extend, blk, smem, st>>>(A, it);
            lt.mark(KC_EXTEND, st, false);
        };
        if (iters > 0) launch_extend(0);
        for (int it = 0; it < iters; ++it) {
            if (overlap && it > 0 && (e = cudaStreamWaitEvent(st, W.ev_shadow, 0)) != cudaSuccess)
                return e;
            lt.mark(KC_SHADE, st, true);
            if (A.sort_key >= 2) {
                if ((e = cudaMemsetAsync(A.hist_s, 0, (size_t)kSortBins * 4, st)) != cudaSuccess)
                    return e;
            }
            const bool sort_next = A.sort_key == 3 && it + 1 < iters;
            if (sort_next &&
                (e = cudaMemsetAsync(A.hist_e, 0, (size_t)kSortBinsE * 4, st)) != cudaSuccess)
                return e;
            wf_shade<COUNT, ONE><<<occ.grid_shade, blk, 0, st>>>(A, it);
            if (A.sort_key >= 2) {
                wf_sort_scan<<<kSortChunks, kSortChunk, 0, st>>>(A.hist_s, A.chunk_off);
                wf_sort_chunks<kSortChunks><<<1, kSortChunk, 0, st>>>(A.chunk_off);
                wf_sort_scatter<<<occ.grid_scatter, kWfBlock, 0, st>>>(
                    A.tmp_s, A.tcnt + 2 * it + 1, A.key_s, A.hist_s, A.chunk_off, A.qs);
                n_launch += 3;
            }
            if (sort_next) {
                // the survivors shade just queued (unsorted) -> qe in key order
                wf_sort_scan<<<kSortChunksE, kSortChunk, 0, st>>>(A.hist_e, A.chunk_off_e);
                wf_sort_chunks<kSortChunksE><<<1, kSortChunk, 0, st>>>(A.chunk_off_e);
                wf_sort_scatter<<<occ.grid_scatter, kWfBlock, 0, st>>>(
                    A.q[(it + 1) & 1], A.counts + (it + 1) * kOctants, A.key_e, A.hist_e,
                    A.chunk_off_e, A.qe);
                n_launch += 3;
            }
            lt.mark(KC_SHADE, st, false);
            if (overlap) {
                if ((e = cudaEventRecord(W.ev_shaded, st)) != cudaSuccess) return e;
                if ((e = cudaStreamWaitEvent(W.side, W.ev_shaded, 0)) != cudaSuccess) return e;
                wf_shadow<COUNT, ONE><<<occ.grid_shadow, blk, smem, W.side>>>(A, it);
                if ((e = cudaEventRecord(W.ev_shadow, W.side)) != cudaSuccess) return e;
                if (it + 1 < iters) launch_extend(it + 1);
            } else {
                lt.mark(KC_SHADOW, st, true);
                wf_shadow<COUNT, ONE><<<occ.grid_shadow, blk, smem, st>>>(A, it);
                lt.mark(KC_SHADOW, st, false);
                if (it + 1 < iters) launch_extend(it + 1);
            }
            n_launch += 3;
        }
        if (overlap && iters > 0 && (e = cudaStreamWaitEvent(st, W.ev_shadow, 0)) != cudaSuccess)
            return e;
        const unsigned ablocks = accumulate_blocks(pixels, occ.grid_accumulate, blk);
        lt.mark(KC_ACCUMULATE, st, true);
        wf_accumulate<<<ablocks, blk, 0, st>>>(A, pix_begin, (int)pixels, path_begin);
        lt.mark(KC_ACCUMULATE, st, false);
        n_launch += 1;
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (launches) *launches = n_launch;
    return cudaSuccess;
}

// Render jobs through the wavefront. Views/lights are host copies used to
// size the scratch; `views_dev_src` are the SceneViews to upload.
cudaError_t wavefront_render(WfScratch& W, const std::vector<SceneView>& views,
                             const std::vector<std::vector<DevLight>>& lights,
                             const std::vector<int>& job_view, const std::vector<RenderCfg>& cfgs,
                             const std::vector<float*>& outs, const std::vector<float*>& m2s,
                             unsigned long long* counters, cudaStream_t st, bool use_graph,
                             int* launches, int* status_out, double* kernel_ms) {
    const int n = (int)cfgs.size();
    std::vector<WfJob> jobs(n);
    long long path_off = 0, pix_off = 0;
    int iters = 0, maxS = 1, max_spp = 1;
    long long total_paths = 0;
    bool count = false;
    int qcap = 0, sort_key = 0, refill = 0, block = 0;
    bool packets = true;
    for (int k = 0; k < n; ++k) {
        const RenderCfg& c = cfgs[k];
        WfJob& J = jobs[k];
        J.P = PathParams{c.W, c.H, c.n, c.spp, c.depth, c.mode, c.rng, c.glass, c.soft, c.bias,
                         c.salt, c.sample_offset, c.mis ? 1 : 0, c.win[0], c.win[1], c.win[2],
                         c.win[3], 0};
        J.view = job_view[k];
        J.path_off = path_off;
        J.pix_off = pix_off;
        J.G = lanes_for(c.spp);
        J.out = outs[k];
        J.m2 = m2s[k];
        path_off += c.pixels() * c.spp;
        pix_off += c.pixels();
        iters = std::max(iters, c.depth);
        max_spp = std::max(max_spp, c.spp);
        maxS = std::max(maxS, max_shadow_records(views[J.view], lights[J.view], c.soft));
        count = count || c.count;
        if (c.queue_capacity > 0) qcap = c.queue_capacity;
        sort_key = c.sort_key;
        if (c.refill > 0) refill = c.refill;
        if (c.block > 0) block = c.block;
        packets = packets && c.packets;
    }
    total_paths = path_off;
    // Fault injection, host side: PGPU_INJECT_SHADOW_RECORDS=k gives every
    // path vertex room for only k shadow records, so that a scene needing
    // more makes shade report the overflow (it stores no record beyond the
    // room it has) and the call returns PGPU_ERR_QUEUE_OVERFLOW.
    if (const char* inj = std::getenv("PGPU_INJECT_SHADOW_RECORDS")) {
        const int k = std::atoi(inj);
        if (k >= 1 && k < maxS) maxS = k;
    }
    long long Q = qcap > 0 ? qcap : (1LL << 22);
    Q = std::max<long long>(Q, max_spp);
    Q = std::min<long long>(Q, total_paths);
    Q = std::max<long long>(Q, 1);
    cudaError_t e = ensure_scratch(W, (int)Q, maxS, iters, n, (int)views.size());
    if (e != cudaSuccess) return e;
    W.args.n_jobs = n;
    W.args.counters = counters;
    W.args.sort_key = sort_key;
    W.args.packets = packets ? 1 : 0;
    W.args.refill_below = refill > 0 ? refill : kDefaultRefill;
    W.args.maxS = maxS;
    W.block = block > 0 ? block : kWfBlock;
    const bool one = n == 1;
    if (one) {
        W.args.view0 = views[jobs[0].view];
        W.args.job0 = jobs[0];
    }
    if ((e = cudaMemcpyAsync(W.d_views, views.data(), views.size() * sizeof(SceneView),
                             cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return e;
    if ((e = cudaMemcpyAsync(W.d_jobs, jobs.data(), jobs.size() * sizeof(WfJob),
                             cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return e;
    if ((e = cudaMemsetAsync(W.args.status, 0, 4, st)) != cudaSuccess) return e;
    if (!W.side) {
        if ((e = cudaStreamCreateWithFlags(&W.side, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&W.ev_shaded, cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&W.ev_shadow, cudaEventDisableTiming)) != cudaSuccess)
            return e;
    }
    // A graph is reused while the frame's shape is unchanged.
    unsigned long long key = 1469598103934665603ull;
    auto mix = [&](unsigned long long v) { key = (key ^ v) * 1099511628211ull; };
    mix((unsigned long long)n);
    mix((unsigned long long)Q);
    mix((unsigned long long)maxS);
    mix((unsigned long long)sort_key);
    mix((unsigned long long)W.args.packets);
    mix((unsigned long long)W.args.refill_below);
    mix((unsigned long long)W.block);
    mix((unsigned long long)count);
    for (const auto& J : jobs) {
        mix((unsigned long long)J.P.W); mix((unsigned long long)J.P.H);
        mix((unsigned long long)J.P.spp); mix((unsigned long long)J.P.depth);
        mix((unsigned long long)J.P.tile_w); mix((unsigned long long)J.P.tile_h);
    }
    mix((unsigned long long)iters);
    mix((unsigned long long)one);
    // a one-scene graph also bakes the scene and job into its kernel
    // parameters: it is reused only while they are byte for byte the same
    const bool same_params =
        !one || (std::memcmp(&W.graph_view0, &W.args.view0, sizeof(SceneView)) == 0 &&
                 std::memcmp(&W.graph_job0, &W.args.job0, sizeof(WfJob)) == 0);
    int nl = 0;
    LaunchTimer lt;
    lt.on = kernel_ms != nullptr;
    auto enqueue = [&](int* nl_out) {
        return count ? (one ? enqueue_frame<true, true>(W, jobs, iters, (int)Q, st, nl_out, lt)
                            : enqueue_frame<true, false>(W, jobs, iters, (int)Q, st, nl_out, lt))
                     : (one ? enqueue_frame<false, true>(W, jobs, iters, (int)Q, st, nl_out, lt)
                            : enqueue_frame<false, false>(W, jobs, iters, (int)Q, st, nl_out, lt));
    };
    if (lt.on) use_graph = false;
    // a frame shape met for the first time runs as direct launches: a graph
    // pays for its capture and instantiation only when the shape repeats
    if (use_graph && !(W.graph && W.graph_key == key) && W.last_key != key) use_graph = false;
    W.last_key = key;
    if (use_graph) {
        if (!W.graph || W.graph_key != key || !same_params) {
            // same shape, another scene or job: the captured graph has the
            // executable graph's topology, whose parameters are updated in
            // place (no new instantiation)
            const bool same_shape = W.graph && W.graph_key == key;
            if (W.graph && !same_shape) { cudaGraphExecDestroy(W.graph); W.graph = nullptr; }
            cudaGraph_t g = nullptr;
            if ((e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
                return e;
            cudaError_t ee = enqueue(&nl);
            if (ee != cudaSuccess) {
                // a failed enqueue may leave the side stream forked off the
                // capture: join it so that the capture ends on both streams
                cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
                if (cudaStreamIsCapturing(W.side, &cs) == cudaSuccess &&
                    cs != cudaStreamCaptureStatusNone &&
                    cudaEventRecord(W.ev_shadow, W.side) == cudaSuccess)
                    cudaStreamWaitEvent(st, W.ev_shadow, 0);
            }
            e = cudaStreamEndCapture(st, &g);
            if (ee != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                (void)cudaGetLastError();   // the failure is reported once, here
                return ee;
            }
            if (e != cudaSuccess) return e;
            bool updated = false;
            if (same_shape) {
                cudaGraphExecUpdateResultInfo info;
                updated = cudaGraphExecUpdate(W.graph, g, &info) == cudaSuccess;
                if (!updated) {
                    (void)cudaGetLastError();
                    cudaGraphExecDestroy(W.graph);
                    W.graph = nullptr;
                }
            }
            if (!updated) {
                e = cudaGraphInstantiate(&W.graph, g, 0);
                if (e != cudaSuccess) {
                    cudaGraphDestroy(g);
                    W.graph = nullptr;
                    return e;
                }
            }
            cudaGraphDestroy(g);
            W.graph_key = key;
            W.graph_view0 = W.args.view0;
            W.graph_job0 = W.args.job0;
        }
        if ((e = cudaGraphLaunch(W.graph, st)) != cudaSuccess) return e;
        if (launches) *launches = 1;
    } else {
        e = enqueue(&nl);
        if (e != cudaSuccess) return e;
        if (launches) *launches = nl;
        if (lt.on) {
            if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
            lt.collect(kernel_ms);
        }
    }
    if (status_out) {
        if ((e = cudaMemcpyAsync(status_out, W.args.status, 4, cudaMemcpyDeviceToHost, st)) !=
            cudaSuccess)
            return e;
    }
    return cudaSuccess;
}

void wavefront_release(WfScratch& W) {
    if (W.graph) cudaGraphExecDestroy(W.graph);
    W.graph = nullptr;
    if (W.mem) cudaFree(W.mem);
    W.mem = nullptr;
    W.bytes = 0;
    W.Q = 0;
}

WfScratch* wavefront_new() { return new WfScratch(); }
void wavefront_delete(WfScratch* W) {
    if (!W) return;
    wavefront_release(*W);
    if (W->ev_shaded) cudaEventDestroy(W->ev_shaded);
    if (W->ev_shadow) cudaEventDestroy(W->ev_shadow);
    if (W->side) cudaStreamDestroy(W->side);
    delete W;
}

}  // namespace pgpu

// ---- rendering without allocating -------------------------------------------------
// pgpu_render_noalloc: the same wavefront kernels driven over one statically
// sized device array instead of context-owned scratch, for callers that may
// not allocate device memory during a render. The array belongs to this
// translation unit's module: every GPU that loads it holds it until exit.
namespace pgpu {

constexpr int kStaticSlots = 65536;       // paths in flight per chunk
constexpr int kStaticShadow = 4;          // shadow records per vertex
constexpr int kStaticMaxDepth = 64;       // bounces (iterations per chunk)
constexpr size_t static_al(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kStaticArray = static_al((size_t)kStaticSlots * 16);
constexpr size_t kStaticBytes =
    8 * kStaticArray +                                           // path state
    4 * (size_t)kStaticShadow * kStaticArray +                   // shadow records (64 B)
    2 * static_al((size_t)kStaticSlots * 4) +                    // queues (one bin each)
    static_al((size_t)(kStaticMaxDepth + 2) * kOctants * 4) +    // queue counts
    static_al((size_t)(kStaticMaxDepth + 2) * 3 * 4) +           // fetch cursors
    static_al(4) +                                               // status word
    static_al(sizeof(SceneView)) + static_al(sizeof(WfJob));

static __device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

size_t static_scratch_bytes() { return kStaticBytes; }

// Device address of g_static_scratch on the current device, looked up once
// per device (cudaGetSymbolAddress) and cached for the life of the process.
// The cache assumes the device's primary context lives as long as the
// library: after a cudaDeviceReset the cached address would be stale.
static std::mutex g_static_mu;
static void* g_static_ptr[64];

cudaError_t static_scratch_address(int device, void** out) {
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
    if (!g_static_ptr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return e;
        g_static_ptr[device] = p;
    }
    *out = g_static_ptr[device];
    return cudaSuccess;
}

// Render one job over the static scratch. Returns cudaSuccess, or sets *why
// (a constant string) and returns cudaErrorInvalidValue when the job exceeds
// the scratch's fixed capacity. No allocation on the host or the device.
cudaError_t wavefront_render_static(int device, const SceneView& view, const DevLight* lights,
                                    int n_lights, bool has_glass, const RenderCfg& c, float* out,
                                    float* m2, cudaStream_t st, int* status_host, int* launches,
                                    const char** why) {
    *why = nullptr;
    // shadow records a vertex can make: path-trace vertices one per light;
    // Whitted vertices (the Whitted mode, or after glass) the soft-shadow
    // samples of every point/directional light
    int pt = 0, wh = 0;
    for (int k = 0; k < n_lights; ++k) {
        pt += 1;
        if (lights[k].kind != 2) wh += lights[k].radius > 0.0f ? c.soft : 1;
    }
    const bool whitted_vertices = c.mode == kModeWhitted || has_glass;
    const int maxS = (whitted_vertices && wh > pt) ? wh : pt;
    if (maxS > kStaticShadow) {
        *why = "the scene needs more than 4 shadow rays per path vertex, the most the "
               "no-allocation render holds";
        return cudaErrorInvalidValue;
    }
    if (c.depth > kStaticMaxDepth) {
        *why = "depth above 64 is beyond the no-allocation render";
        return cudaErrorInvalidValue;
    }
    if (c.spp > kStaticSlots) {
        *why = "more than 65536 samples per pixel do not fit the no-allocation render's "
               "paths in flight";
        return cudaErrorInvalidValue;
    }
    if (c.sort_key != 0 || c.count || c.profile) {
        *why = "the no-allocation render takes no ray sorting, counting or profiling";
        return cudaErrorInvalidValue;
    }
    void* base = nullptr;
    cudaError_t e = static_scratch_address(device, &base);
    if (e != cudaSuccess) return e;
    const int Q = kStaticSlots;
    unsigned char* p = static_cast<unsigned char*>(base);
    auto take = [&](size_t b) { unsigned char* r = p; p += static_al(b); return r; };
    WfArgs A{};
    A.n_jobs = 1;
    A.Q = Q;
    A.maxS = kStaticShadow;
    A.ray_o = reinterpret_cast<float4*>(take((size_t)Q * 16));
    A.ray_d = reinterpret_cast<float4*>(take((size_t)Q * 16));
    A.T = reinterpret_cast<float4*>(take((size_t)Q * 16));
    A.L = reinterpret_cast<float4*>(take((size_t)Q * 16));
    A.st = reinterpret_cast<uint4*>(take((size_t)Q * 16));
    A.hit = reinterpret_cast<float4*>(take((size_t)Q * 16));
    A.pb = reinterpret_cast<float4*>(take((size_t)Q * 16));
    A.pw = reinterpret_cast<float4*>(take((size_t)Q * 16));
    A.rec = reinterpret_cast<float4*>(take((size_t)kStaticShadow * Q * 64));
    A.q[0] = reinterpret_cast<int*>(take((size_t)Q * 4));
    A.q[1] = reinterpret_cast<int*>(take((size_t)Q * 4));
    A.counts = reinterpret_cast<int*>(take((size_t)(kStaticMaxDepth + 2) * kOctants * 4));
    A.work = reinterpret_cast<unsigned int*>(take((size_t)(kStaticMaxDepth + 2) * 3 * 4));
    A.status = reinterpret_cast<int*>(take(4));
    SceneView* d_view = reinterpret_cast<SceneView*>(take(sizeof(SceneView)));
    WfJob* d_job = reinterpret_cast<WfJob*>(take(sizeof(WfJob)));
    A.views = d_view;
    A.jobs = d_job;
    A.counters = nullptr;
    A.sort_key = 0;
    A.refill_below = kDefaultRefill;
    WfJob J{};
    J.P = PathParams{c.W, c.H, c.n, c.spp, c.depth, c.mode, c.rng, c.glass, c.soft, c.bias,
                     c.salt, c.sample_offset, c.mis ? 1 : 0, 0, 0, 0, 0, 0};
    J.view = 0;
    J.path_off = 0;
    J.pix_off = 0;
    J.G = lanes_for(c.spp);
    J.out = out;
    J.m2 = m2;
    // Every call shares the array: the tables are rewritten and the status
    // word, queue counts and fetch cursors are cleared before they are read.
    if ((e = cudaMemcpyAsync(d_view, &view, sizeof(SceneView), cudaMemcpyHostToDevice, st)) !=
        cudaSuccess)
        return e;
    if ((e = cudaMemcpyAsync(d_job, &J, sizeof(WfJob), cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return e;
    if ((e = cudaMemsetAsync(A.status, 0, 4, st)) != cudaSuccess) return e;
    A.view0 = view;
    A.job0 = J;
    WfOccupancy occ;
    if ((e = occupancy<false, true>(occ)) != cudaSuccess) return e;
    const size_t smem = (size_t)kWfShared * kWfBlock * 8;
    const long long npix = (long long)c.W * c.H;
    const long long ppc = Q / c.spp;
    int n_launch = 0;
    for (long long pix0 = 0; pix0 < npix; pix0 += ppc) {
        const long long pixels = (npix - pix0) < ppc ? (npix - pix0) : ppc;
        const long long slots = pixels * c.spp;
        const long long path0 = pix0 * c.spp;
        if ((e = cudaMemsetAsync(A.counts, 0, (size_t)(c.depth + 2) * kOctants * 4, st)) !=
            cudaSuccess)
            return e;
        if ((e = cudaMemsetAsync(A.work, 0, (size_t)(c.depth + 2) * 3 * 4, st)) != cudaSuccess)
            return e;
        wf_generate<false, true><<<(unsigned)((slots + kWfBlock - 1) / kWfBlock), kWfBlock, 0, st>>>(
            A, path0, (int)slots);
        for (int it = 0; it < c.depth; ++it) {
            wf_extend<false, true><<<occ.grid_extend, kWfBlock, smem, st>>>(A, it);
            wf_shade<false, true><<<occ.grid_shade, kWfBlock, 0, st>>>(A, it);
            wf_shadow<false, true><<<occ.grid_shadow, kWfBlock, smem, st>>>(A, it);
        }
        wf_accumulate<<<accumulate_blocks(pixels, occ.grid_accumulate), kWfBlock, 0, st>>>(
            A, pix0, (int)pixels, path0);
        n_launch += 2 + 3 * c.depth;
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (launches) *launches = n_launch;
    return cudaMemcpyAsync(status_host, A.status, 4, cudaMemcpyDeviceToHost, st);
}

}  // namespace pgpu
