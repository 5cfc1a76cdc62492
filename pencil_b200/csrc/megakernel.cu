// megakernel.cu - the plain GPU path tracer: one thread per (pixel, sample
// lane), every bounce, shadow ray and the Whitted continuation in one kernel.
// It traverses the same 4-wide tree as the wavefront by default (the
// baseline the wavefront is measured against), or Pencil's binary tree with
// PGPU_FLAG_BINARY_TREE.
//
// Thread mapping. Counter RNG: G = largest power of two <= min(spp, 32)
// lanes share a pixel; lane g traces samples g, g + G, ... and the G partial
// sums are combined by a butterfly of warp shuffles, so the pixel sum is
// deterministic. Per-pixel RNG: one thread per pixel consumes Pencil's
// per-pixel xorshift32 stream over its samples in Pencil's order.
#include <cuda_runtime.h>

#include "host_internal.h"
#include "path.cuh"

namespace pgpu {

constexpr int kMkShared = 16;   // stack entries per thread kept in shared memory
// Held to 64 registers (eight blocks of 128 threads per SM): more resident
// warps hide more of the divergent paths' load latency than the spilled
// words cost. Sphere-cloud frame 85.8 ms at the compiler's choice (96-128
// registers) -> 73.4 at 72 -> 71.8 at 64; mesh frame 443.5 -> 378.0 ->
// 382.3 ms.
constexpr int kMkMinBlocks = 8;

template <bool COUNT, bool TREE, bool PIXEL_SEQ, bool WIDE>
__global__ void __launch_bounds__(128, kMkMinBlocks)
mk_render(SceneView S, PathParams P, int G, float* __restrict__ out, float* __restrict__ m2,
          unsigned long long* __restrict__ counters) {
    extern __shared__ int smem[];
    TravStack<kMkShared> stk;
    stk.sref = smem + threadIdx.x;
    stk.st = reinterpret_cast<float*>(smem + kMkShared * blockDim.x) + threadIdx.x;
    stk.stride = blockDim.x;
    RayCount rc = {};
    Tracer<kMkShared, COUNT, WIDE> tr{S, P, stk, rc};

    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool tile = P.tile_w > 0;
    const int outW = tile ? P.tile_w : P.W, outH = tile ? P.tile_h : P.H;
    const long long npix = (long long)outW * outH;
    const long long pix = gid / G;
    const int lane_g = (int)(gid % G);
    const bool active = pix < npix;
    V3 acc = v3(0, 0, 0), acc2 = v3(0, 0, 0);
    if (active) {
        // pixel of the full image
        const int i = (int)(pix % outW) + (tile ? P.tile_x : 0);
        const int j = (int)(pix / outW) + (tile ? P.tile_y : 0);
        if (PIXEL_SEQ) {
            Rng rng{pixel_seed(i, j)};
            for (int sy = 0; sy < P.n; ++sy) {
                for (int sx = 0; sx < P.n; ++sx) {
                    float u, v;
                    sample_uv(i, j, sx, sy, P.W, P.H, P.n, rng, u, v, P.worker != 0);
                    V3 c = tr.template sample<TREE>(camera_ray(S.cam, u, v), rng);
                    acc = acc + c;
                    acc2 = acc2 + c * c;
                }
            }
        } else {
            for (int s = lane_g; s < P.spp; s += G) {
                Rng rng{path_seed(i, j, s + P.sample_offset, P.salt)};
                float u, v;
                sample_uv(i, j, s % P.n, s / P.n, P.W, P.H, P.n, rng, u, v, P.worker != 0);
                V3 c = tr.template sample<TREE>(camera_ray(S.cam, u, v), rng);
                acc = acc + c;
                acc2 = acc2 + c * c;
            }
        }
    }
    for (int off = G >> 1; off > 0; off >>= 1) {
        acc.x += __shfl_xor_sync(0xffffffffu, acc.x, off);
        acc.y += __shfl_xor_sync(0xffffffffu, acc.y, off);
        acc.z += __shfl_xor_sync(0xffffffffu, acc.z, off);
        acc2.x += __shfl_xor_sync(0xffffffffu, acc2.x, off);
        acc2.y += __shfl_xor_sync(0xffffffffu, acc2.y, off);
        acc2.z += __shfl_xor_sync(0xffffffffu, acc2.z, off);
    }
    if (active && lane_g == 0) {
        const float denom = (float)P.spp;
        out[3 * pix + 0] = acc.x / denom;
        out[3 * pix + 1] = acc.y / denom;
        out[3 * pix + 2] = acc.z / denom;
        if (m2) {
            m2[3 * pix + 0] = acc2.x / denom;
            m2[3 * pix + 1] = acc2.y / denom;
            m2[3 * pix + 2] = acc2.z / denom;
        }
    }
    if (COUNT) {
        unsigned long long v[6] = {rc.ext, rc.shadow, rc.ref, rc.tc.nodes, rc.tc.leaf_bytes,
                                   rc.tc.prims};
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            unsigned long long x = v[k];
            for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
            if ((threadIdx.x & 31) == 0) atomicAdd(counters + k, x);
        }
    }
}

template <bool COUNT, bool TREE, bool PIXEL_SEQ, bool WIDE>
static cudaError_t launch_mk(const SceneView& S, const PathParams& P, int G, float* out,
                             float* m2, unsigned long long* counters, cudaStream_t st) {
    const int block = 128;
    long long threads = (P.tile_w > 0 ? (long long)P.tile_w * P.tile_h : (long long)P.W * P.H) * G;
    long long blocks = (threads + block - 1) / block;
    size_t smem = (size_t)kMkShared * block * 8;
    mk_render<COUNT, TREE, PIXEL_SEQ, WIDE><<<(unsigned)blocks, block, smem, st>>>(S, P, G, out,
                                                                                     m2, counters);
    return cudaGetLastError();
}

cudaError_t launch_megakernel(const SceneView& S, const RenderCfg& c, float* out, float* m2,
                              unsigned long long* counters, cudaStream_t st) {
    PathParams P{c.W, c.H, c.n, c.spp, c.depth, c.mode, c.rng, c.glass, c.soft, c.bias, c.salt,
                 c.sample_offset, c.mis ? 1 : 0, c.win[0], c.win[1], c.win[2], c.win[3],
                 c.worker ? 1 : 0};
    const bool seq = c.rng == PGPU_RNG_PIXEL_SEQUENTIAL;
    const bool tree = c.glass == PGPU_GLASS_BOTH_BRANCHES;
    int G = 1;
    if (!seq) {
        int lim = c.spp < 32 ? c.spp : 32;
        while (G * 2 <= lim) G *= 2;
    }
    const bool wide = !c.binary_tree;
#define PGPU_MK_CASE(CNT, TR, SQ)                                                \
    if (c.count == CNT && tree == TR && seq == SQ)                               \
        return wide ? launch_mk<CNT, TR, SQ, true>(S, P, G, out, m2, counters, st) \
                    : launch_mk<CNT, TR, SQ, false>(S, P, G, out, m2, counters, st);
    PGPU_MK_CASE(false, false, false)
    PGPU_MK_CASE(false, false, true)
    PGPU_MK_CASE(false, true, false)
    PGPU_MK_CASE(false, true, true)
    PGPU_MK_CASE(true, false, false)
    PGPU_MK_CASE(true, false, true)
    PGPU_MK_CASE(true, true, false)
    PGPU_MK_CASE(true, true, true)
#undef PGPU_MK_CASE
    return cudaErrorInvalidValue;
}

}  // namespace pgpu
