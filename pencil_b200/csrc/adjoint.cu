// adjoint.cu - gradients of an image loss with respect to per-material
// albedo and emission and per-light intensity, by path replay.
//
// Each thread replays the paths of its (pixel, sample lane) from their
// counter-RNG seeds: the same camera rays, hits, next-event samples, Russian
// roulette decisions and scatter directions as the production renderer
// (shade_vertex in path.cuh; the control flow and random-number use below
// follow it step for step), traced on the 4-wide tree the renderers walk
// (the same hits as Pencil's binary tree; at 80 registers, six blocks per
// SM, 17.5 ms per gradient there against 19.8 ms on the binary tree -- at
// 128 registers the binary tree had been the faster). No state of the
// forward render is kept: the replay records a short tape per path (at most
// kMaxTape vertices) and sweeps it backwards.
//
// Per colour channel a path's radiance is L = sum_k T_k * A_k with
// T_{k+1} = T_k * f_k. At vertex k with material m and albedo a:
//   A_k = e_k + a * B_k   (e_k: emission and Phong terms, B_k: the light and
//                          ambient terms that albedo scales)
//   f_k = a * g_k          (g_k: reflectivity, the Russian-roulette 1/p, 0 at
//                          the end of the path)
// so with R_k = A_k + f_k * R_{k+1} (the radiance leaving vertex k per unit
// throughput) the albedo's share of dL is T_k * (B_k + g_k * R_{k+1}). The
// Russian-roulette probability is treated as a constant (detached).
// dL/d(emission of m) = T_k (times the Whitted scale) where the emission is
// counted; dL/d(intensity of light l) = T_k * dA_k/dI_l.
//
// Each path's contribution is weighted by dLoss/dI of its pixel / spp.
// Material gradients are summed across a warp in FP32 (lanes with the same
// material grouped by __match_any_sync) and added in FP64 atomics; light
// gradients are summed per thread, reduced across the warp and added in FP64.
#include <cuda_runtime.h>

#include "host_internal.h"
#include "path.cuh"

namespace pgpu {

constexpr int kAdjShared = 16;
constexpr int kMaxTape = 16;        // vertices per path (depth <= 16)
constexpr int kMaxAdjLights = 8;    // lights whose gradient a thread accumulates
constexpr int kAdjBlock = 128;

struct AdjArgs {
    SceneView S;
    PathParams P;
    int G;
    const float* dl;       // dLoss/dimage, W*H*3
    double* d_albedo;      // 3 per material
    double* d_emission;    // 3 per material
    double* d_light;       // 3 per light
    float* out;            // forward image of the replayed samples (or null)
    unsigned long long* counters;
};

// One path vertex on the tape. g (reflectivity times the Russian-roulette
// 1/p, 0 at the end of the path) is the same for the three channels. E is
// the weight of the vertex's emission term, counted when `emits`.
struct TapeV {
    int mat;               // -1: background (miss)
    int emits;
    float g;
    V3 T, B, A, E;
};

// Add the contribution v of every lane that `has` one to grad[key*3 + c]:
// lanes with equal keys are summed in FP32 first (ascending lane order),
// then one FP64 atomic per key and channel. Called by the whole warp.
__device__ __forceinline__ void flush_contrib(bool has, int key, V3 v, double* grad) {
    const int lane = threadIdx.x & 31;
    const unsigned live = __ballot_sync(0xffffffffu, has);
    if (!has) return;
    const unsigned peers = __match_any_sync(live, key);
    V3 sum = v3(0, 0, 0);
    unsigned rem = peers;
    while (rem) {
        const int src = __ffs(rem) - 1;
        rem &= rem - 1;
        sum.x += __shfl_sync(peers, v.x, src);
        sum.y += __shfl_sync(peers, v.y, src);
        sum.z += __shfl_sync(peers, v.z, src);
    }
    if (lane == __ffs(peers) - 1) {
        atomicAdd(grad + 3 * (size_t)key + 0, (double)sum.x);
        atomicAdd(grad + 3 * (size_t)key + 1, (double)sum.y);
        atomicAdd(grad + 3 * (size_t)key + 2, (double)sum.z);
    }
}

template <bool COUNT>
struct Replay {
    const SceneView& S;
    const PathParams& P;
    TravStack<kAdjShared>& stk;
    RayCount& rc;

    __device__ __forceinline__ bool occluded(const Ray& r, float tmin, float tmax) {
        if (COUNT) rc.shadow++;
        return any_hit4<kAdjShared, COUNT>(S, r, tmin, tmax, stk, &rc.tc);
    }

    // Replay one path; fills the tape (returns its length; each vertex with
    // its emission weight) and the per-light gradient sums (weighted by w),
    // and returns the path radiance in L.
    __device__ int path(Ray r, Rng& rng, V3 w, TapeV* tape, V3* dlight, V3& Lout) {
        V3 T = v3(1, 1, 1), L = v3(0, 0, 0);
        int depth = P.depth;
        uint32_t flags = P.mode == kModeWhitted ? kFlagWhitted : 0u;
        int nt = 0;
        if (COUNT) rc.ref++;
        bool alive = depth > 0;
        while (alive && nt < kMaxTape) {
            TapeV& tv = tape[nt++];
            tv.T = T;
            tv.B = v3(0, 0, 0);
            tv.g = 0.0f;
            tv.emits = 0;
            if (COUNT) rc.ext++;
            float tb;
            int bref;
            int slot = closest_hit4<kAdjShared, COUNT>(S, r, 1e-4f, 1e9f, tb, bref, stk, &rc.tc);
            if (slot < 0) {
                tv.mat = -1;
                tv.A = ld3(S.bg);
                L = L + T * tv.A;
                break;
            }
            Hit h;
            make_hit(S, bref, slot, r, 1e-4f, tb, h);
            const DevMaterial& m = S.mats[h.mat];
            const V3 albedo = ld3(m.albedo);
            const bool metal = m.kind == 1 && m.reflectivity > 0.0f;
            const bool glass = m.kind == 2;
            const V3 sorg = h.p + h.n * P.bias;
            tv.mat = h.mat;
            V3 e = v3(0, 0, 0);          // albedo-free part of A
            bool dielectric = false;
            alive = false;
            if (!(flags & kFlagWhitted)) {
                const bool diffuse = !metal && !glass;
                if (!glass && !((flags & kFlagSkipArea) && m.area_emitter)) {
                    e = ld3(m.emission);
                    tv.E = w * T;
                    tv.emits = 1;
                }
                for (int li = 0; li < S.n_lights; ++li) {
                    const DevLight& l = S.lights[li];
                    if (l.kind == 2) continue;
                    V3 Ld;
                    float dist;
                    light_dir(l, h.p, rng, Ld, dist);
                    float ndotl = clampf(dot(h.n, Ld), 0.0f, 1.0f);
                    bool vis = l.is_emissive || !occluded(Ray{sorg, Ld}, P.bias, dist - P.bias);
                    if (!vis) continue;
                    tv.B = tv.B + ld3(l.intensity) * ndotl;
                    if (li < kMaxAdjLights) dlight[li] = dlight[li] + w * T * albedo * ndotl;
                }
                if (S.has_quad_lights && diffuse && depth - 1 > 0) {
                    for (int li = 0; li < S.n_lights; ++li) {
                        const DevLight& l = S.lights[li];
                        if (l.kind != 2) continue;
                        V3 Ld;
                        float tmax, wq;
                        if (!quad_sample(l, h.p, h.n, sorg, P.bias, rng, Ld, tmax, wq)) continue;
                        if (occluded(Ray{sorg, Ld}, P.bias, tmax)) continue;
                        tv.B = tv.B + ld3(l.intensity) * wq;
                        if (li < kMaxAdjLights) dlight[li] = dlight[li] + w * T * albedo * wq;
                    }
                }
                tv.B = tv.B + ld3(S.amb);
                tv.A = e + albedo * tv.B;
                L = L + T * tv.A;
                float inv_p = 1.0f;
                if (P.depth - depth > 3) {
                    float p = fmaxf(T.x, fmaxf(T.y, T.z));
                    if (rng.unit() > p) break;
                    T = T / p;
                    inv_p = 1.0f / p;
                }
                if (!glass) {
                    V3 nd;
                    if (metal) {
                        nd = metal_dir(r.d, h.n, rng);
                        T = T * albedo * m.reflectivity;
                        tv.g = inv_p * m.reflectivity;
                    } else {
                        nd = diffuse_dir(h.n, rng);
                        T = T * albedo;
                        tv.g = inv_p;
                    }
                    flags = (diffuse && S.has_quad_lights) ? kFlagSkipArea : 0u;
                    r = Ray{sorg, nd};
                    depth--;
                    alive = depth > 0;
                    if (!alive) tv.g = 0.0f;
                    continue;
                }
                tv.g = inv_p;
                dielectric = true;
            } else {
                // Whitted vertex: A = s * (emission + Phong + a * (lights + ambient))
                V3 sum_a = v3(0, 0, 0), sum_e = v3(0, 0, 0);
                float s = 1.0f;
                if (!glass) {
                    sum_e = ld3(m.emission);
                    s = metal ? 1.0f - m.reflectivity : 1.0f;
                }
                for (int li = 0; li < S.n_lights; ++li) {
                    const DevLight& l = S.lights[li];
                    if (l.kind == 2) continue;
                    int ns = (l.radius > 0.0f) ? P.soft : 1;
                    V3 ca = v3(0, 0, 0), ce = v3(0, 0, 0);
                    for (int k = 0; k < ns; ++k) {
                        V3 Ld;
                        float dist;
                        light_dir(l, h.p, rng, Ld, dist);
                        if (glass) continue;
                        float ndotl = clampf(dot(h.n, Ld), 0.0f, 1.0f);
                        V3 phong = v3(0, 0, 0);
                        if (m.specular > 0.0f && ndotl > 0.0f) {
                            V3 V = -normalized(r.d);
                            V3 H = normalized(Ld + V);
                            float ndoth = clampf(dot(h.n, H), 0.0f, 1.0f);
                            float spec = powf(ndoth, m.shininess);
                            phong = ld3(m.specular_color) * (spec * m.specular);
                        }
                        if (!l.is_emissive && occluded(Ray{sorg, Ld}, P.bias, dist - P.bias)) continue;
                        ca = ca + ld3(l.intensity) * ndotl;
                        ce = ce + ld3(l.intensity) * phong;
                        if (li < kMaxAdjLights)
                            dlight[li] = dlight[li] + w * T * ((albedo * ndotl + phong) *
                                                               (s / (float)ns));
                    }
                    sum_a = sum_a + ca / (float)ns;
                    sum_e = sum_e + ce / (float)ns;
                }
                if (!glass) {
                    tv.E = w * T * s;
                    tv.emits = 1;
                    tv.B = (sum_a + ld3(S.amb)) * s;
                    tv.A = sum_e * s + albedo * tv.B;
                    L = L + T * tv.A;
                    if (metal) {
                        T = T * albedo * m.reflectivity;
                        tv.g = m.reflectivity;
                        r = Ray{sorg, normalized(reflect(normalized(r.d), h.n))};
                        depth--;
                        alive = depth > 0;
                        if (!alive) tv.g = 0.0f;
                        if (COUNT && alive) rc.ref++;
                    }
                    continue;
                }
                tv.A = v3(0, 0, 0);
                tv.g = 1.0f;
                dielectric = true;
            }
            if (dielectric) {
                Dielectric D = dielectric_setup(r, h, m.ior, P.bias);
                if (D.tir || rng.unit() < D.kr) r = D.refl;
                else r = D.refr;
                T = T * albedo;
                depth--;
                flags = kFlagWhitted;
                alive = depth > 0;
                if (!alive) tv.g = 0.0f;
                if (COUNT && alive) rc.ref++;
            }
        }
        Lout = L;
        return nt;
    }
};

// Held to 72 registers (seven blocks of 128 threads per SM): the tape lives
// in local memory either way, and the extra resident warps hide more of its
// latency (per gradient: 16.45 ms; 17.49 at 80 registers, 16.70 at 64).
constexpr int kAdjMinBlocks = 7;

template <bool COUNT>
__global__ void __launch_bounds__(kAdjBlock, kAdjMinBlocks)
adjoint_kernel(AdjArgs A) {
    extern __shared__ int smem[];
    TravStack<kAdjShared> stk;
    stk.sref = smem + threadIdx.x;
    stk.st = reinterpret_cast<float*>(smem + kAdjShared * blockDim.x) + threadIdx.x;
    stk.stride = blockDim.x;
    RayCount rc = {};
    const PathParams& P = A.P;
    Replay<COUNT> rp{A.S, P, stk, rc};
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long npix = (long long)P.W * P.H;
    const long long pix = gid / A.G;
    const int lane_g = (int)(gid % A.G);
    const bool active = pix < npix;
    TapeV tape[kMaxTape];
    V3 dlight[kMaxAdjLights];
    for (int k = 0; k < kMaxAdjLights; ++k) dlight[k] = v3(0, 0, 0);
    V3 acc = v3(0, 0, 0);
    V3 w = v3(0, 0, 0);
    int i = 0, j = 0;
    if (active) {
        i = (int)(pix % P.W);
        j = (int)(pix / P.W);
        const float inv = 1.0f / (float)P.spp;
        w = v3(A.dl[3 * pix] * inv, A.dl[3 * pix + 1] * inv, A.dl[3 * pix + 2] * inv);
    }
    const int per_lane = (P.spp + A.G - 1) / A.G;
    for (int q = 0; q < per_lane; ++q) {
        const int s = lane_g + q * A.G;
        int nt = 0;
        if (active && s < P.spp) {
            Rng rng{path_seed(i, j, s + P.sample_offset, P.salt)};
            float u, v;
            sample_uv(i, j, s % P.n, s / P.n, P.W, P.H, P.n, rng, u, v);
            V3 L;
            nt = rp.path(camera_ray(A.S.cam, u, v), rng, w, tape, dlight, L);
            acc = acc + L;
        }
        // backward sweep over the tape, step b of every lane together
        // (its vertex nt-1-b): each step's albedo and emission terms go
        // straight to the warp's sums, so no per-lane list is kept
        int most = nt;
        for (int off = 16; off > 0; off >>= 1)
            most = max(most, __shfl_xor_sync(0xffffffffu, most, off));
        V3 R = v3(0, 0, 0);
        for (int b = 0; b < most; ++b) {
            const bool on = b < nt;
            int mat = -1, emits = 0;
            V3 ca = v3(0, 0, 0), ce = v3(0, 0, 0);
            if (on) {
                const TapeV& tv = tape[nt - 1 - b];
                mat = tv.mat;
                if (tv.mat >= 0) {
                    const V3 a = ld3(A.S.mats[tv.mat].albedo);
                    ca = w * tv.T * (tv.B + R * tv.g);
                    R = tv.A + (a * tv.g) * R;
                    emits = tv.emits;
                    if (emits) ce = tv.E;
                } else {
                    R = tv.A;
                }
            }
            flush_contrib(mat >= 0, mat, ca, A.d_albedo);
            flush_contrib(emits != 0, mat, ce, A.d_emission);
        }
    }
    // per-light sums: reduce across the warp, one FP64 atomic per channel
    const int nl = A.S.n_lights < kMaxAdjLights ? A.S.n_lights : kMaxAdjLights;
    for (int l = 0; l < nl; ++l) {
        V3 d = dlight[l];
        for (int off = 16; off > 0; off >>= 1) {
            d.x += __shfl_xor_sync(0xffffffffu, d.x, off);
            d.y += __shfl_xor_sync(0xffffffffu, d.y, off);
            d.z += __shfl_xor_sync(0xffffffffu, d.z, off);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(A.d_light + 3 * l + 0, (double)d.x);
            atomicAdd(A.d_light + 3 * l + 1, (double)d.y);
            atomicAdd(A.d_light + 3 * l + 2, (double)d.z);
        }
    }
    // forward image of the same samples (the megakernel's lane order)
    for (int off = A.G >> 1; off > 0; off >>= 1) {
        acc.x += __shfl_xor_sync(0xffffffffu, acc.x, off);
        acc.y += __shfl_xor_sync(0xffffffffu, acc.y, off);
        acc.z += __shfl_xor_sync(0xffffffffu, acc.z, off);
    }
    if (A.out && active && lane_g == 0) {
        const float denom = (float)P.spp;
        A.out[3 * pix + 0] = acc.x / denom;
        A.out[3 * pix + 1] = acc.y / denom;
        A.out[3 * pix + 2] = acc.z / denom;
    }
    if (COUNT) {
        unsigned long long vals[3] = {rc.ext, rc.shadow, rc.ref};
        for (int k = 0; k < 3; ++k) {
            unsigned long long x = vals[k];
            for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
            if ((threadIdx.x & 31) == 0) atomicAdd(A.counters + k, x);
        }
    }
}

cudaError_t launch_adjoint(const SceneView& S, const RenderCfg& c, const float* dl,
                           double* d_albedo, double* d_emission, double* d_light, float* out,
                           unsigned long long* counters, cudaStream_t st) {
    AdjArgs A;
    A.S = S;
    A.P = PathParams{c.W, c.H, c.n, c.spp, c.depth, c.mode, c.rng, c.glass, c.soft, c.bias,
                     c.salt, c.sample_offset, 0};
    int G = 1;
    int lim = c.spp < 32 ? c.spp : 32;
    while (G * 2 <= lim) G *= 2;
    A.G = G;
    A.dl = dl;
    A.d_albedo = d_albedo;
    A.d_emission = d_emission;
    A.d_light = d_light;
    A.out = out;
    A.counters = counters;
    long long threads = (long long)c.W * c.H * G;
    unsigned blocks = (unsigned)((threads + kAdjBlock - 1) / kAdjBlock);
    size_t smem = (size_t)kAdjShared * kAdjBlock * 8;
    if (c.count) adjoint_kernel<true><<<blocks, kAdjBlock, smem, st>>>(A);
    else adjoint_kernel<false><<<blocks, kAdjBlock, smem, st>>>(A);
    return cudaGetLastError();
}

int adjoint_max_depth() { return kMaxTape; }
int adjoint_max_lights() { return kMaxAdjLights; }

}  // namespace pgpu
