// path.cuh - per-path light transport shared by the megakernel and the
// wavefront renderer: trace_path (src/renderer.hpp:829-972), the Whitted
// tracer reached through glass or used as the render mode
// (src/renderer.hpp:403-822, supported subset) and trace_dielectric
// (src/renderer.hpp:1582-1627).
#pragma once

#include "device_common.cuh"

namespace pgpu {

// Render parameters as the kernels see them.
struct PathParams {
    int W, H, n, spp, depth, mode, rng_mode, glass, soft;
    float bias;
    uint32_t salt;
    int sample_offset;
    int mis;          // 1: trace_path_mis's light weights (src/renderer.hpp:1205-1346)
    // A window of the W x H image (tile_w > 0): pixels [tile_x, tile_x +
    // tile_w) x [tile_y, tile_y + tile_h), each seeded and placed as in the
    // full image; the output holds the window's pixels.
    int tile_x, tile_y, tile_w, tile_h;
    // 1: the distributed worker's render_tile (src/distributed.hpp:380-434),
    // whose jitter is half a pixel instead of half a sub-pixel
    int worker;
};

enum { kModePT = 0, kModeWhitted = 1 };
enum { kRngCounter = 0, kRngPixel = 1 };
enum { kGlassSplit = 0, kGlassTree = 1 };

// Per-thread ray counters.
struct RayCount {
    uint32_t ext, shadow, ref;
    TravCount tc;
};

// Light direction and distance at p; soft point lights are jittered on a
// disc facing p (src/renderer.hpp:512-545 and 887-906).
__device__ __forceinline__ void light_dir(const DevLight& l, V3 p, Rng& rng, V3& L,
                                          float& dist) {
    V3 lp = ld3(l.pos);
    if (l.kind == 0 && l.radius > 0.0f) {
        V3 axis = normalized(ld3(l.pos) - p);
        V3 up = (fabsf(axis.y) < 0.9f) ? v3(0, 1, 0) : v3(1, 0, 0);
        V3 t1 = normalized(cross(axis, up));
        V3 t2 = normalized(cross(axis, t1));
        float dx, dy;
        rng.disc(dx, dy);
        lp = ld3(l.pos) + (t1 * dx + t2 * dy) * l.radius;
    }
    if (l.kind == 0) {
        V3 d = lp - p;
        dist = length(d);
        L = d / dist;
    } else {
        L = -ld3(l.pos);
        dist = 1e9f;
    }
}

// Contribution of a visible point/directional light sample at a path-trace
// vertex. trace_path (src/renderer.hpp:912-913): T * albedo * I * (n.L).
// trace_path_mis (src/renderer.hpp:1264-1297): the power-heuristic mix of the
// light-sampled term albedo * I * (n.L) and the BSDF-sampled term albedo * I,
// with a disc light's pdf taken for a light facing down (axis +y, cosine at
// least 0.01), and nothing when n.L <= 0.
__device__ __forceinline__ V3 light_term(const DevLight& l, bool mis, V3 T, V3 albedo, V3 L,
                                         float dist, float ndotl) {
    if (!mis) return T * albedo * ld3(l.intensity) * ndotl;
    if (ndotl <= 0.0f) return v3(0.0f, 0.0f, 0.0f);
    const float pdf_brdf = ndotl / 3.14159265f;
    float pdf_light;
    if (l.kind == 0 && l.radius > 0.0f) {
        const float r = l.radius;
        float cos_at_light = dot(-L, v3(0.0f, 1.0f, 0.0f));
        if (cos_at_light < 0.01f) cos_at_light = 0.01f;
        pdf_light = (dist * dist) / (3.14159265f * r * r * cos_at_light);
    } else {
        pdf_light = 1.0f;
    }
    const float w_light =
        (pdf_light * pdf_light) / (pdf_light * pdf_light + pdf_brdf * pdf_brdf + 1e-9f);
    const float w_brdf = 1.0f - w_light;
    const V3 nee = albedo * ld3(l.intensity) * ndotl;
    const V3 brdf = albedo * ld3(l.intensity);
    return T * (nee * w_light + brdf * w_brdf);
}

// trace_dielectric's two rays and Fresnel weight (src/renderer.hpp:1582-1627).
struct Dielectric {
    Ray refl, refr;
    bool tir;
    float kr;
};
__device__ __forceinline__ Dielectric dielectric_setup(const Ray& r, const Hit& h, float ior,
                                                       float bias) {
    Dielectric D;
    bool entering = h.front;
    float safe = fmaxf(ior, 0.01f);
    float eta = entering ? (1.0f / safe) : safe;
    V3 nd = normalized(r.d);
    float cos_i = fabsf(dot(nd, h.n));
    float sin_t2 = eta * eta * (1.0f - cos_i * cos_i);
    D.refl = Ray{h.p + h.n * bias, normalized(reflect(nd, h.n))};
    D.tir = sin_t2 > 1.0f;
    D.kr = 1.0f;
    if (!D.tir) {
        float cos_t = sqrtf(1.0f - sin_t2);
        D.refr = Ray{h.p - h.n * bias, normalized(nd * eta + h.n * (eta * cos_i - cos_t))};
        D.kr = schlick(entering ? cos_i : cos_t, eta);
    } else {
        D.refr = D.refl;
    }
    return D;
}

// Metal scatter of trace_path: mirror direction perturbed within radius 0.1
// (src/renderer.hpp:932-942).
__device__ __forceinline__ V3 metal_dir(V3 d, V3 n, Rng& rng) {
    V3 refl = normalized(reflect(normalized(d), n));
    V3 up = (fabsf(refl.y) < 0.9f) ? v3(0, 1, 0) : v3(1, 0, 0);
    V3 t1 = normalized(cross(refl, up));
    V3 t2 = normalized(cross(refl, t1));
    float r1 = rng.unit() * 0.1f;
    float r2 = rng.unit() * 6.28f;
    return normalized(refl + t1 * (r1 * cosf(r2)) + t2 * (r1 * sinf(r2)));
}

// Cosine-weighted hemisphere direction (src/renderer.hpp:950-960).
__device__ __forceinline__ V3 diffuse_dir(V3 N, Rng& rng) {
    float r1 = rng.unit() * 6.2831853f;
    float r2 = rng.unit();
    float r2s = sqrtf(r2);
    V3 up = (fabsf(N.y) < 0.9f) ? v3(0, 1, 0) : v3(1, 0, 0);
    V3 T = normalized(cross(up, N));
    V3 B = normalized(cross(N, T));
    return normalized(T * cosf(r1) * r2s + B * sinf(r1) * r2s + N * sqrtf(1.0f - r2));
}

// Uniform point y on a quad light, the unshadowed estimator weight
// cos_x * cos_y * area / (pi * r^2) seen from p, and the extent of the shadow
// test: the shadow ray starts at the biased origin `sorg`, so it meets the
// emitter's plane before |y - p|; visibility is tested up to that plane minus
// the bias, never against the emitter itself. Returns false when the light
// faces away.
__device__ __forceinline__ bool quad_sample(const DevLight& l, V3 p, V3 n, V3 sorg, float bias,
                                            Rng& rng, V3& L, float& tmax, float& w) {
    float u1 = rng.unit();
    float u2 = rng.unit();
    V3 y = ld3(l.pos) + ld3(l.edge_u) * u1 + ld3(l.edge_v) * u2;
    V3 d = y - p;
    float d2 = dot(d, d);
    float dist = sqrtf(d2);
    if (!(dist > 0.0f)) return false;
    L = d / dist;
    float cx = dot(n, L);
    if (cx <= 0.0f) return false;
    const V3 nq = ld3(l.normal);      // normalized(edge_u x edge_v), from the upload
    float ly = dot(nq, L);
    float cy = fabsf(ly);
    w = cx * cy * l.area / (3.14159265f * d2);
    tmax = dot(y - sorg, nq) / ly - bias;
    return w > 0.0f;
}

// ---- single-ray (Fresnel-split) path state machine ------------------------
enum : uint32_t {
    kFlagWhitted = 1u,     // following a trace() call chain (after glass / Whitted mode)
    kFlagSkipArea = 2u,    // previous vertex did quad-light NEE: skip emitter emission
};

struct PathState {
    Ray ray;
    V3 T, L;
    Rng rng;
    int depth;             // PT: remaining bounces; Whitted: depth of the next trace call
    uint32_t flags;
};

// Order-preserving sum of one vertex's next-event terms. The megakernel
// feeds shadow results as it traces them; the wavefront's shadow kernel
// replays the stored records in the same order, so both engines round
// identically. PT: L += c for each visible record, then L += tail.
// Whitted: local = base; per light, local += (sum of visible c) / ns;
// local += tail; L += w * (local * s)   (src/renderer.hpp:505-577, 652-657).
struct NeeAccum {
    int kind;              // 0 nothing pending, 1 path-trace vertex, 2 Whitted vertex
    V3 local, contrib;
    __device__ __forceinline__ void begin_none() { kind = 0; }
    __device__ __forceinline__ void begin_pt() { kind = 1; }
    __device__ __forceinline__ void begin_whitted(V3 base) {
        kind = 2;
        local = base;
        contrib = v3(0, 0, 0);
    }
    __device__ __forceinline__ void add(V3& L, V3 c, int group_end, bool visible) {
        if (kind == 1) {
            if (visible) L = L + c;
        } else {
            if (visible) contrib = contrib + c;
            if (group_end > 0) {
                local = local + contrib / (float)group_end;
                contrib = v3(0, 0, 0);
            }
        }
    }
    __device__ __forceinline__ void finish(V3& L, V3 tail, V3 w, float s) {
        if (kind == 1) {
            L = L + tail;
        } else if (kind == 2) {
            local = local + tail;
            L = L + w * (local * s);
        }
    }
};

// Shade one vertex of a single-ray path and choose its continuation.
// `found`/`h` is the closest hit of ps.ray. Next-event shadow rays go to
// E.shadow(L, ray, tmin, tmax, test, c, group_end) in order and the terms
// applied after them to E.pending(tail, w, s). Returns true when the path
// continues with ps.ray. Semantics: trace_path (src/renderer.hpp:829-972)
// and, after glass, trace (src/renderer.hpp:403-822) followed along the
// Fresnel-chosen branch of trace_dielectric (src/renderer.hpp:1582-1627).
template <class Emit>
__device__ __forceinline__ bool shade_vertex(const SceneView& S, const PathParams& P,
                                             PathState& ps, bool found, const Hit& h, Emit& E) {
    const bool whitted = (ps.flags & kFlagWhitted) != 0;
    if (!found) {
        ps.L = ps.L + ps.T * ld3(S.bg);
        return false;
    }
    const DevMaterial& m = S.mats[h.mat];
    const V3 albedo = ld3(m.albedo);
    const bool metal = m.kind == 1 && m.reflectivity > 0.0f;
    const bool glass = m.kind == 2;
    const V3 sorg = h.p + h.n * P.bias;
    if (!whitted) {
        const bool diffuse = !metal && !glass;
        if (!glass && !((ps.flags & kFlagSkipArea) && m.area_emitter))
            ps.L = ps.L + ps.T * ld3(m.emission);
        E.begin_pt();
        for (int li = 0; li < S.n_lights; ++li) {
            const DevLight& l = S.lights[li];
            if (l.kind == 2) continue;
            V3 L;
            float dist;
            light_dir(l, h.p, ps.rng, L, dist);
            float ndotl = clampf(dot(h.n, L), 0.0f, 1.0f);
            E.shadow(ps.L, Ray{sorg, L}, P.bias, dist - P.bias, !l.is_emissive,
                     light_term(l, P.mis != 0, ps.T, albedo, L, dist, ndotl), 0);
        }
        if (S.has_quad_lights && diffuse && ps.depth - 1 > 0) {
            for (int li = 0; li < S.n_lights; ++li) {
                const DevLight& l = S.lights[li];
                if (l.kind != 2) continue;
                V3 L;
                float tmax, w;
                if (!quad_sample(l, h.p, h.n, sorg, P.bias, ps.rng, L, tmax, w)) continue;
                E.shadow(ps.L, Ray{sorg, L}, P.bias, tmax, true,
                         ps.T * albedo * ld3(l.intensity) * w, 0);
            }
        }
        E.pending(ps.T * albedo * ld3(S.amb), v3(0, 0, 0), 0.0f);
        if (P.depth - ps.depth > 3) {
            float p = fmaxf(ps.T.x, fmaxf(ps.T.y, ps.T.z));
            if (ps.rng.unit() > p) return false;
            ps.T = ps.T / p;
        }
        if (!glass) {
            V3 nd;
            if (metal) {
                nd = metal_dir(ps.ray.d, h.n, ps.rng);
                ps.T = ps.T * albedo * m.reflectivity;
            } else {
                nd = diffuse_dir(h.n, ps.rng);
                ps.T = ps.T * albedo;
            }
            ps.flags = (diffuse && S.has_quad_lights) ? kFlagSkipArea : 0u;
            ps.ray = Ray{sorg, nd};
            ps.depth--;
            return ps.depth > 0;
        }
    } else {
        if (glass) E.begin_none();
        else E.begin_whitted(ld3(m.emission));
        for (int li = 0; li < S.n_lights; ++li) {
            const DevLight& l = S.lights[li];
            if (l.kind == 2) continue;
            int ns = (l.radius > 0.0f) ? P.soft : 1;
            for (int k = 0; k < ns; ++k) {
                V3 L;
                float dist;
                light_dir(l, h.p, ps.rng, L, dist);
                if (glass) continue;
                float ndotl = clampf(dot(h.n, L), 0.0f, 1.0f);
                V3 c = albedo * ld3(l.intensity) * ndotl;
                if (m.specular > 0.0f && ndotl > 0.0f) {
                    V3 V = -normalized(ps.ray.d);
                    V3 H = normalized(L + V);
                    float ndoth = clampf(dot(h.n, H), 0.0f, 1.0f);
                    float spec = powf(ndoth, m.shininess);
                    c = c + ld3(m.specular_color) * ld3(l.intensity) * (spec * m.specular);
                }
                E.shadow(ps.L, Ray{sorg, L}, P.bias, dist - P.bias, !l.is_emissive, c,
                         k == ns - 1 ? ns : 0);
            }
        }
        if (!glass) {
            if (metal) {
                E.pending(albedo * ld3(S.amb), ps.T, 1.0f - m.reflectivity);
                ps.T = ps.T * albedo * m.reflectivity;
                ps.ray = Ray{sorg, normalized(reflect(normalized(ps.ray.d), h.n))};
                ps.depth--;
                return ps.depth > 0;
            }
            E.pending(albedo * ld3(S.amb), ps.T, 1.0f);
            return false;
        }
    }
    // dielectric: follow one branch of trace_dielectric, chosen with the
    // Fresnel weight (always the reflection under total internal reflection)
    Dielectric D = dielectric_setup(ps.ray, h, m.ior, P.bias);
    if (D.tir || ps.rng.unit() < D.kr) ps.ray = D.refl;
    else ps.ray = D.refr;
    ps.T = ps.T * albedo;
    ps.depth--;
    ps.flags = kFlagWhitted;
    return ps.depth > 0;
}

// One path traced to the end by one thread (megakernel). WIDE: traversal of
// the 4-wide tree the wavefront walks (ClosestTrav4/AnyTrav4); otherwise
// Pencil's binary tree (the tree BVHNode::hit walks, src/bvh.hpp:31-48) in
// its child-pair layout, nearest child first.
template <int kShared, bool COUNT, bool WIDE = false>
struct Tracer {
    const SceneView& S;
    const PathParams& P;
    TravStack<kShared>& stk;
    RayCount& rc;

    __device__ __forceinline__ int closest(const Ray& r, Hit& h) {
        if (COUNT) rc.ext++;
        float tb;
        int bref;
        int slot = WIDE ? closest_hit4<kShared, COUNT>(S, r, 1e-4f, 1e9f, tb, bref, stk, &rc.tc)
                        : closest_hit<kShared, COUNT>(S, r, 1e-4f, 1e9f, tb, bref, stk, &rc.tc);
        if (slot >= 0) make_hit(S, bref, slot, r, 1e-4f, tb, h);
        return slot;
    }
    __device__ __forceinline__ bool occluded(const Ray& r, float tmin, float tmax) {
        if (COUNT) rc.shadow++;
        return WIDE ? any_hit4<kShared, COUNT>(S, r, tmin, tmax, stk, &rc.tc)
                    : any_hit<kShared, COUNT>(S, r, tmin, tmax, stk, &rc.tc);
    }

    // Direct light of a Whitted vertex: emission + point/directional lights
    // with soft-shadow samples and Phong + ambient (src/renderer.hpp:482-577).
    // For glass the shadow rays are skipped (its local colour is replaced by
    // trace_dielectric) but the random numbers are still drawn.
    __device__ V3 whitted_local(const Ray& r, const Hit& h, const DevMaterial& m, Rng& rng,
                                bool shade) {
        V3 albedo = ld3(m.albedo);
        V3 local = ld3(m.emission);
        for (int li = 0; li < S.n_lights; ++li) {
            const DevLight& l = S.lights[li];
            if (l.kind == 2) continue;
            V3 contrib = v3(0, 0, 0);
            int ns = (l.radius > 0.0f) ? P.soft : 1;
            for (int k = 0; k < ns; ++k) {
                V3 L;
                float dist;
                light_dir(l, h.p, rng, L, dist);
                if (!shade) continue;
                Ray sr{h.p + h.n * P.bias, L};
                if (!l.is_emissive && occluded(sr, P.bias, dist - P.bias)) continue;
                float ndotl = clampf(dot(h.n, L), 0.0f, 1.0f);
                V3 c = albedo * ld3(l.intensity) * ndotl;
                if (m.specular > 0.0f && ndotl > 0.0f) {
                    V3 V = -normalized(r.d);
                    V3 H = normalized(L + V);
                    float ndoth = clampf(dot(h.n, H), 0.0f, 1.0f);
                    float spec = powf(ndoth, m.shininess);
                    c = c + ld3(m.specular_color) * ld3(l.intensity) * (spec * m.specular);
                }
                contrib = contrib + c;
            }
            local = local + contrib / (float)ns;
        }
        return local + albedo * ld3(S.amb);
    }

    // trace(r, depth) evaluated as Pencil's recursion does: both dielectric
    // branches, results combined bottom-up in the reference's order. With
    // start_glass the evaluation starts at trace_dielectric(r0, h0, ...) of a
    // path-trace vertex instead of at a trace call.
    struct Frame {
        int kind;          // 0 metal, 1 glass awaiting reflection, 2 awaiting refraction
        int child_depth;
        float w;           // metal reflectivity or glass kr
        V3 albedo;
        V3 acc;            // metal: local colour; glass: reflected colour
        Ray refr;
        bool tir;
    };
    static constexpr int kMaxFrames = 32;

    __device__ V3 whitted_tree(Ray r, int depth, Rng& rng, bool start_glass, const Hit* h0,
                               const DevMaterial* m0) {
        Frame F[kMaxFrames];
        int sp = 0;
        V3 ret;
        if (start_glass) {
            Dielectric D = dielectric_setup(r, *h0, m0->ior, P.bias);
            F[0] = Frame{1, depth - 1, D.kr, ld3(m0->albedo), v3(0, 0, 0), D.refr, D.tir};
            sp = 1;
            r = D.refl;
            depth = depth - 1;
        }
        while (true) {
            // descend: evaluate trace(r, depth) until it needs a child
            bool need_child = false;
            if (COUNT) rc.ref++;
            if (depth <= 0) {
                ret = v3(0, 0, 0);
            } else {
                Hit h;
                if (closest(r, h) < 0) {
                    ret = ld3(S.bg);
                } else {
                    const DevMaterial& m = S.mats[h.mat];
                    bool glass = m.kind == PGPU_MAT_DIELECTRIC_;
                    V3 local = whitted_local(r, h, m, rng, !glass);
                    if (m.kind == 1 && m.reflectivity > 0.0f && sp < kMaxFrames) {
                        F[sp++] = Frame{0, depth - 1, m.reflectivity, ld3(m.albedo), local, r, false};
                        r = Ray{h.p + h.n * P.bias, normalized(reflect(normalized(r.d), h.n))};
                        depth = depth - 1;
                        need_child = true;
                    } else if (glass && sp < kMaxFrames) {
                        Dielectric D = dielectric_setup(r, h, m.ior, P.bias);
                        F[sp++] = Frame{1, depth - 1, D.kr, ld3(m.albedo), v3(0, 0, 0), D.refr, D.tir};
                        r = D.refl;
                        depth = depth - 1;
                        need_child = true;
                    } else {
                        ret = local;
                    }
                }
            }
            if (need_child) continue;
            // ascend: fold the result into pending frames
            bool descend = false;
            while (sp > 0 && !descend) {
                Frame& f = F[sp - 1];
                if (f.kind == 0) {
                    ret = f.acc * (1.0f - f.w) + ret * f.albedo * f.w;
                    --sp;
                } else if (f.kind == 1) {
                    if (f.tir) {
                        ret = ret * f.albedo;
                        --sp;
                    } else {
                        f.acc = ret;
                        f.kind = 2;
                        r = f.refr;
                        depth = f.child_depth;
                        descend = true;
                    }
                } else {
                    ret = (f.acc * f.w + ret * (1.0f - f.w)) * f.albedo;
                    --sp;
                }
            }
            if (!descend) return ret;
        }
    }

    static constexpr int PGPU_MAT_DIELECTRIC_ = 2;

    // One camera sample. TREE: both glass branches (Pencil's recursion, used
    // with the per-pixel RNG for bit-level comparison); otherwise the
    // Fresnel-split single-ray continuation.
    template <bool TREE>
    __device__ V3 sample(Ray r, Rng& rng) {
        if (P.mode == kModeWhitted) {
            if (TREE) return whitted_tree(r, P.depth, rng, false, nullptr, nullptr);
            return split_path(r, rng, true);
        }
        if (!TREE) return split_path(r, rng, false);
        // trace_path with Pencil's glass recursion
        if (COUNT) rc.ref++;
        V3 T = v3(1, 1, 1), rad = v3(0, 0, 0);
        int bounces = P.depth, depth = bounces;
        bool skip_area = false;
        while (depth > 0) {
            Hit h;
            if (closest(r, h) < 0) {
                rad = rad + T * ld3(S.bg);
                break;
            }
            const DevMaterial& m = S.mats[h.mat];
            if (!(skip_area && m.area_emitter)) rad = rad + T * ld3(m.emission);
            V3 albedo = ld3(m.albedo);
            bool diffuse = !(m.kind == 1 && m.reflectivity > 0.0f) && m.kind != 2;
            pt_direct(h, m, T, rng, rad, diffuse && depth - 1 > 0);
            if (bounces - depth > 3) {
                float p = fmaxf(T.x, fmaxf(T.y, T.z));
                if (rng.unit() > p) break;
                T = T / p;
            }
            V3 nT = T * albedo;
            V3 nd;
            if (m.kind == 1 && m.reflectivity > 0.0f) {
                nd = metal_dir(r.d, h.n, rng);
                nT = T * albedo * m.reflectivity;
            } else if (m.kind == 2) {
                V3 g = whitted_tree(r, depth, rng, true, &h, &m);
                rad = rad + (T * g - T * ld3(m.emission));
                break;
            } else {
                nd = diffuse_dir(h.n, rng);
            }
            skip_area = diffuse && S.has_quad_lights;
            r = Ray{h.p + h.n * P.bias, nd};
            T = nT;
            depth--;
        }
        return rad;
    }

    // NEE and ambient of a path-trace vertex (src/renderer.hpp:886-919), plus
    // quad-light NEE at diffuse vertices whose bounce would be traced.
    __device__ __forceinline__ void pt_direct(const Hit& h, const DevMaterial& m, V3 T, Rng& rng,
                                              V3& rad, bool quad_nee) {
        V3 albedo = ld3(m.albedo);
        for (int li = 0; li < S.n_lights; ++li) {
            const DevLight& l = S.lights[li];
            if (l.kind == 2) continue;
            V3 L;
            float dist;
            light_dir(l, h.p, rng, L, dist);
            Ray sr{h.p + h.n * P.bias, L};
            if (!l.is_emissive && occluded(sr, P.bias, dist - P.bias)) continue;
            float ndotl = clampf(dot(h.n, L), 0.0f, 1.0f);
            rad = rad + light_term(l, P.mis != 0, T, albedo, L, dist, ndotl);
        }
        if (quad_nee) {
            for (int li = 0; li < S.n_lights; ++li) {
                const DevLight& l = S.lights[li];
                if (l.kind != 2) continue;
                V3 L;
                float tmax, w;
                V3 sorg = h.p + h.n * P.bias;
                if (!quad_sample(l, h.p, h.n, sorg, P.bias, rng, L, tmax, w)) continue;
                Ray sr{sorg, L};
                if (occluded(sr, P.bias, tmax)) continue;
                rad = rad + T * albedo * ld3(l.intensity) * w;
            }
        }
        rad = rad + T * albedo * ld3(S.amb);
    }

    // Single-ray path (Fresnel-split glass): shade_vertex with every shadow
    // ray resolved on the spot.
    __device__ V3 split_path(Ray r, Rng& rng, bool whitted) {
        PathState ps;
        ps.ray = r;
        ps.T = v3(1, 1, 1);
        ps.L = v3(0, 0, 0);
        ps.rng = rng;
        ps.depth = P.depth;
        ps.flags = whitted ? kFlagWhitted : 0;
        if (COUNT) rc.ref++;
        bool alive = ps.depth > 0;
        while (alive) {
            Hit h;
            bool found = closest(ps.ray, h) >= 0;
            InlineNee emit{*this};
            alive = shade_vertex(S, P, ps, found, h, emit);
            emit.acc.finish(ps.L, emit.tail, emit.w, emit.s);
            if (COUNT && alive && (ps.flags & kFlagWhitted)) rc.ref++;
        }
        rng = ps.rng;
        return ps.L;
    }

    // Shadow rays of one vertex traced as they are made.
    struct InlineNee {
        Tracer& tr;
        NeeAccum acc;
        V3 tail, w;
        float s;
        __device__ InlineNee(Tracer& t) : tr(t), tail(v3(0, 0, 0)), w(v3(0, 0, 0)), s(0.0f) {
            acc.kind = 0;
        }
        __device__ __forceinline__ void begin_none() { acc.begin_none(); }
        __device__ __forceinline__ void begin_pt() { acc.begin_pt(); }
        __device__ __forceinline__ void begin_whitted(V3 base) { acc.begin_whitted(base); }
        __device__ __forceinline__ void shadow(V3& L, const Ray& sr, float tmin, float tmax,
                                               bool test, V3 c, int group_end) {
            bool vis = !test || !tr.occluded(sr, tmin, tmax);
            acc.add(L, c, group_end, vis);
        }
        __device__ __forceinline__ void pending(V3 tl, V3 ww, float ss) { tail = tl; w = ww; s = ss; }
    };
};

}  // namespace pgpu
