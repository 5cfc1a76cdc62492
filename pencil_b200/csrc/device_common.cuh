// device_common.cuh - device functions shared by every renderer: Pencil's
// float32 arithmetic (compiled with --fmad=false, IEEE division and square
// root, so that each expression rounds exactly as the reference's x86-64
// build does), xorshift32 sampling, camera rays, primitive tests and BVH
// traversal.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "scene_layout.h"

namespace pgpu {

// ---- Vec3 (src/vec3.hpp:24-92) -----------------------------------------------
struct V3 {
    float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ V3 operator/(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ V3 operator*(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float length(V3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ V3 normalized(V3 a) {
    float l = length(a);
    return (l > 1e-12f) ? a / l : v3(0.0f, 0.0f, 0.0f);
}
__device__ __forceinline__ V3 reflect(V3 v, V3 n) { return v - n * (2.0f * dot(v, n)); }
__device__ __forceinline__ float clampf(float v, float lo, float hi) {
    return (v < lo) ? lo : (v > hi) ? hi : v;
}
__device__ __forceinline__ float schlick(float c, float ratio) {
    float r0 = (1.0f - ratio) / (1.0f + ratio);
    r0 = r0 * r0;
    return r0 + (1.0f - r0) * powf(1.0f - c, 5.0f);
}
__device__ __forceinline__ V3 ld3(const float* p) { return v3(p[0], p[1], p[2]); }
__device__ __forceinline__ float comp(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
__device__ __forceinline__ void set_comp(V3& a, int i, float v) {
    if (i == 0) a.x = v; else if (i == 1) a.y = v; else a.z = v;
}

// ---- Rng (src/rng.hpp:13-45) --------------------------------------------------
struct Rng {
    uint32_t s;
    __device__ __forceinline__ uint32_t u32() {
        s ^= s << 13u;
        s ^= s >> 17u;
        s ^= s << 5u;
        return s;
    }
    __device__ __forceinline__ float unit() { return (float)u32() / 4294967296.0f; }
    __device__ __forceinline__ float sym() { return unit() * 2.0f - 1.0f; }
    __device__ __forceinline__ void disc(float& dx, float& dy) {
        float r1 = unit();
        float r2 = unit();
        float sx = 2.0f * r1 - 1.0f;
        float sy = 2.0f * r2 - 1.0f;
        if (sx == 0.0f && sy == 0.0f) { dx = 0.0f; dy = 0.0f; return; }
        float theta, r;
        if (fabsf(sx) > fabsf(sy)) {
            r = sx;
            theta = (3.14159265f / 4.0f) * (sy / sx);
        } else {
            r = sy;
            theta = (3.14159265f / 2.0f) - (3.14159265f / 4.0f) * (sx / sy);
        }
        dx = r * cosf(theta);
        dy = r * sinf(theta);
    }
};

__device__ __forceinline__ uint32_t mix32(uint32_t x) {
    x ^= x >> 16; x *= 0x7feb352dU;
    x ^= x >> 15; x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

// Counter-RNG seed of path (pixel i, j; sample s): Pencil's per-pixel seed
// (src/renderer.hpp:313) hashed with the sample index.
__device__ __forceinline__ uint32_t path_seed(int i, int j, int sample, uint32_t salt) {
    uint32_t pix = (uint32_t)i * 97861u + (uint32_t)j * 1973u + 1u;
    uint32_t s = mix32(pix ^ mix32((uint32_t)sample * 0x9E3779B9u + salt + 0x632BE5ABu));
    return s ? s : 0x6D2B79F5u;
}
__device__ __forceinline__ uint32_t pixel_seed(int i, int j) {
    return (uint32_t)i * 97861u + (uint32_t)j * 1973u + 1u;
}

// ---- rays ------------------------------------------------------------------------
struct Ray {
    V3 o, d;
};

// Camera::ray_at without aperture (src/camera.cpp:48-68).
__device__ __forceinline__ Ray camera_ray(const float* cam, float u, float v) {
    V3 org = ld3(cam), ll = ld3(cam + 3), hor = ld3(cam + 6), ver = ld3(cam + 9);
    V3 dir = ll + hor * u + ver * v - org;
    return Ray{org, normalized(dir)};
}

// Jittered image-plane point of sample (sx, sy) (src/renderer.hpp:363-366);
// `tile`: the distributed worker's jitter of half a pixel
// (src/distributed.hpp:416-419).
__device__ __forceinline__ void sample_uv(int i, int j, int sx, int sy, int W, int H, int n,
                                          Rng& rng, float& u, float& v, bool tile = false) {
    u = (i + (sx + 0.5f) / n) / (float)W;
    v = 1.0f - (j + (sy + 0.5f) / n) / (float)H;
    u += rng.sym() * (tile ? 0.5f / W : 0.5f / (W * n));
    v += rng.sym() * (tile ? 0.5f / H : 0.5f / (H * n));
}

// Per-ray constants of the slab test. AABB::hit (src/primitives.hpp:38-49)
// recomputes 1/d for every box; computing it once gives the same value.
struct RayPre {
    V3 o, inv;
    bool nx, ny, nz;  // inv < 0: near plane is the box max
    int ox, oy, oz;   // wide nodes: row of the near planes (0: lo, 3: hi), times G
};
__device__ __forceinline__ RayPre prep(const Ray& r) {
    RayPre p;
    p.o = r.o;
    p.inv = v3(1.0f / r.d.x, 1.0f / r.d.y, 1.0f / r.d.z);
    p.nx = p.inv.x < 0.0f;
    p.ny = p.inv.y < 0.0f;
    p.nz = p.inv.z < 0.0f;
    p.ox = p.nx ? 3 : 0;
    p.oy = p.ny ? 3 : 0;
    p.oz = p.nz ? 3 : 0;
    return p;
}

// Three-input min/max (PTX ISA 8.8, sm_100). Like fminf/fmaxf they ignore
// NaN operands; min and max round nothing, so any grouping gives the same
// value.
__device__ __forceinline__ float fmax3f(float a, float b, float c) {
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float fmin3f(float a, float b, float c) {
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// AABB::hit: sequential per-axis clipping with NaN-ignoring selects equals
// clipping by the max of near distances and the min of far distances.
// `entry` returns the clipped entry distance (independent of tmax).
__device__ __forceinline__ bool slab(float lox, float loy, float loz, float hix, float hiy,
                                     float hiz, const RayPre& r, float tmin, float tmax,
                                     float& entry) {
    float t0x = ((r.nx ? hix : lox) - r.o.x) * r.inv.x;
    float t1x = ((r.nx ? lox : hix) - r.o.x) * r.inv.x;
    float t0y = ((r.ny ? hiy : loy) - r.o.y) * r.inv.y;
    float t1y = ((r.ny ? loy : hiy) - r.o.y) * r.inv.y;
    float t0z = ((r.nz ? hiz : loz) - r.o.z) * r.inv.z;
    float t1z = ((r.nz ? loz : hiz) - r.o.z) * r.inv.z;
    float en = fmax3f(fmaxf(tmin, t0x), t0y, t0z);
    float ex = fmin3f(fminf(tmax, t1x), t1y, t1z);
    entry = en;
    return !(ex < en);
}

// ---- primitives (src/primitives.hpp) --------------------------------------------
struct Hit {
    V3 p, n;
    float t;
    int mat;
    bool front;
};

__device__ __forceinline__ void set_face(Hit& h, const Ray& r, V3 outward) {
    h.front = dot(r.d, outward) < 0.0f;
    h.n = h.front ? outward : -outward;
}

// Sphere::hit (src/primitives.hpp:98-120)
template <bool REC>
__device__ __forceinline__ bool hit_sphere(float4 g, const Ray& r, float tmin, float tmax,
                                           float& t_out, Hit* h) {
    V3 c = v3(g.x, g.y, g.z);
    float rad = g.w;
    V3 oc = r.o - c;
    float a = dot(r.d, r.d);
    float hb = dot(oc, r.d);
    float cc = dot(oc, oc) - rad * rad;
    float disc = hb * hb - a * cc;
    if (disc < 0.0f) return false;
    float sq = sqrtf(disc);
    float t = (-hb - sq) / a;
    if (t < tmin || t > tmax) {
        t = (-hb + sq) / a;
        if (t < tmin || t > tmax) return false;
    }
    t_out = t;
    if (REC) {
        h->t = t;
        h->p = r.o + r.d * t;
        set_face(*h, r, (h->p - c) / rad);
    }
    return true;
}

// Triangle::hit, Moller-Trumbore (src/primitives.hpp:145-170)
// The edges e1 = v1 - v0 and e2 = v2 - v0 come rounded as the reference
// rounds them (the upload stores them in the leaf slot).
template <bool REC>
__device__ __forceinline__ bool hit_triangle(V3 v0, V3 e1, V3 e2, const Ray& r, float tmin,
                                             float tmax, float& t_out, Hit* h) {
    V3 hh = cross(r.d, e2);
    float a = dot(e1, hh);
    if (fabsf(a) < 1e-8f) return false;
    float f = 1.0f / a;
    V3 s = r.o - v0;
    float u = f * dot(s, hh);
    if (u < 0.0f || u > 1.0f) return false;
    V3 q = cross(s, e1);
    float v = f * dot(r.d, q);
    if (v < 0.0f || u + v > 1.0f) return false;
    float t = f * dot(e2, q);
    if (t < tmin || t > tmax) return false;
    t_out = t;
    if (REC) {
        h->t = t;
        h->p = r.o + r.d * t;
        set_face(*h, r, normalized(cross(e1, e2)));
    }
    return true;
}

// Cube::hit (src/primitives.hpp:201-238)
template <bool REC>
__device__ __forceinline__ bool hit_cube(float4 g, const Ray& r, float tmin, float tmax,
                                         float& t_out, Hit* h) {
    V3 c = v3(g.x, g.y, g.z);
    float hf = g.w;
    V3 lo = c - v3(hf, hf, hf);
    V3 hi = c + v3(hf, hf, hf);
    float t_near = -INFINITY, t_far = INFINITY;
    int near_axis = -1, far_axis = -1;
    float near_sign = 1.0f, far_sign = -1.0f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float d = comp(r.d, a);
        const float o = comp(r.o, a);
        if (fabsf(d) < 1e-12f) {
            if (o < comp(lo, a) || o > comp(hi, a)) return false;
            continue;
        }
        float tn = (comp(lo, a) - o) / d;
        float tf = (comp(hi, a) - o) / d;
        float ns = -1.0f, fs = 1.0f;
        if (tn > tf) {
            float x = tn; tn = tf; tf = x;
            x = ns; ns = fs; fs = x;
        }
        if (tn > t_near) { t_near = tn; near_axis = a; near_sign = ns; }
        if (tf < t_far) { t_far = tf; far_axis = a; far_sign = fs; }
        if (t_far < t_near) return false;
    }
    const bool use_near = t_near >= tmin;
    const float th = use_near ? t_near : t_far;
    const int ax = use_near ? near_axis : far_axis;
    const float sg = use_near ? near_sign : far_sign;
    if (ax < 0 || th < tmin || th > tmax) return false;
    t_out = th;
    if (REC) {
        h->t = th;
        h->p = r.o + r.d * th;
        V3 n = v3(0.0f, 0.0f, 0.0f);
        set_comp(n, ax, sg);
        set_face(*h, r, n);
    }
    return true;
}

// Plane::hit (src/primitives.hpp:261-272)
template <bool REC>
__device__ __forceinline__ bool hit_plane(float4 ga, float4 gb, const Ray& r, float tmin,
                                          float tmax, float& t_out, Hit* h) {
    V3 pt = v3(ga.x, ga.y, ga.z), n = v3(gb.x, gb.y, gb.z);
    float denom = dot(n, r.d);
    if (fabsf(denom) < 1e-6f) return false;
    float t = dot(pt - r.o, n) / denom;
    if (t < tmin || t > tmax) return false;
    t_out = t;
    if (REC) {
        h->t = t;
        h->p = r.o + r.d * t;
        set_face(*h, r, n);
    }
    return true;
}

// Disc cap shared by Cylinder::hit_cap and Cone::hit_base
// (src/primitives.hpp:486-504, 588-605).
template <bool REC>
__device__ __forceinline__ bool hit_disc(V3 center, V3 n, float rad, const Ray& r, float tmin,
                                         float tmax, float& t_out, Hit* h) {
    float denom = dot(n, r.d);
    if (fabsf(denom) < 1e-6f) return false;
    float t = dot(center - r.o, n) / denom;
    if (t < tmin || t > tmax) return false;
    V3 p = r.o + r.d * t;
    V3 d = p - center;
    if (dot(d, d) > rad * rad) return false;
    t_out = t;
    if (REC) {
        h->t = t;
        h->p = p;
        set_face(*h, r, n);
    }
    return true;
}

// Cylinder::hit_side (src/primitives.hpp:440-484)
template <bool REC>
__device__ __forceinline__ bool cyl_side(V3 c, V3 ax, float rad, float hh, const Ray& r,
                                         float tmin, float tmax, float& t_out, Hit* h) {
    V3 oc = r.o - c;
    float dda = dot(r.d, ax);
    float oca = dot(oc, ax);
    V3 dp = r.d - ax * dda;
    V3 op = oc - ax * oca;
    float a = dot(dp, dp);
    float b = 2.0f * dot(op, dp);
    float cc = dot(op, op) - rad * rad;
    if (a < 1e-9f) {
        if (fabsf(b) < 1e-9f) return false;
        const float t = -cc / b;
        if (t < tmin || t > tmax) return false;
        const float hgt = oca + t * dda;
        if (fabsf(hgt) > hh) return false;
        t_out = t;
        if (REC) {
            h->t = t;
            h->p = r.o + r.d * t;
            set_face(*h, r, (h->p - (c + ax * hgt)) / rad);
        }
        return true;
    }
    float disc = b * b - 4.0f * a * cc;
    if (disc < 0.0f) return false;
    float sq = sqrtf(disc);
    float t0 = (-b - sq) / (2.0f * a);
    float t1 = (-b + sq) / (2.0f * a);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        float t = k == 0 ? t0 : t1;
        if (t < tmin || t > tmax) continue;
        float hgt = (oca + t * dda);
        if (fabsf(hgt) > hh) continue;
        t_out = t;
        if (REC) {
            h->t = t;
            h->p = r.o + r.d * t;
            set_face(*h, r, (h->p - (c + ax * hgt)) / rad);
        }
        return true;
    }
    return false;
}

// Cylinder::hit (src/primitives.hpp:406-422)
template <bool REC>
__device__ __forceinline__ bool hit_cylinder(float4 ga, float4 gb, const Ray& r, float tmin,
                                             float tmax, float& t_out, Hit* h) {
    V3 c = v3(ga.x, ga.y, ga.z), ax = v3(gb.x, gb.y, gb.z);
    float rad = ga.w, hh = gb.w;
    bool found = false;
    float closest = tmax, t;
    if (cyl_side<REC>(c, ax, rad, hh, r, tmin, closest, t, h)) { closest = t; found = true; }
    if (hit_disc<REC>(c + ax * (1.0f * hh), ax * 1.0f, rad, r, tmin, closest, t, h)) {
        closest = t; found = true;
    }
    if (hit_disc<REC>(c + ax * (-1.0f * hh), ax * -1.0f, rad, r, tmin, closest, t, h)) {
        closest = t; found = true;
    }
    t_out = closest;
    return found;
}

// Cone::hit_side (src/primitives.hpp:551-586)
template <bool REC>
__device__ __forceinline__ bool cone_side(V3 apex, V3 ax, float rad, float hgt, const Ray& r,
                                          float tmin, float tmax, float& t_out, Hit* h) {
    V3 oc = r.o - apex;
    float dda = dot(r.d, ax);
    float oca = dot(oc, ax);
    float k = rad / hgt;
    float k2 = k * k;
    V3 dp = r.d - ax * dda;
    V3 op = oc - ax * oca;
    float a = dot(dp, dp) - k2 * dda * dda;
    float b = 2.0f * (dot(dp, op) - k2 * dda * oca);
    float cc = dot(op, op) - k2 * oca * oca;
    float disc = b * b - 4.0f * a * cc;
    if (disc < 0.0f || fabsf(a) < 1e-12f) return false;
    float sq = sqrtf(disc);
    float t0 = (-b - sq) / (2.0f * a);
    float t1 = (-b + sq) / (2.0f * a);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        float t = q == 0 ? t0 : t1;
        if (t < tmin || t > tmax) continue;
        float hh = oca + t * dda;
        if (hh < 0.0f || hh > hgt) continue;
        t_out = t;
        if (REC) {
            h->t = t;
            h->p = r.o + r.d * t;
            V3 radial = h->p - (apex + ax * hh);
            set_face(*h, r, normalized(normalized(radial) - ax * k));
        }
        return true;
    }
    return false;
}

// Cone::hit (src/primitives.hpp:517-531)
template <bool REC>
__device__ __forceinline__ bool hit_cone(float4 ga, float4 gb, const Ray& r, float tmin,
                                         float tmax, float& t_out, Hit* h) {
    V3 apex = v3(ga.x, ga.y, ga.z), ax = v3(gb.x, gb.y, gb.z);
    float rad = ga.w, hgt = gb.w;
    V3 base = apex - ax * hgt;
    bool found = false;
    float closest = tmax, t;
    if (cone_side<REC>(apex, ax, rad, hgt, r, tmin, closest, t, h)) { closest = t; found = true; }
    if (hit_disc<REC>(base, -ax, rad, r, tmin, closest, t, h)) { closest = t; found = true; }
    t_out = closest;
    return found;
}

// Test one leaf. With REC the full hit record (point, face normal) is made.
template <bool REC>
__device__ __forceinline__ bool hit_leaf(const SceneView& S, int ref, const Ray& r, float tmin,
                                         float tmax, float& t, Hit* h) {
    int code = ~ref;
    int type = code >> kLeafTypeShift;
    int slot = code & kLeafSlotMask;
    float4 ga = __ldg(S.geo_a + slot);
    switch (type) {
        case LEAF_SPHERE:
            return hit_sphere<REC>(ga, r, tmin, tmax, t, h);
        case LEAF_TRIANGLE: {
            const float4 b = __ldg(S.geo_b + slot), c = __ldg(S.geo_c + slot);
            return hit_triangle<REC>(v3(ga.x, ga.y, ga.z), v3(b.x, b.y, b.z), v3(c.x, c.y, c.z),
                                     r, tmin, tmax, t, h);
        }
        case LEAF_CUBE:
            return hit_cube<REC>(ga, r, tmin, tmax, t, h);
        case LEAF_PLANE:
            return hit_plane<REC>(ga, __ldg(S.geo_b + slot), r, tmin, tmax, t, h);
        case LEAF_CYLINDER:
            return hit_cylinder<REC>(ga, __ldg(S.geo_b + slot), r, tmin, tmax, t, h);
        case LEAF_CONE:
            return hit_cone<REC>(ga, __ldg(S.geo_b + slot), r, tmin, tmax, t, h);
        default:
            return false;
    }
}

// Bytes a leaf test reads (for the algorithmic-byte counters).
__device__ __forceinline__ int leaf_bytes(int ref) {
    int type = (~ref) >> kLeafTypeShift;
    switch (type) {
        case LEAF_SPHERE: case LEAF_CUBE: return 16;
        case LEAF_TRIANGLE: return 3 * 16;
        default: return 32;
    }
}

// ---- traversal -----------------------------------------------------------------
// Counters of one thread's traversal work (used when COUNT is set).
struct TravCount {
    uint32_t nodes;
    uint32_t leaf_bytes;
    uint32_t prims;
};

constexpr int kMaxStack = 64;   // the uploader rejects deeper trees

// Per-thread traversal stack: the top kShared entries live in shared memory
// (this warp's slice of the block's stack array, column per lane), deeper
// entries spill to local memory.
template <int kShared>
struct TravStack {
    int* sref;      // shared: sref[level * stride]
    float* st;      // shared: st[level * stride]
    int stride;
    int lref[kMaxStack - kShared];
    float lt[kMaxStack - kShared];
    __device__ __forceinline__ void push(int sp, int ref, float t) {
        if (sp < kShared) { sref[sp * stride] = ref; st[sp * stride] = t; }
        else { lref[sp - kShared] = ref; lt[sp - kShared] = t; }
    }
    __device__ __forceinline__ void pop(int sp, int& ref, float& t) const {
        if (sp < kShared) { ref = sref[sp * stride]; t = st[sp * stride]; }
        else { ref = lref[sp - kShared]; t = lt[sp - kShared]; }
    }
    // any hit: the entries carry no distance
    __device__ __forceinline__ void push_ref(int sp, int ref) {
        if (sp < kShared) sref[sp * stride] = ref;
        else lref[sp - kShared] = ref;
    }
    __device__ __forceinline__ int pop_ref(int sp) const {
        return sp < kShared ? sref[sp * stride] : lref[sp - kShared];
    }
};

// Resumable closest-hit traversal: init() tests the root, step() processes
// one interior node; both return true once the traversal has finished.
// Result: the primitive with the smallest t in [tmin, tmax]; among equal t
// the one later in DFS leaf order wins, which is the primitive BVHNode::hit
// (src/bvh.hpp:31-37) returns, since it visits leaves left to right and
// accepts t <= t_max. Children are visited nearest first; the box test is
// AABB::hit's arithmetic. Split into steps so that a persistent kernel can
// give a lane a new ray as soon as its old one finishes.
template <int kShared, bool COUNT>
struct ClosestTrav {
    Ray ray;
    RayPre rp;
    float tmin, t_best;
    int best, best_ref;
    int node, sp;

    __device__ __forceinline__ void test_leaf(const SceneView& S, int ref, TravCount* cnt) {
        float t;
        if (COUNT) { cnt->prims++; cnt->leaf_bytes += leaf_bytes(ref); }
        if (hit_leaf<false>(S, ref, ray, tmin, t_best, t, nullptr)) {
            int slot = (~ref) & kLeafSlotMask;
            if (t < t_best || slot > best) { t_best = t; best = slot; best_ref = ref; }
        }
    }

    __device__ __forceinline__ bool init(const SceneView& S, const Ray& r, float tmin_,
                                         float tmax, TravCount* cnt) {
        ray = r;
        tmin = tmin_;
        t_best = tmax;
        best = -1;
        best_ref = 0;
        sp = 0;
        node = 0;
        if (S.root_ref == kEmptyRoot) return true;
        rp = prep(r);
        float e;
        if (!slab(S.root_min[0], S.root_min[1], S.root_min[2], S.root_max[0], S.root_max[1],
                  S.root_max[2], rp, tmin, tmax, e))
            return true;
        if (S.root_ref < 0) {
            test_leaf(S, S.root_ref, cnt);
            return true;
        }
        return false;
    }

    __device__ __forceinline__ bool step(const SceneView& S, TravStack<kShared>& stk,
                                         TravCount* cnt) {
        const float4* np = S.nodes + 4 * (size_t)node;
        float4 a = __ldg(np), b = __ldg(np + 1), c = __ldg(np + 2);
        int4 rr = __ldg(reinterpret_cast<const int4*>(np + 3));
        if (COUNT) cnt->nodes++;
        float eL, eR;
        bool hL = slab(a.x, a.y, a.z, a.w, b.x, b.y, rp, tmin, t_best, eL);
        bool hR = slab(b.z, b.w, c.x, c.y, c.z, c.w, rp, tmin, t_best, eR);
        if (hL && rr.x < 0) { test_leaf(S, rr.x, cnt); hL = false; }
        if (hR && rr.y < 0) { if (eR <= t_best) test_leaf(S, rr.y, cnt); hR = false; }
        hL = hL && eL <= t_best;
        hR = hR && eR <= t_best;
        if (hL && hR) {
            if (eR < eL) { stk.push(sp, rr.x, eL); node = rr.y; }
            else { stk.push(sp, rr.y, eR); node = rr.x; }
            ++sp;
            return false;
        }
        if (hL) { node = rr.x; return false; }
        if (hR) { node = rr.y; return false; }
        while (sp > 0) {
            --sp;
            int ref;
            float te;
            stk.pop(sp, ref, te);
            if (te <= t_best) { node = ref; return false; }
        }
        return true;
    }
};

// Resumable any-hit traversal (BVHNode::occluded, src/bvh.hpp:39-48). With a
// fixed t_max the box test is order independent, so the answer equals the
// reference's.
template <int kShared, bool COUNT>
struct AnyTrav {
    Ray ray;
    RayPre rp;
    float tmin, tmax;
    int node, sp;
    bool hit;

    __device__ __forceinline__ bool test_leaf(const SceneView& S, int ref, TravCount* cnt) {
        float t;
        if (COUNT) { cnt->prims++; cnt->leaf_bytes += leaf_bytes(ref); }
        return hit_leaf<false>(S, ref, ray, tmin, tmax, t, nullptr);
    }

    __device__ __forceinline__ bool init(const SceneView& S, const Ray& r, float tmin_,
                                         float tmax_, TravCount* cnt) {
        ray = r;
        tmin = tmin_;
        tmax = tmax_;
        hit = false;
        sp = 0;
        node = 0;
        if (S.root_ref == kEmptyRoot) return true;
        rp = prep(r);
        float e;
        if (!slab(S.root_min[0], S.root_min[1], S.root_min[2], S.root_max[0], S.root_max[1],
                  S.root_max[2], rp, tmin, tmax, e))
            return true;
        if (S.root_ref < 0) {
            hit = test_leaf(S, S.root_ref, cnt);
            return true;
        }
        return false;
    }

    __device__ __forceinline__ bool step(const SceneView& S, TravStack<kShared>& stk,
                                         TravCount* cnt) {
        const float4* np = S.nodes + 4 * (size_t)node;
        float4 a = __ldg(np), b = __ldg(np + 1), c = __ldg(np + 2);
        int4 rr = __ldg(reinterpret_cast<const int4*>(np + 3));
        if (COUNT) cnt->nodes++;
        float eL, eR;
        bool hL = slab(a.x, a.y, a.z, a.w, b.x, b.y, rp, tmin, tmax, eL);
        bool hR = slab(b.z, b.w, c.x, c.y, c.z, c.w, rp, tmin, tmax, eR);
        if (hL && rr.x < 0) {
            if (test_leaf(S, rr.x, cnt)) { hit = true; return true; }
            hL = false;
        }
        if (hR && rr.y < 0) {
            if (test_leaf(S, rr.y, cnt)) { hit = true; return true; }
            hR = false;
        }
        if (hL && hR) {
            if (eR < eL) { stk.push_ref(sp, rr.x); node = rr.y; }
            else { stk.push_ref(sp, rr.y); node = rr.x; }
            ++sp;
            return false;
        }
        if (hL) { node = rr.x; return false; }
        if (hR) { node = rr.y; return false; }
        if (sp == 0) return true;
        --sp;
        node = stk.pop_ref(sp);
        return false;
    }
};

// ---- wide traversal (both engines) ---------------------------------------------
// One wide node as one ray sees it: its children's near and far planes per
// axis (rows of four, SoA float4) and refs. A node stores the lo planes of
// x, y, z, then the hi planes; the ray's octant picks which are near, so the
// loads, not per-child selects, put the planes in slab order.
// A 4-wide node is held whole (six plane rows and the refs); an 8-wide node
// keeps its refs and its address, and its plane rows are loaded a group of
// four children at a time by slab_wide (a whole 8-wide node would take 56
// registers).
struct WideNode {
    float4 nr[3][1], fr[3][1];   // 4-wide: the plane rows (unused when 8-wide)
    const float4* np;
    int4 ref[kWideGroups];
};
__device__ __forceinline__ WideNode load_wide(const float4* wide, int node, const RayPre& r) {
    const float4* np = wide + (size_t)kWideNodeFloat4 * node;
    constexpr int G = kWideGroups;
    WideNode w;
    w.np = np;
    if constexpr (kWideWidth == 4) {
        w.nr[0][0] = __ldg(np + r.ox);
        w.fr[0][0] = __ldg(np + 3 - r.ox);
        w.nr[1][0] = __ldg(np + 1 + r.oy);
        w.fr[1][0] = __ldg(np + 4 - r.oy);
        w.nr[2][0] = __ldg(np + 2 + r.oz);
        w.fr[2][0] = __ldg(np + 5 - r.oz);
    }
#pragma unroll
    for (int g = 0; g < G; ++g) w.ref[g] = __ldg(reinterpret_cast<const int4*>(np + 6 * G + g));
    return w;
}

// AABB::hit with the near and far planes already chosen (the same
// arithmetic as slab).
__device__ __forceinline__ bool slab_nf(float nx, float ny, float nz, float fx, float fy,
                                        float fz, const RayPre& r, float tmin, float tmax,
                                        float& entry) {
    const float t0x = (nx - r.o.x) * r.inv.x;
    const float t1x = (fx - r.o.x) * r.inv.x;
    const float t0y = (ny - r.o.y) * r.inv.y;
    const float t1y = (fy - r.o.y) * r.inv.y;
    const float t0z = (nz - r.o.z) * r.inv.z;
    const float t1z = (fz - r.o.z) * r.inv.z;
    const float en = fmax3f(fmaxf(tmin, t0x), t0y, t0z);
    const float ex = fmin3f(fminf(tmax, t1x), t1y, t1z);
    entry = en;
    return !(ex < en);
}

__device__ __forceinline__ float f4c(const float4& v, int c) {
    return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w;
}
__device__ __forceinline__ int i4c(const int4& v, int c) {
    return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w;
}

// Slab tests of every child: bit k of the result is child k's hit, e[k] its
// entry distance.
__device__ __forceinline__ unsigned slab_wide(const WideNode& w, const RayPre& r, float tmin,
                                              float tmax, float (&e)[kWideWidth]) {
    unsigned m = 0;
    if constexpr (kWideWidth == 4) {
        m |= slab_nf(w.nr[0][0].x, w.nr[1][0].x, w.nr[2][0].x, w.fr[0][0].x, w.fr[1][0].x,
                     w.fr[2][0].x, r, tmin, tmax, e[0]) ? 1u : 0u;
        m |= slab_nf(w.nr[0][0].y, w.nr[1][0].y, w.nr[2][0].y, w.fr[0][0].y, w.fr[1][0].y,
                     w.fr[2][0].y, r, tmin, tmax, e[1]) ? 2u : 0u;
        m |= slab_nf(w.nr[0][0].z, w.nr[1][0].z, w.nr[2][0].z, w.fr[0][0].z, w.fr[1][0].z,
                     w.fr[2][0].z, r, tmin, tmax, e[2]) ? 4u : 0u;
        m |= slab_nf(w.nr[0][0].w, w.nr[1][0].w, w.nr[2][0].w, w.fr[0][0].w, w.fr[1][0].w,
                     w.fr[2][0].w, r, tmin, tmax, e[3]) ? 8u : 0u;
        return m;
    }
    else {
        constexpr int G = kWideGroups;
#pragma unroll
        for (int g = 0; g < G; ++g) {
            const float4 n0 = __ldg(w.np + r.ox * G + g), f0 = __ldg(w.np + (3 - r.ox) * G + g);
            const float4 n1 = __ldg(w.np + (1 + r.oy) * G + g);
            const float4 f1 = __ldg(w.np + (4 - r.oy) * G + g);
            const float4 n2 = __ldg(w.np + (2 + r.oz) * G + g);
            const float4 f2 = __ldg(w.np + (5 - r.oz) * G + g);
#pragma unroll
            for (int c = 0; c < 4; ++c)
                m |= slab_nf(f4c(n0, c), f4c(n1, c), f4c(n2, c), f4c(f0, c), f4c(f1, c),
                             f4c(f2, c), r, tmin, tmax, e[4 * g + c]) ? (1u << (4 * g + c)) : 0u;
        }
        return m;
    }
}

// Child k's ref / entry distance by a select chain (no local-memory indexing).
__device__ __forceinline__ int pick_ref(const WideNode& w, int k) {
    if constexpr (kWideWidth == 4) {
        const int4& r = w.ref[0];
        return k == 0 ? r.x : k == 1 ? r.y : k == 2 ? r.z : r.w;
    }
    int v = w.ref[0].x;
#pragma unroll
    for (int j = 1; j < kWideWidth; ++j) v = k == j ? i4c(w.ref[j >> 2], j & 3) : v;
    return v;
}
__device__ __forceinline__ float pick_e(const float (&e)[kWideWidth], int k) {
    if constexpr (kWideWidth == 4) return k == 0 ? e[0] : k == 1 ? e[1] : k == 2 ? e[2] : e[3];
    float v = e[0];
#pragma unroll
    for (int j = 1; j < kWideWidth; ++j) v = k == j ? e[j] : v;
    return v;
}
// Children of a wide node whose ref is a leaf, as bits.
__device__ __forceinline__ unsigned leaf_bits(const WideNode& w) {
    if constexpr (kWideWidth == 4) {
        const int4& r = w.ref[0];
        return (r.x < 0 ? 1u : 0u) | (r.y < 0 ? 2u : 0u) | (r.z < 0 ? 4u : 0u) |
               (r.w < 0 ? 8u : 0u);
    }
    unsigned m = 0;
#pragma unroll
    for (int k = 0; k < kWideWidth; ++k) m |= i4c(w.ref[k >> 2], k & 3) < 0 ? (1u << k) : 0u;
    return m;
}

// Sorts four (key, ref) pairs by key, ascending (a five-exchange network).
__device__ __forceinline__ void sort4(float& k0, int& r0, float& k1, int& r1, float& k2, int& r2,
                                      float& k3, int& r3) {
    auto cs = [](float& ka, int& ra, float& kb, int& rb) {
        const bool sw = kb < ka;
        const float tk = ka;
        const int tr = ra;
        ka = sw ? kb : ka;
        ra = sw ? rb : ra;
        kb = sw ? tk : kb;
        rb = sw ? tr : rb;
    };
    cs(k0, r0, k1, r1);
    cs(k2, r2, k3, r3);
    cs(k0, r0, k2, r2);
    cs(k1, r1, k3, r3);
    cs(k1, r1, k2, r2);
}

// The interior children of mask `im` with entries e: all but the nearest
// stacked, farthest first (so they pop nearest first); returns the nearest.
// 4-wide nodes sort their four keys with a network; 8-wide nodes take the
// farthest remaining child at each push.
template <int kShared>
__device__ __forceinline__ int push_children(const WideNode& w, unsigned im,
                                             const float (&e)[kWideWidth],
                                             TravStack<kShared>& stk, int& sp, bool keyed) {
    if constexpr (kWideWidth == 4) {
        float k0 = (im & 1u) ? e[0] : INFINITY;
        float k1 = (im & 2u) ? e[1] : INFINITY;
        float k2 = (im & 4u) ? e[2] : INFINITY;
        float k3 = (im & 8u) ? e[3] : INFINITY;
        int r0 = w.ref[0].x, r1 = w.ref[0].y, r2 = w.ref[0].z, r3 = w.ref[0].w;
        sort4(k0, r0, k1, r1, k2, r2, k3, r3);
        if (keyed) {
            if (k3 != INFINITY) stk.push(sp++, r3, k3);
            if (k2 != INFINITY) stk.push(sp++, r2, k2);
            if (k1 != INFINITY) stk.push(sp++, r1, k1);
        } else {
            if (k3 != INFINITY) stk.push_ref(sp++, r3);
            if (k2 != INFINITY) stk.push_ref(sp++, r2);
            if (k1 != INFINITY) stk.push_ref(sp++, r1);
        }
        return r0;
    } else if (!keyed) {
        // any hit: the nearest child next, the others in child order
        int kn = __ffs(im) - 1;
        float en = INFINITY;
#pragma unroll
        for (int k = 0; k < kWideWidth; ++k)
            if (((im >> k) & 1u) && e[k] < en) { en = e[k]; kn = k; }
        im &= ~(1u << kn);
        while (im) {
            const int k = 31 - __clz(im);
            im &= ~(1u << k);
            stk.push_ref(sp++, pick_ref(w, k));
        }
        return pick_ref(w, kn);
    } else {
        while (__popc(im) > 1) {
            int kf = 0;
            float ef = -INFINITY;
#pragma unroll
            for (int k = 0; k < kWideWidth; ++k)
                if (((im >> k) & 1u) && e[k] >= ef) { ef = e[k]; kf = k; }
            stk.push(sp++, pick_ref(w, kf), keyed ? ef : 0.0f);
            im &= ~(1u << kf);
        }
        return pick_ref(w, __ffs(im) - 1);
    }
}

// Resumable closest-hit traversal of the wide tree. Same result rule as
// ClosestTrav (smallest t, ties to the later DFS leaf); children are taken
// nearest first, the others stacked with their entry distance.
template <int kShared, bool COUNT>
struct ClosestTrav4 {
    Ray ray;
    RayPre rp;
    float tmin, t_best;
    int best, best_ref;
    int node, sp;

    __device__ __forceinline__ void test_leaf(const SceneView& S, int ref, TravCount* cnt) {
        float t;
        if (COUNT) { cnt->prims++; cnt->leaf_bytes += leaf_bytes(ref); }
        if (hit_leaf<false>(S, ref, ray, tmin, t_best, t, nullptr)) {
            int slot = (~ref) & kLeafSlotMask;
            if (t < t_best || slot > best) { t_best = t; best = slot; best_ref = ref; }
        }
    }

    __device__ __forceinline__ bool init(const SceneView& S, const Ray& r, float tmin_,
                                         float tmax, TravCount* cnt) {
        ray = r;
        tmin = tmin_;
        t_best = tmax;
        best = -1;
        best_ref = 0;
        sp = 0;
        node = 0;
        if (S.root_ref == kEmptyRoot) return true;
        rp = prep(r);
        float e;
        if (!slab(S.root_min[0], S.root_min[1], S.root_min[2], S.root_max[0], S.root_max[1],
                  S.root_max[2], rp, tmin, tmax, e))
            return true;
        if (S.root_ref < 0) {
            test_leaf(S, S.root_ref, cnt);
            return true;
        }
        return false;
    }

    __device__ __forceinline__ bool step(const SceneView& S, TravStack<kShared>& stk,
                                         TravCount* cnt) {
        const WideNode w = load_wide(S.wide, node, rp);
        if (COUNT) cnt->nodes++;
        float e[kWideWidth];
        unsigned m = slab_wide(w, rp, tmin, t_best, e);
        unsigned lm = m & leaf_bits(w);
        m &= ~lm;
        while (lm) {
            const int k = __ffs(lm) - 1;
            lm &= lm - 1;
            if (pick_e(e, k) <= t_best) test_leaf(S, pick_ref(w, k), cnt);
        }
        // interior children still in reach, nearest first
        unsigned im = 0;
#pragma unroll
        for (int k = 0; k < kWideWidth; ++k)
            if (((m >> k) & 1u) && e[k] <= t_best) im |= 1u << k;
        if (im) {
            node = push_children(w, im, e, stk, sp, true);
            return false;
        }
        while (sp > 0) {
            --sp;
            int ref;
            float te;
            stk.pop(sp, ref, te);
            if (te <= t_best) { node = ref; return false; }
        }
        return true;
    }
};

// Resumable any-hit traversal of the wide tree (BVHNode::occluded,
// src/bvh.hpp:39-48): with a fixed t_max the set of boxes entered does not
// depend on the order, so the answer equals the reference's whatever order
// the children are taken in.
template <int kShared, bool COUNT>
struct AnyTrav4 {
    Ray ray;
    RayPre rp;
    float tmin, tmax;
    int node, sp;
    bool hit;

    __device__ __forceinline__ bool test_leaf(const SceneView& S, int ref, TravCount* cnt) {
        float t;
        if (COUNT) { cnt->prims++; cnt->leaf_bytes += leaf_bytes(ref); }
        return hit_leaf<false>(S, ref, ray, tmin, tmax, t, nullptr);
    }

    __device__ __forceinline__ bool init(const SceneView& S, const Ray& r, float tmin_,
                                         float tmax_, TravCount* cnt) {
        ray = r;
        tmin = tmin_;
        tmax = tmax_;
        hit = false;
        sp = 0;
        node = 0;
        if (S.root_ref == kEmptyRoot) return true;
        rp = prep(r);
        float e;
        if (!slab(S.root_min[0], S.root_min[1], S.root_min[2], S.root_max[0], S.root_max[1],
                  S.root_max[2], rp, tmin, tmax, e))
            return true;
        if (S.root_ref < 0) {
            hit = test_leaf(S, S.root_ref, cnt);
            return true;
        }
        return false;
    }

    __device__ __forceinline__ bool step(const SceneView& S, TravStack<kShared>& stk,
                                         TravCount* cnt) {
        const WideNode w = load_wide(S.wide, node, rp);
        if (COUNT) cnt->nodes++;
        float e[kWideWidth];
        unsigned m = slab_wide(w, rp, tmin, tmax, e);
        unsigned lm = m & leaf_bits(w);
        m &= ~lm;
        while (lm) {
            const int k = __ffs(lm) - 1;
            lm &= lm - 1;
            if (test_leaf(S, pick_ref(w, k), cnt)) { hit = true; return true; }
        }
        if (m) {
            // nearest child first, the others stacked so that the nearer pop
            // first: an occluder near the ray's origin ends the walk early
            node = push_children(w, m, e, stk, sp, false);
            return false;
        }
        if (sp == 0) return true;
        --sp;
        node = stk.pop_ref(sp);
        return false;
    }
};

// Closest hit of one ray, traced to the end in one loop (megakernel,
// queries): the same traversal as ClosestTrav, written as a single loop,
// which compiles to fewer registers inside the megakernel. Returns the leaf
// slot or -1.
template <int kShared, bool COUNT>
__device__ int closest_hit(const SceneView& S, const Ray& ray, float tmin, float tmax,
                           float& t_best, int& best_ref, TravStack<kShared>& stk,
                           TravCount* cnt) {
    t_best = tmax;
    best_ref = 0;
    int best = -1;
    if (S.root_ref == kEmptyRoot) return -1;
    RayPre rp = prep(ray);
    float e;
    if (!slab(S.root_min[0], S.root_min[1], S.root_min[2], S.root_max[0], S.root_max[1],
              S.root_max[2], rp, tmin, tmax, e))
        return -1;
    auto test_leaf = [&](int ref) {
        float t;
        if (COUNT) { cnt->prims++; cnt->leaf_bytes += leaf_bytes(ref); }
        if (hit_leaf<false>(S, ref, ray, tmin, t_best, t, nullptr)) {
            int slot = (~ref) & kLeafSlotMask;
            if (t < t_best || slot > best) { t_best = t; best = slot; best_ref = ref; }
        }
    };
    if (S.root_ref < 0) {
        test_leaf(S.root_ref);
        return best;
    }
    int node = 0;
    int sp = 0;
    while (true) {
        const float4* np = S.nodes + 4 * (size_t)node;
        float4 a = __ldg(np), b = __ldg(np + 1), c = __ldg(np + 2);
        int4 rr = __ldg(reinterpret_cast<const int4*>(np + 3));
        if (COUNT) cnt->nodes++;
        float eL, eR;
        bool hL = slab(a.x, a.y, a.z, a.w, b.x, b.y, rp, tmin, t_best, eL);
        bool hR = slab(b.z, b.w, c.x, c.y, c.z, c.w, rp, tmin, t_best, eR);
        if (hL && rr.x < 0) { test_leaf(rr.x); hL = false; }
        if (hR && rr.y < 0) { if (eR <= t_best) test_leaf(rr.y); hR = false; }
        hL = hL && eL <= t_best;
        hR = hR && eR <= t_best;
        if (hL && hR) {
            if (eR < eL) { stk.push(sp, rr.x, eL); node = rr.y; }
            else { stk.push(sp, rr.y, eR); node = rr.x; }
            ++sp;
        } else if (hL) {
            node = rr.x;
        } else if (hR) {
            node = rr.y;
        } else {
            bool found = false;
            while (sp > 0) {
                --sp;
                int ref;
                float te;
                stk.pop(sp, ref, te);
                if (te <= t_best) { node = ref; found = true; break; }
            }
            if (!found) break;
        }
    }
    return best;
}

// Any hit of one ray in [tmin, tmax], traced to the end in one loop.
template <int kShared, bool COUNT>
__device__ bool any_hit(const SceneView& S, const Ray& ray, float tmin, float tmax,
                        TravStack<kShared>& stk, TravCount* cnt) {
    if (S.root_ref == kEmptyRoot) return false;
    RayPre rp = prep(ray);
    float e;
    if (!slab(S.root_min[0], S.root_min[1], S.root_min[2], S.root_max[0], S.root_max[1],
              S.root_max[2], rp, tmin, tmax, e))
        return false;
    auto test_leaf = [&](int ref) -> bool {
        float t;
        if (COUNT) { cnt->prims++; cnt->leaf_bytes += leaf_bytes(ref); }
        return hit_leaf<false>(S, ref, ray, tmin, tmax, t, nullptr);
    };
    if (S.root_ref < 0) return test_leaf(S.root_ref);
    int node = 0;
    int sp = 0;
    while (true) {
        const float4* np = S.nodes + 4 * (size_t)node;
        float4 a = __ldg(np), b = __ldg(np + 1), c = __ldg(np + 2);
        int4 rr = __ldg(reinterpret_cast<const int4*>(np + 3));
        if (COUNT) cnt->nodes++;
        float eL, eR;
        bool hL = slab(a.x, a.y, a.z, a.w, b.x, b.y, rp, tmin, tmax, eL);
        bool hR = slab(b.z, b.w, c.x, c.y, c.z, c.w, rp, tmin, tmax, eR);
        if (hL && rr.x < 0) { if (test_leaf(rr.x)) return true; hL = false; }
        if (hR && rr.y < 0) { if (test_leaf(rr.y)) return true; hR = false; }
        if (hL && hR) {
            if (eR < eL) { stk.push_ref(sp, rr.x); node = rr.y; }
            else { stk.push_ref(sp, rr.y); node = rr.x; }
            ++sp;
        } else if (hL) {
            node = rr.x;
        } else if (hR) {
            node = rr.y;
        } else {
            if (sp == 0) return false;
            --sp;
            node = stk.pop_ref(sp);
        }
    }
}

// Closest hit / any hit of one ray on the 4-wide tree, traced to the end
// (megakernel): the wavefront's resumable traversals run in one loop, so
// both engines walk the same tree in the same order.
template <int kShared, bool COUNT>
__device__ __forceinline__ int closest_hit4(const SceneView& S, const Ray& ray, float tmin,
                                            float tmax, float& t_best, int& best_ref,
                                            TravStack<kShared>& stk, TravCount* cnt) {
    ClosestTrav4<kShared, COUNT> tr;
    if (!tr.init(S, ray, tmin, tmax, cnt))
        while (!tr.step(S, stk, cnt)) {
        }
    t_best = tr.t_best;
    best_ref = tr.best_ref;
    return tr.best;
}
template <int kShared, bool COUNT>
__device__ __forceinline__ bool any_hit4(const SceneView& S, const Ray& ray, float tmin,
                                         float tmax, TravStack<kShared>& stk, TravCount* cnt) {
    AnyTrav4<kShared, COUNT> tr;
    if (!tr.init(S, ray, tmin, tmax, cnt))
        while (!tr.step(S, stk, cnt)) {
        }
    return tr.hit;
}

// Full hit record of the closest hit found by closest_hit.
// A sphere's or a triangle's record depends on the hit only through t: the
// point is ray.at(t) and the normal follows from it (sphere) or is the
// face's own (triangle), as Sphere::hit / Triangle::hit make them
// (src/primitives.hpp:98-120, 145-170); the other primitives test again.
__device__ __forceinline__ void make_hit(const SceneView& S, int best_ref, int slot,
                                         const Ray& ray, float tmin, float t_best, Hit& h) {
    const int code = ~best_ref;
    const int type = code >> kLeafTypeShift;
    const int s = code & kLeafSlotMask;
    if (type == LEAF_SPHERE) {
        const float4 g = __ldg(S.geo_a + s);
        h.t = t_best;
        h.p = ray.o + ray.d * t_best;
        set_face(h, ray, (h.p - v3(g.x, g.y, g.z)) / g.w);
    } else if (type == LEAF_TRIANGLE) {
        // the face normal, normalized(e1 x e2), stored by the upload in the
        // w words of the slot
        const float nx = __ldg(&S.geo_a[s].w), ny = __ldg(&S.geo_b[s].w), nz = __ldg(&S.geo_c[s].w);
        h.t = t_best;
        h.p = ray.o + ray.d * t_best;
        set_face(h, ray, v3(nx, ny, nz));
    } else {
        float t;
        hit_leaf<true>(S, best_ref, ray, tmin, t_best, t, &h);
    }
    h.mat = __ldg(S.leaf_mat + slot);
}

}  // namespace pgpu
