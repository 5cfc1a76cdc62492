/*
 * oracle.c - CPU restatement of Pencil's per-pixel path-tracing loop.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product): see oracle.h
 * for the list of reference functions restated here and their file:line.
 * Every expression keeps the reference's float32 operation order so that,
 * built with -ffp-contract=off, results match the reference bit for bit.
 */
#include "oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ---- Vec3 (src/vec3.hpp:24-92) ------------------------------------------ */
typedef struct { float x, y, z; } v3;

static inline v3 mk(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 neg(v3 a) { return mk(-a.x, -a.y, -a.z); }
static inline v3 mulf(v3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
static inline v3 divf(v3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }
static inline v3 mulv(v3 a, v3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross(v3 a, v3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float len(v3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
static inline v3 nrm(v3 a) {
    float l = len(a);
    return (l > 1e-12f) ? divf(a, l) : mk(0.0f, 0.0f, 0.0f);
}
static inline v3 reflect(v3 v, v3 n) { return sub(v, mulf(n, 2.0f * dot(v, n))); }
static inline float comp(v3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
static inline v3 ld3(const float* p) { return mk(p[0], p[1], p[2]); }
static inline float clampf(float v, float lo, float hi) {
    return (v < lo) ? lo : (v > hi) ? hi : v;
}
static inline float schlick(float c, float ratio) {
    float r0 = (1.0f - ratio) / (1.0f + ratio);
    r0 = r0 * r0;
    return r0 + (1.0f - r0) * powf(1.0f - c, 5.0f);
}

/* ---- Rng (src/rng.hpp:13-45) --------------------------------------------- */
typedef struct { uint32_t s; } rng_t;
static inline uint32_t rng_u32(rng_t* r) {
    r->s ^= r->s << 13u;
    r->s ^= r->s >> 17u;
    r->s ^= r->s << 5u;
    return r->s;
}
static inline float rng_unit(rng_t* r) { return (float)rng_u32(r) / 4294967296.0f; }
static inline float rng_sym(rng_t* r) { return rng_unit(r) * 2.0f - 1.0f; }
static inline void rng_disc(rng_t* r, float* dx, float* dy) {
    float r1 = rng_unit(r);
    float r2 = rng_unit(r);
    float sx = 2.0f * r1 - 1.0f;
    float sy = 2.0f * r2 - 1.0f;
    if (sx == 0.0f && sy == 0.0f) { *dx = 0; *dy = 0; return; }
    float theta, rad;
    if (fabsf(sx) > fabsf(sy)) {
        rad = sx;
        theta = (3.14159265f / 4.0f) * (sy / sx);
    } else {
        rad = sy;
        theta = (3.14159265f / 2.0f) - (3.14159265f / 4.0f) * (sx / sy);
    }
    *dx = rad * cosf(theta);
    *dy = rad * sinf(theta);
}

static uint32_t mix32(uint32_t x) {
    x ^= x >> 16; x *= 0x7feb352dU;
    x ^= x >> 15; x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

uint32_t orc_path_seed(int32_t i, int32_t j, int32_t sample, uint32_t salt) {
    uint32_t pix = (uint32_t)i * 97861u + (uint32_t)j * 1973u + 1u;
    uint32_t s = mix32(pix ^ mix32((uint32_t)sample * 0x9E3779B9u + salt + 0x632BE5ABu));
    return s ? s : 0x6D2B79F5u;
}

/* ---- hit record (src/primitives.hpp:70-81) ------------------------------- */
typedef struct {
    v3 p, n;
    float t;
    int mat;
    int front;
    int prim;
} hitrec;

typedef struct { v3 o, d; } ray_t;
static inline v3 ray_at(ray_t r, float t) { return add(r.o, mulf(r.d, t)); }
static inline void set_face(hitrec* h, ray_t r, v3 outward) {
    h->front = dot(r.d, outward) < 0.0f;
    h->n = h->front ? outward : neg(outward);
}

/* ---- primitives ---------------------------------------------------------- */
static int hit_sphere(const pgpu_prim* pr, ray_t r, float tmin, float tmax, hitrec* h) {
    v3 c = ld3(pr->p);
    float rad = pr->p[3];
    v3 oc = sub(r.o, c);
    float a = dot(r.d, r.d);
    float hb = dot(oc, r.d);
    float cc = dot(oc, oc) - rad * rad;
    float disc = hb * hb - a * cc;
    if (disc < 0.0f) return 0;
    float sq = sqrtf(disc);
    float t = (-hb - sq) / a;
    if (t < tmin || t > tmax) {
        t = (-hb + sq) / a;
        if (t < tmin || t > tmax) return 0;
    }
    h->t = t;
    h->p = ray_at(r, t);
    set_face(h, r, divf(sub(h->p, c), rad));
    h->mat = pr->material;
    return 1;
}

static int hit_triangle(const pgpu_prim* pr, ray_t r, float tmin, float tmax, hitrec* h) {
    v3 v0 = ld3(pr->p), v1 = ld3(pr->p + 3), v2 = ld3(pr->p + 6);
    v3 e1 = sub(v1, v0), e2 = sub(v2, v0);
    v3 hh = cross(r.d, e2);
    float a = dot(e1, hh);
    if (fabsf(a) < 1e-8f) return 0;
    float f = 1.0f / a;
    v3 s = sub(r.o, v0);
    float u = f * dot(s, hh);
    if (u < 0.0f || u > 1.0f) return 0;
    v3 q = cross(s, e1);
    float v = f * dot(r.d, q);
    if (v < 0.0f || u + v > 1.0f) return 0;
    float t = f * dot(e2, q);
    if (t < tmin || t > tmax) return 0;
    h->t = t;
    h->p = ray_at(r, t);
    set_face(h, r, nrm(cross(e1, e2)));
    h->mat = pr->material;
    return 1;
}

static int hit_cube(const pgpu_prim* pr, ray_t r, float tmin, float tmax, hitrec* h) {
    v3 c = ld3(pr->p);
    float hf = pr->p[3];
    v3 lo = sub(c, mk(hf, hf, hf));
    v3 hi = add(c, mk(hf, hf, hf));
    float t_near = -INFINITY, t_far = INFINITY;
    int near_axis = -1, far_axis = -1;
    float near_sign = 1.0f, far_sign = -1.0f;
    for (int a = 0; a < 3; ++a) {
        const float d = comp(r.d, a);
        const float o = comp(r.o, a);
        if (fabsf(d) < 1e-12f) {
            if (o < comp(lo, a) || o > comp(hi, a)) return 0;
            continue;
        }
        float tn = (comp(lo, a) - o) / d;
        float tf = (comp(hi, a) - o) / d;
        float ns = -1.0f, fs = 1.0f;
        if (tn > tf) { float x = tn; tn = tf; tf = x; x = ns; ns = fs; fs = x; }
        if (tn > t_near) { t_near = tn; near_axis = a; near_sign = ns; }
        if (tf < t_far) { t_far = tf; far_axis = a; far_sign = fs; }
        if (t_far < t_near) return 0;
    }
    const int use_near = t_near >= tmin;
    const float th = use_near ? t_near : t_far;
    const int ax = use_near ? near_axis : far_axis;
    const float sg = use_near ? near_sign : far_sign;
    if (ax < 0 || th < tmin || th > tmax) return 0;
    h->t = th;
    h->p = ray_at(r, th);
    v3 n = mk(0.0f, 0.0f, 0.0f);
    if (ax == 0) n.x = sg; else if (ax == 1) n.y = sg; else n.z = sg;
    set_face(h, r, n);
    h->mat = pr->material;
    return 1;
}

static int hit_plane(const pgpu_prim* pr, ray_t r, float tmin, float tmax, hitrec* h) {
    v3 pt = ld3(pr->p), n = ld3(pr->p + 3);
    float denom = dot(n, r.d);
    if (fabsf(denom) < 1e-6f) return 0;
    float t = dot(sub(pt, r.o), n) / denom;
    if (t < tmin || t > tmax) return 0;
    h->t = t;
    h->p = ray_at(r, t);
    set_face(h, r, n);
    h->mat = pr->material;
    return 1;
}

static int cyl_side(const pgpu_prim* pr, ray_t r, float tmin, float tmax, hitrec* h) {
    v3 c = ld3(pr->p), ax = ld3(pr->p + 3);
    float rad = pr->p[6], hh = pr->p[7];
    v3 oc = sub(r.o, c);
    float dda = dot(r.d, ax);
    float oca = dot(oc, ax);
    v3 dp = sub(r.d, mulf(ax, dda));
    v3 op = sub(oc, mulf(ax, oca));
    float a = dot(dp, dp);
    float b = 2.0f * dot(op, dp);
    float cc = dot(op, op) - rad * rad;
    if (a < 1e-9f) {
        if (fabsf(b) < 1e-9f) return 0;
        const float t = -cc / b;
        if (t < tmin || t > tmax) return 0;
        const float hgt = oca + t * dda;
        if (fabsf(hgt) > hh) return 0;
        h->t = t;
        h->p = ray_at(r, t);
        v3 apt = add(c, mulf(ax, hgt));
        set_face(h, r, divf(sub(h->p, apt), rad));
        h->mat = pr->material;
        return 1;
    }
    float disc = b * b - 4.0f * a * cc;
    if (disc < 0.0f) return 0;
    float sq = sqrtf(disc);
    float ts[2];
    ts[0] = (-b - sq) / (2.0f * a);
    ts[1] = (-b + sq) / (2.0f * a);
    for (int k = 0; k < 2; ++k) {
        float t = ts[k];
        if (t < tmin || t > tmax) continue;
        float hgt = (oca + t * dda);
        if (fabsf(hgt) > hh) continue;
        h->t = t;
        h->p = ray_at(r, t);
        v3 apt = add(c, mulf(ax, hgt));
        set_face(h, r, divf(sub(h->p, apt), rad));
        h->mat = pr->material;
        return 1;
    }
    return 0;
}

static int disc_cap(v3 center, v3 n, float rad, int mat, ray_t r, float tmin, float tmax, hitrec* h) {
    float denom = dot(n, r.d);
    if (fabsf(denom) < 1e-6f) return 0;
    float t = dot(sub(center, r.o), n) / denom;
    if (t < tmin || t > tmax) return 0;
    v3 p = ray_at(r, t);
    v3 d = sub(p, center);
    if (dot(d, d) > rad * rad) return 0;
    h->t = t;
    h->p = p;
    set_face(h, r, n);
    h->mat = mat;
    return 1;
}

static int hit_cylinder(const pgpu_prim* pr, ray_t r, float tmin, float tmax, hitrec* h) {
    v3 c = ld3(pr->p), ax = ld3(pr->p + 3);
    float rad = pr->p[6], hh = pr->p[7];
    int found = 0;
    float closest = tmax;
    hitrec best;
    if (cyl_side(pr, r, tmin, closest, &best)) { closest = best.t; *h = best; found = 1; }
    if (disc_cap(add(c, mulf(ax, 1.0f * hh)), mulf(ax, 1.0f), rad, pr->material, r, tmin, closest, &best)) {
        closest = best.t; *h = best; found = 1;
    }
    if (disc_cap(add(c, mulf(ax, -1.0f * hh)), mulf(ax, -1.0f), rad, pr->material, r, tmin, closest, &best)) {
        closest = best.t; *h = best; found = 1;
    }
    return found;
}

static int cone_side(const pgpu_prim* pr, ray_t r, float tmin, float tmax, hitrec* h) {
    v3 apex = ld3(pr->p), ax = ld3(pr->p + 3);
    float rad = pr->p[6], hgt = pr->p[7];
    v3 oc = sub(r.o, apex);
    float dda = dot(r.d, ax);
    float oca = dot(oc, ax);
    float k = rad / hgt;
    float k2 = k * k;
    v3 dp = sub(r.d, mulf(ax, dda));
    v3 op = sub(oc, mulf(ax, oca));
    float a = dot(dp, dp) - k2 * dda * dda;
    float b = 2.0f * (dot(dp, op) - k2 * dda * oca);
    float cc = dot(op, op) - k2 * oca * oca;
    float disc = b * b - 4.0f * a * cc;
    if (disc < 0.0f || fabsf(a) < 1e-12f) return 0;
    float sq = sqrtf(disc);
    float ts[2];
    ts[0] = (-b - sq) / (2.0f * a);
    ts[1] = (-b + sq) / (2.0f * a);
    for (int q = 0; q < 2; ++q) {
        float t = ts[q];
        if (t < tmin || t > tmax) continue;
        float hh = oca + t * dda;
        if (hh < 0.0f || hh > hgt) continue;
        h->t = t;
        h->p = ray_at(r, t);
        v3 apt = add(apex, mulf(ax, hh));
        v3 radial = sub(h->p, apt);
        set_face(h, r, nrm(sub(nrm(radial), mulf(ax, k))));
        h->mat = pr->material;
        return 1;
    }
    return 0;
}

static int hit_cone(const pgpu_prim* pr, ray_t r, float tmin, float tmax, hitrec* h) {
    v3 apex = ld3(pr->p), ax = ld3(pr->p + 3);
    float rad = pr->p[6], hgt = pr->p[7];
    v3 base = sub(apex, mulf(ax, hgt));
    int found = 0;
    float closest = tmax;
    hitrec best;
    if (cone_side(pr, r, tmin, closest, &best)) { closest = best.t; *h = best; found = 1; }
    if (disc_cap(base, neg(ax), rad, pr->material, r, tmin, closest, &best)) {
        closest = best.t; *h = best; found = 1;
    }
    return found;
}

static int hit_prim(const pgpu_prim* pr, ray_t r, float tmin, float tmax, hitrec* h) {
    switch (pr->type) {
        case PGPU_PRIM_SPHERE:   return hit_sphere(pr, r, tmin, tmax, h);
        case PGPU_PRIM_TRIANGLE: return hit_triangle(pr, r, tmin, tmax, h);
        case PGPU_PRIM_CUBE:     return hit_cube(pr, r, tmin, tmax, h);
        case PGPU_PRIM_PLANE:    return hit_plane(pr, r, tmin, tmax, h);
        case PGPU_PRIM_CYLINDER: return hit_cylinder(pr, r, tmin, tmax, h);
        case PGPU_PRIM_CONE:     return hit_cone(pr, r, tmin, tmax, h);
        default: return 0;
    }
}

/* Bytes of a primitive's record as the GPU tables hold it (counters only). */
static int prim_bytes(const pgpu_prim* pr) {
    switch (pr->type) {
        case PGPU_PRIM_SPHERE:   return 16;
        case PGPU_PRIM_TRIANGLE: return 36;
        case PGPU_PRIM_CUBE:     return 16;
        case PGPU_PRIM_PLANE:    return 24;
        default:                 return 32;
    }
}

/* ---- BVH (src/bvh.hpp:31-48, AABB::hit src/primitives.hpp:38-49) -------- */
static int box_hit(const pgpu_bvh_node* nd, ray_t r, float tmin, float tmax) {
    for (int a = 0; a < 3; ++a) {
        float inv = 1.0f / comp(r.d, a);
        float t0 = (nd->bmin[a] - comp(r.o, a)) * inv;
        float t1 = (nd->bmax[a] - comp(r.o, a)) * inv;
        if (inv < 0.0f) { float x = t0; t0 = t1; t1 = x; }
        tmin = (t0 > tmin) ? t0 : tmin;
        tmax = (t1 < tmax) ? t1 : tmax;
        if (tmax < tmin) return 0;
    }
    return 1;
}

typedef struct {
    const orc_scene* s;
    uint64_t* cnt;   /* may be NULL */
} trav_t;

static int node_hit(const trav_t* tv, int idx, ray_t r, float tmin, float tmax, hitrec* h) {
    const pgpu_bvh_node* nd = &tv->s->nodes[idx];
    if (tv->cnt) tv->cnt[ORC_CNT_NODE_VISITS]++;
    if (!box_hit(nd, r, tmin, tmax)) return 0;
    if (nd->left < 0) {
        if (tv->cnt) {
            tv->cnt[ORC_CNT_PRIM_TESTS]++;
            tv->cnt[ORC_CNT_PRIM_BYTES] += (uint64_t)prim_bytes(&tv->s->prims[nd->right]);
        }
        int ok = hit_prim(&tv->s->prims[nd->right], r, tmin, tmax, h);
        if (ok) h->prim = nd->right;
        return ok;
    }
    int hl = node_hit(tv, nd->left, r, tmin, tmax, h);
    int hr = node_hit(tv, nd->right, r, tmin, hl ? h->t : tmax, h);
    return hl || hr;
}

static int node_occ(const trav_t* tv, int idx, ray_t r, float tmin, float tmax) {
    const pgpu_bvh_node* nd = &tv->s->nodes[idx];
    if (tv->cnt) tv->cnt[ORC_CNT_NODE_VISITS]++;
    if (!box_hit(nd, r, tmin, tmax)) return 0;
    if (nd->left < 0) {
        hitrec tmp;
        if (tv->cnt) {
            tv->cnt[ORC_CNT_PRIM_TESTS]++;
            tv->cnt[ORC_CNT_PRIM_BYTES] += (uint64_t)prim_bytes(&tv->s->prims[nd->right]);
        }
        return hit_prim(&tv->s->prims[nd->right], r, tmin, tmax, &tmp);
    }
    if (node_occ(tv, nd->left, r, tmin, tmax)) return 1;
    if (node_occ(tv, nd->right, r, tmin, tmax)) return 1;
    return 0;
}

/* Scene::hit / Scene::occluded (src/scene.hpp:55-81), BVH branch. */
/* The work of one walk, added to the counters of its kind. */
static void split_counts(uint64_t* cnt, const uint64_t before[3], int nodes, int prims,
                         int bytes) {
    cnt[nodes] += cnt[ORC_CNT_NODE_VISITS] - before[0];
    cnt[prims] += cnt[ORC_CNT_PRIM_TESTS] - before[1];
    cnt[bytes] += cnt[ORC_CNT_PRIM_BYTES] - before[2];
}
static int scene_hit(const trav_t* tv, ray_t r, float tmin, float tmax, hitrec* h) {
    if (tv->cnt) tv->cnt[ORC_CNT_EXTENSION_RAYS]++;
    if (tv->s->n_nodes <= 0) return 0;
    if (!tv->cnt) return node_hit(tv, 0, r, tmin, tmax, h);
    const uint64_t before[3] = {tv->cnt[ORC_CNT_NODE_VISITS], tv->cnt[ORC_CNT_PRIM_TESTS],
                                tv->cnt[ORC_CNT_PRIM_BYTES]};
    int ok = node_hit(tv, 0, r, tmin, tmax, h);
    split_counts(tv->cnt, before, ORC_CNT_EXT_NODES, ORC_CNT_EXT_PRIMS, ORC_CNT_EXT_PRIM_BYTES);
    return ok;
}
static int scene_occ(const trav_t* tv, ray_t r, float tmin, float tmax) {
    if (tv->cnt) tv->cnt[ORC_CNT_SHADOW_RAYS]++;
    if (tv->s->n_nodes <= 0) return 0;
    if (!tv->cnt) return node_occ(tv, 0, r, tmin, tmax);
    const uint64_t before[3] = {tv->cnt[ORC_CNT_NODE_VISITS], tv->cnt[ORC_CNT_PRIM_TESTS],
                                tv->cnt[ORC_CNT_PRIM_BYTES]};
    int ok = node_occ(tv, 0, r, tmin, tmax);
    split_counts(tv->cnt, before, ORC_CNT_SH_NODES, ORC_CNT_SH_PRIMS, ORC_CNT_SH_PRIM_BYTES);
    return ok;
}

/* ---- camera (src/camera.hpp:67-86, src/camera.cpp:48-68) ---------------- */
void orc_camera_basis(const pgpu_camera* c, float out[21]) {
    v3 eye = ld3(c->eye), look = ld3(c->look), up = ld3(c->up);
    v3 w = nrm(sub(eye, look));
    v3 u = nrm(cross(up, w));
    v3 v = cross(w, u);
    float theta = c->vfov_deg * 3.14159265358979323846f / 180.0f;
    float half_h = tanf(theta * 0.5f);
    float half_w = c->aspect * half_h;
    v3 hor = mulf(u, 2.0f * half_w * c->focus_dist);
    v3 ver = mulf(v, 2.0f * half_h * c->focus_dist);
    v3 ll = sub(sub(sub(eye, mulf(hor, 0.5f)), mulf(ver, 0.5f)), mulf(w, c->focus_dist));
    v3 all[7] = {eye, ll, hor, ver, u, v, w};
    for (int k = 0; k < 7; ++k) {
        out[3 * k + 0] = all[k].x; out[3 * k + 1] = all[k].y; out[3 * k + 2] = all[k].z;
    }
}

static ray_t camera_ray(const orc_scene* s, float u, float v) {
    v3 org = ld3(s->cam), ll = ld3(s->cam + 3), hor = ld3(s->cam + 6), ver = ld3(s->cam + 9);
    v3 dir = sub(add(add(ll, mulf(hor, u)), mulf(ver, v)), org);
    ray_t r = {org, nrm(dir)};
    return r;
}

/* ---- shading ------------------------------------------------------------- */
typedef struct {
    const orc_scene* s;
    const pgpu_render_params* p;
    trav_t tv;
    uint64_t* cnt;
} ctx_t;

/* Light direction for one light at p (soft disc jitter included):
 * src/renderer.hpp:512-545 and 887-906 share this computation. */
static void light_dir(const pgpu_light* l, v3 p, rng_t* rng, v3* L, float* dist) {
    v3 lpos = ld3(l->pos);
    if (l->kind == PGPU_LIGHT_POINT && l->radius > 0.0f) {
        v3 to = sub(ld3(l->pos), p);
        v3 axis = nrm(to);
        v3 upv = (fabsf(axis.y) < 0.9f) ? mk(0, 1, 0) : mk(1, 0, 0);
        v3 t1 = nrm(cross(axis, upv));
        v3 t2 = nrm(cross(axis, t1));
        float dx, dy;
        rng_disc(rng, &dx, &dy);
        lpos = add(ld3(l->pos), mulf(add(mulf(t1, dx), mulf(t2, dy)), l->radius));
    }
    if (l->kind == PGPU_LIGHT_POINT) {
        v3 d = sub(lpos, p);
        *dist = len(d);
        *L = divf(d, *dist);
    } else {
        *L = neg(ld3(l->pos));
        *dist = 1e9f;
    }
}

static v3 whitted(ctx_t* c, ray_t r, int depth, rng_t* rng);

static v3 dielectric(ctx_t* c, ray_t r, const hitrec* rec, const pgpu_material* m,
                     v3 albedo, int depth, rng_t* rng) {
    float bias = c->p->shadow_bias;
    float ior = m->ior;
    int entering = rec->front;
    float safe = fmaxf(ior, 0.01f);
    float eta = entering ? (1.0f / safe) : safe;
    v3 nf = rec->n;
    float cos_i = fabsf(dot(nrm(r.d), rec->n));
    float sin_t2 = eta * eta * (1.0f - cos_i * cos_i);
    v3 rdir = nrm(reflect(nrm(r.d), rec->n));
    ray_t rr = {add(rec->p, mulf(rec->n, bias)), rdir};
    v3 rc = whitted(c, rr, depth - 1, rng);
    if (sin_t2 > 1.0f) return mulv(rc, albedo);
    float cos_t = sqrtf(1.0f - sin_t2);
    v3 tdir = nrm(add(mulf(nrm(r.d), eta), mulf(nf, eta * cos_i - cos_t)));
    ray_t tr = {sub(rec->p, mulf(nf, bias)), tdir};
    v3 tc = whitted(c, tr, depth - 1, rng);
    float cf = entering ? cos_i : cos_t;
    float kr = schlick(cf, eta);
    float kt = 1.0f - kr;
    v3 g = add(mulf(rc, kr), mulf(tc, kt));
    return mulv(g, albedo);
}

static v3 whitted(ctx_t* c, ray_t r, int depth, rng_t* rng) {
    const orc_scene* s = c->s;
    float bias = c->p->shadow_bias;
    if (c->cnt) c->cnt[ORC_CNT_REFERENCE_RAYS]++;
    if (depth <= 0) return mk(0, 0, 0);
    hitrec rec;
    if (!scene_hit(&c->tv, r, 1e-4f, 1e9f, &rec)) return ld3(s->background);
    const pgpu_material* m = &s->materials[rec.mat];
    v3 albedo = ld3(m->albedo);
    v3 sn = rec.n;
    v3 local = ld3(m->emission);
    for (int li = 0; li < s->n_lights; ++li) {
        const pgpu_light* l = &s->lights[li];
        if (l->kind == PGPU_LIGHT_QUAD) continue;
        v3 contrib = mk(0, 0, 0);
        int ns = (l->radius > 0.0f) ? c->p->soft_shadow_samples : 1;
        for (int k = 0; k < ns; ++k) {
            v3 L; float dist;
            light_dir(l, rec.p, rng, &L, &dist);
            ray_t sr = {add(rec.p, mulf(rec.n, bias)), L};
            if (!l->is_emissive && scene_occ(&c->tv, sr, bias, dist - bias)) continue;
            float ndotl = clampf(dot(sn, L), 0.0f, 1.0f);
            v3 col = mulf(mulv(albedo, ld3(l->intensity)), ndotl);
            if (m->specular > 0.0f && ndotl > 0.0f) {
                v3 V = neg(nrm(r.d));
                v3 H = nrm(add(L, V));
                float ndoth = clampf(dot(sn, H), 0.0f, 1.0f);
                float spec = powf(ndoth, m->shininess);
                col = add(col, mulf(mulv(ld3(m->specular_color), ld3(l->intensity)), spec * m->specular));
            }
            contrib = add(contrib, col);
        }
        local = add(local, divf(contrib, (float)ns));
    }
    local = add(local, mulv(albedo, ld3(s->ambient)));
    if (m->kind == PGPU_MAT_METAL && m->reflectivity > 0.0f) {
        v3 rd = nrm(reflect(nrm(r.d), rec.n));
        ray_t rr = {add(rec.p, mulf(rec.n, bias)), rd};
        v3 inc = whitted(c, rr, depth - 1, rng);
        v3 refl = mulf(mulv(inc, albedo), m->reflectivity);
        local = add(mulf(local, 1.0f - m->reflectivity), refl);
    } else if (m->kind == PGPU_MAT_DIELECTRIC) {
        local = dielectric(c, r, &rec, m, albedo, depth, rng);
    }
    return local;
}

/* Contribution of a visible point/directional light sample at a path-trace
 * vertex: trace_path (src/renderer.hpp:912-913) or, with PGPU_FLAG_MIS,
 * trace_path_mis (src/renderer.hpp:1264-1297): the power heuristic of the
 * light pdf (a disc light's, for a light facing down, cosine >= 0.01) and the
 * cosine BSDF pdf, mixing albedo*I*(n.L) and albedo*I; nothing when n.L <= 0. */
static v3 light_term(const pgpu_light* l, int mis, v3 T, v3 albedo, v3 L, float dist,
                     float ndotl) {
    if (!mis) return mulf(mulv(mulv(T, albedo), ld3(l->intensity)), ndotl);
    if (ndotl <= 0.0f) return mk(0, 0, 0);
    float pdf_brdf = ndotl / 3.14159265f;
    float pdf_light;
    if (l->kind == PGPU_LIGHT_POINT && l->radius > 0.0f) {
        float r = l->radius;
        float cos_at_light = dot(mk(-L.x, -L.y, -L.z), mk(0, 1, 0));
        if (cos_at_light < 0.01f) cos_at_light = 0.01f;
        pdf_light = (dist * dist) / (3.14159265f * r * r * cos_at_light);
    } else {
        pdf_light = 1.0f;
    }
    float w_light = (pdf_light * pdf_light) / (pdf_light * pdf_light + pdf_brdf * pdf_brdf + 1e-9f);
    float w_brdf = 1.0f - w_light;
    v3 nee = mulf(mulv(albedo, ld3(l->intensity)), ndotl);
    v3 brdf = mulv(albedo, ld3(l->intensity));
    return mulv(T, add(mulf(nee, w_light), mulf(brdf, w_brdf)));
}

static v3 trace_path(ctx_t* c, ray_t r, int bounces, rng_t* rng) {
    const orc_scene* s = c->s;
    float bias = c->p->shadow_bias;
    if (c->cnt) c->cnt[ORC_CNT_REFERENCE_RAYS]++;
    v3 T = mk(1, 1, 1);
    v3 rad = mk(0, 0, 0);
    ray_t cur = r;
    int depth = bounces;
    while (depth > 0) {
        hitrec rec;
        if (!scene_hit(&c->tv, cur, 1e-4f, 1e9f, &rec)) {
            rad = add(rad, mulv(T, ld3(s->background)));
            break;
        }
        const pgpu_material* m = &s->materials[rec.mat];
        rad = add(rad, mulv(T, ld3(m->emission)));
        v3 albedo = ld3(m->albedo);
        v3 sn = rec.n;
        for (int li = 0; li < s->n_lights; ++li) {
            const pgpu_light* l = &s->lights[li];
            if (l->kind == PGPU_LIGHT_QUAD) continue;
            v3 L; float dist;
            light_dir(l, rec.p, rng, &L, &dist);
            ray_t sr = {add(rec.p, mulf(rec.n, bias)), L};
            if (!l->is_emissive && scene_occ(&c->tv, sr, bias, dist - bias)) continue;
            float ndotl = clampf(dot(sn, L), 0.0f, 1.0f);
            rad = add(rad, light_term(l, (c->p->flags & PGPU_FLAG_MIS) != 0, T, albedo, L, dist,
                                      ndotl));
        }
        rad = add(rad, mulv(mulv(T, albedo), ld3(s->ambient)));
        if (bounces - depth > 3) {
            float p = fmaxf(T.x, fmaxf(T.y, T.z));
            if (rng_unit(rng) > p) break;
            T = divf(T, p);
        }
        v3 nd;
        v3 nT = mulv(T, albedo);
        if (m->kind == PGPU_MAT_METAL && m->reflectivity > 0.0f) {
            v3 refl = nrm(reflect(nrm(cur.d), sn));
            v3 upv = (fabsf(refl.y) < 0.9f) ? mk(0, 1, 0) : mk(1, 0, 0);
            v3 t1 = nrm(cross(refl, upv));
            v3 t2 = nrm(cross(refl, t1));
            float r1 = rng_unit(rng) * 0.1f;
            float r2 = rng_unit(rng) * 6.28f;
            nd = nrm(add(add(refl, mulf(t1, r1 * cosf(r2))), mulf(t2, r1 * sinf(r2))));
            nT = mulf(mulv(T, albedo), m->reflectivity);
        } else if (m->kind == PGPU_MAT_DIELECTRIC) {
            v3 g = dielectric(c, cur, &rec, m, albedo, depth, rng);
            rad = add(rad, sub(mulv(T, g), mulv(T, ld3(m->emission))));
            break;
        } else {
            float r1 = rng_unit(rng) * 6.2831853f;
            float r2 = rng_unit(rng);
            float r2s = sqrtf(r2);
            v3 N = sn;
            v3 upv = (fabsf(N.y) < 0.9f) ? mk(0, 1, 0) : mk(1, 0, 0);
            v3 Tn = nrm(cross(upv, N));
            v3 B = nrm(cross(N, Tn));
            nd = nrm(add(add(mulf(mulf(Tn, cosf(r1)), r2s), mulf(mulf(B, sinf(r1)), r2s)),
                         mulf(N, sqrtf(1.0f - r2))));
        }
        cur.o = add(rec.p, mulf(rec.n, bias));
        cur.d = nd;
        T = nT;
        depth--;
    }
    return rad;
}

/* ---- render_tile_region (src/renderer.hpp:309-390) ----------------------- */
typedef struct {
    const orc_scene* s;
    const pgpu_render_params* p;
    float* out;          /* the window's pixels, row-major */
    float* m2;
    int x0, y0, ww, wh;  /* window of the image: pixels [x0, x0+ww) x [y0, y0+wh) */
    int row0, stride;    /* window rows row0, row0 + stride, ... */
    uint64_t cnt[ORC_CNT_N];
} job_t;

static void render_pixel(const job_t* jb, ctx_t* c, int i, int j) {
    const pgpu_render_params* p = jb->p;
    const int W = p->width, H = p->height, n = p->samples;
    rng_t rng = {(uint32_t)(i * 97861u + j * 1973u + 1u)};
    v3 acc = mk(0, 0, 0);
    v3 sq = mk(0, 0, 0);
    for (int sy = 0; sy < n; ++sy) {
        for (int sx = 0; sx < n; ++sx) {
            float u = (i + (sx + 0.5f) / n) / (float)W;
            float v = 1.0f - (j + (sy + 0.5f) / n) / (float)H;
            u += rng_sym(&rng) * (0.5f / (W * n));
            v += rng_sym(&rng) * (0.5f / (H * n));
            ray_t r = camera_ray(jb->s, u, v);
            v3 col = (p->mode == PGPU_MODE_PATHTRACE) ? trace_path(c, r, p->depth, &rng)
                                                      : whitted(c, r, p->depth, &rng);
            acc = add(acc, col);
            sq = add(sq, mulv(col, col));
        }
    }
    acc = divf(acc, (float)(n * n));
    size_t o = ((size_t)(j - jb->y0) * jb->ww + (i - jb->x0)) * 3;
    jb->out[o + 0] = acc.x; jb->out[o + 1] = acc.y; jb->out[o + 2] = acc.z;
    if (jb->m2) {
        sq = divf(sq, (float)(n * n));
        jb->m2[o + 0] = sq.x; jb->m2[o + 1] = sq.y; jb->m2[o + 2] = sq.z;
    }
}

static void* render_thread(void* arg) {
    job_t* jb = (job_t*)arg;
    ctx_t c;
    c.s = jb->s;
    c.p = jb->p;
    c.cnt = jb->cnt;
    c.tv.s = jb->s;
    c.tv.cnt = jb->cnt;
    for (int j = jb->row0; j < jb->wh; j += jb->stride)
        for (int i = 0; i < jb->ww; ++i) render_pixel(jb, &c, jb->x0 + i, jb->y0 + j);
    return NULL;
}

/* A window of the image, checked against the image size; NULL: all of it. */
static int window_of(const pgpu_render_params* p, const int32_t* win, int w[4]) {
    if (!win) { w[0] = 0; w[1] = 0; w[2] = p->width; w[3] = p->height; return 0; }
    for (int k = 0; k < 4; ++k) w[k] = win[k];
    if (w[0] < 0 || w[1] < 0 || w[2] <= 0 || w[3] <= 0 || w[0] + w[2] > p->width ||
        w[1] + w[3] > p->height)
        return -1;
    return 0;
}

int32_t orc_render(const orc_scene* s, const pgpu_render_params* p, float* out_rgb,
                   float* out_m2, int32_t n_threads, uint64_t* counters) {
    return orc_render_window(s, p, NULL, out_rgb, out_m2, n_threads, counters);
}

int32_t orc_render_window(const orc_scene* s, const pgpu_render_params* p, const int32_t* win,
                          float* out_rgb, float* out_m2, int32_t n_threads, uint64_t* counters) {
    if (!s || !p || !out_rgb || p->width <= 0 || p->height <= 0 || p->samples <= 0) return -1;
    if (p->mode != PGPU_MODE_PATHTRACE && p->mode != PGPU_MODE_WHITTED) return -1;
    int w[4];
    if (window_of(p, win, w)) return -1;
    if (n_threads < 1) n_threads = 1;
    if (n_threads > w[3]) n_threads = w[3];
    job_t* jobs = (job_t*)calloc((size_t)n_threads, sizeof(job_t));
    pthread_t* th = (pthread_t*)calloc((size_t)n_threads, sizeof(pthread_t));
    char* live = (char*)calloc((size_t)n_threads, 1);
    for (int k = 0; k < n_threads; ++k) {
        jobs[k].s = s; jobs[k].p = p; jobs[k].out = out_rgb; jobs[k].m2 = out_m2;
        jobs[k].x0 = w[0]; jobs[k].y0 = w[1]; jobs[k].ww = w[2]; jobs[k].wh = w[3];
        jobs[k].row0 = k; jobs[k].stride = n_threads;
    }
    for (int k = 1; k < n_threads; ++k)
        live[k] = pthread_create(&th[k], NULL, render_thread, &jobs[k]) == 0;
    render_thread(&jobs[0]);
    for (int k = 1; k < n_threads; ++k) {
        if (live[k]) pthread_join(th[k], NULL);
        else render_thread(&jobs[k]);
    }
    if (counters) {
        for (int q = 0; q < ORC_CNT_N; ++q) {
            uint64_t acc = 0;
            for (int k = 0; k < n_threads; ++k) acc += jobs[k].cnt[q];
            counters[q] = acc;
        }
    }
    free(live);
    free(jobs);
    free(th);
    return 0;
}

/* The distributed worker's tile (render_tile, src/distributed.hpp:380-434):
 * pixels of the full W x H image seeded as render_tile_region does, jittered
 * by half a pixel, traced with trace (Whitted) to p->depth. */
int32_t orc_render_tile(const orc_scene* s, const pgpu_render_params* p, int32_t tx, int32_t ty,
                        int32_t tw, int32_t th, float* out_rgb) {
    if (!s || !p || !out_rgb || p->width <= 0 || p->height <= 0 || p->samples <= 0) return -1;
    if (tw <= 0 || th <= 0 || tx < 0 || ty < 0 || tx + tw > p->width || ty + th > p->height)
        return -1;
    uint64_t cnt[ORC_CNT_N] = {0};
    ctx_t c;
    c.s = s;
    c.p = p;
    c.cnt = cnt;
    c.tv.s = s;
    c.tv.cnt = cnt;
    const int W = p->width, H = p->height, n = p->samples;
    for (int j = 0; j < th; ++j) {
        for (int i = 0; i < tw; ++i) {
            const int px = tx + i, py = ty + j;
            rng_t rng = {(uint32_t)(px * 97861u + py * 1973u + 1u)};
            v3 acc = mk(0, 0, 0);
            for (int sy = 0; sy < n; ++sy) {
                for (int sx = 0; sx < n; ++sx) {
                    float u = (px + (sx + 0.5f) / n) / (float)W;
                    float v = 1.0f - (py + (sy + 0.5f) / n) / (float)H;
                    u += rng_sym(&rng) * (0.5f / W);
                    v += rng_sym(&rng) * (0.5f / H);
                    ray_t r = camera_ray(s, u, v);
                    acc = add(acc, whitted(&c, r, p->depth, &rng));
                }
            }
            acc = divf(acc, (float)(n * n));
            size_t o = ((size_t)j * tw + i) * 3;
            out_rgb[o + 0] = acc.x; out_rgb[o + 1] = acc.y; out_rgb[o + 2] = acc.z;
        }
    }
    return 0;
}

/* ---- the GPU core's single-ray estimator, restated ---------------------------
 * Test-only restatement of pencil_b200/csrc/path.cuh (shade_vertex, NeeAccum)
 * and of the megakernel's per-pixel accumulation: counter RNG seeded by
 * orc_path_seed, dielectric continuation along one Fresnel-chosen branch,
 * quad-light NEE at diffuse vertices with the emitter's emission skipped on
 * the following BSDF hit. Same float32 operation order as the device code,
 * so GPU and oracle agree path for path up to libm's last bits. */
enum { SPL_WHITTED = 1, SPL_SKIP_AREA = 2 };

typedef struct {
    int kind;          /* 0 none, 1 path-trace vertex, 2 Whitted vertex */
    v3 local, contrib;
} nee_acc;

static void nee_add(nee_acc* a, v3* L, v3 c, int group_end, int visible) {
    if (a->kind == 1) {
        if (visible) *L = add(*L, c);
    } else {
        if (visible) a->contrib = add(a->contrib, c);
        if (group_end > 0) {
            a->local = add(a->local, divf(a->contrib, (float)group_end));
            a->contrib = mk(0, 0, 0);
        }
    }
}

static void nee_finish(nee_acc* a, v3* L, v3 tail, v3 w, float sc) {
    if (a->kind == 1) {
        *L = add(*L, tail);
    } else if (a->kind == 2) {
        a->local = add(a->local, tail);
        *L = add(*L, mulv(w, mulf(a->local, sc)));
    }
}

static int quad_sample(const pgpu_light* l, float area, v3 p, v3 n, v3 sorg, float bias,
                       rng_t* rng, v3* L, float* tmax, float* w) {
    float u1 = rng_unit(rng);
    float u2 = rng_unit(rng);
    v3 y = add(add(ld3(l->pos), mulf(ld3(l->edge_u), u1)), mulf(ld3(l->edge_v), u2));
    v3 d = sub(y, p);
    float d2 = dot(d, d);
    float dist = sqrtf(d2);
    if (!(dist > 0.0f)) return 0;
    *L = divf(d, dist);
    float cx = dot(n, *L);
    if (cx <= 0.0f) return 0;
    v3 nq = nrm(cross(ld3(l->edge_u), ld3(l->edge_v)));
    float ly = dot(nq, *L);
    float cy = fabsf(ly);
    *w = cx * cy * area / (3.14159265f * d2);
    /* the biased shadow origin meets the emitter plane before |y - p|: test
     * visibility up to that plane, never against the emitter itself */
    *tmax = dot(sub(y, sorg), nq) / ly - bias;
    return *w > 0.0f;
}

typedef struct {
    ctx_t* c;
    const char* area_emitter;   /* per material */
    const float* quad_area;     /* per light */
    int has_quad;
} split_t;

/* shade_vertex of path.cuh with every shadow ray resolved on the spot. */
static int split_vertex(split_t* sp, ray_t* ray, v3* T, v3* L, rng_t* rng, int* depth,
                        unsigned* flags, int found, const hitrec* h) {
    ctx_t* c = sp->c;
    const orc_scene* s = c->s;
    const pgpu_render_params* P = c->p;
    const int whitted = (*flags & SPL_WHITTED) != 0;
    nee_acc acc;
    acc.kind = 0;
    v3 tail = mk(0, 0, 0), w = mk(0, 0, 0);
    float sc = 0.0f;
    int alive = 0;
    if (!found) {
        *L = add(*L, mulv(*T, ld3(s->background)));
        return 0;
    }
    const pgpu_material* m = &s->materials[h->mat];
    const v3 albedo = ld3(m->albedo);
    const int metal = m->kind == PGPU_MAT_METAL && m->reflectivity > 0.0f;
    const int glass = m->kind == PGPU_MAT_DIELECTRIC;
    const v3 sorg = add(h->p, mulf(h->n, P->shadow_bias));
    int dielectric = 0;
    if (!whitted) {
        const int diffuse = !metal && !glass;
        if (!glass && !((*flags & SPL_SKIP_AREA) && sp->area_emitter[h->mat]))
            *L = add(*L, mulv(*T, ld3(m->emission)));
        acc.kind = 1;
        for (int li = 0; li < s->n_lights; ++li) {
            const pgpu_light* l = &s->lights[li];
            if (l->kind == PGPU_LIGHT_QUAD) continue;
            v3 Ld; float dist;
            light_dir(l, h->p, rng, &Ld, &dist);
            float ndotl = clampf(dot(h->n, Ld), 0.0f, 1.0f);
            v3 cc = light_term(l, (P->flags & PGPU_FLAG_MIS) != 0, *T, albedo, Ld, dist, ndotl);
            ray_t sr = {sorg, Ld};
            int vis = l->is_emissive || !scene_occ(&c->tv, sr, P->shadow_bias, dist - P->shadow_bias);
            nee_add(&acc, L, cc, 0, vis);
        }
        if (sp->has_quad && diffuse && *depth - 1 > 0) {
            for (int li = 0; li < s->n_lights; ++li) {
                const pgpu_light* l = &s->lights[li];
                if (l->kind != PGPU_LIGHT_QUAD) continue;
                v3 Ld; float tmax, wq;
                if (!quad_sample(l, sp->quad_area[li], h->p, h->n, sorg, P->shadow_bias, rng,
                                 &Ld, &tmax, &wq)) continue;
                v3 cc = mulf(mulv(mulv(*T, albedo), ld3(l->intensity)), wq);
                ray_t sr = {sorg, Ld};
                int vis = !scene_occ(&c->tv, sr, P->shadow_bias, tmax);
                nee_add(&acc, L, cc, 0, vis);
            }
        }
        tail = mulv(mulv(*T, albedo), ld3(s->ambient));
        if (P->depth - *depth > 3) {
            float pr = fmaxf(T->x, fmaxf(T->y, T->z));
            if (rng_unit(rng) > pr) { nee_finish(&acc, L, tail, w, sc); return 0; }
            *T = divf(*T, pr);
        }
        if (!glass) {
            v3 nd;
            if (metal) {
                v3 refl = nrm(reflect(nrm(ray->d), h->n));
                v3 upv = (fabsf(refl.y) < 0.9f) ? mk(0, 1, 0) : mk(1, 0, 0);
                v3 t1 = nrm(cross(refl, upv));
                v3 t2 = nrm(cross(refl, t1));
                float r1 = rng_unit(rng) * 0.1f;
                float r2 = rng_unit(rng) * 6.28f;
                nd = nrm(add(add(refl, mulf(t1, r1 * cosf(r2))), mulf(t2, r1 * sinf(r2))));
                *T = mulf(mulv(*T, albedo), m->reflectivity);
            } else {
                float r1 = rng_unit(rng) * 6.2831853f;
                float r2 = rng_unit(rng);
                float r2s = sqrtf(r2);
                v3 N = h->n;
                v3 upv = (fabsf(N.y) < 0.9f) ? mk(0, 1, 0) : mk(1, 0, 0);
                v3 Tn = nrm(cross(upv, N));
                v3 B = nrm(cross(N, Tn));
                nd = nrm(add(add(mulf(mulf(Tn, cosf(r1)), r2s), mulf(mulf(B, sinf(r1)), r2s)),
                             mulf(N, sqrtf(1.0f - r2))));
                *T = mulv(*T, albedo);
            }
            *flags = (diffuse && sp->has_quad) ? SPL_SKIP_AREA : 0u;
            ray->o = sorg;
            ray->d = nd;
            *depth -= 1;
            alive = *depth > 0;
        } else {
            dielectric = 1;
        }
    } else {
        if (glass) acc.kind = 0;
        else { acc.kind = 2; acc.local = ld3(m->emission); acc.contrib = mk(0, 0, 0); }
        for (int li = 0; li < s->n_lights; ++li) {
            const pgpu_light* l = &s->lights[li];
            if (l->kind == PGPU_LIGHT_QUAD) continue;
            int ns = (l->radius > 0.0f) ? P->soft_shadow_samples : 1;
            for (int k = 0; k < ns; ++k) {
                v3 Ld; float dist;
                light_dir(l, h->p, rng, &Ld, &dist);
                if (glass) continue;
                float ndotl = clampf(dot(h->n, Ld), 0.0f, 1.0f);
                v3 cc = mulf(mulv(albedo, ld3(l->intensity)), ndotl);
                if (m->specular > 0.0f && ndotl > 0.0f) {
                    v3 V = neg(nrm(ray->d));
                    v3 H = nrm(add(Ld, V));
                    float ndoth = clampf(dot(h->n, H), 0.0f, 1.0f);
                    float spec = powf(ndoth, m->shininess);
                    cc = add(cc, mulf(mulv(ld3(m->specular_color), ld3(l->intensity)), spec * m->specular));
                }
                ray_t sr = {sorg, Ld};
                int vis = l->is_emissive || !scene_occ(&c->tv, sr, P->shadow_bias, dist - P->shadow_bias);
                nee_add(&acc, L, cc, k == ns - 1 ? ns : 0, vis);
            }
        }
        if (!glass) {
            tail = mulv(albedo, ld3(s->ambient));
            w = *T;
            if (metal) {
                sc = 1.0f - m->reflectivity;
                nee_finish(&acc, L, tail, w, sc);
                *T = mulf(mulv(*T, albedo), m->reflectivity);
                ray->o = sorg;
                ray->d = nrm(reflect(nrm(ray->d), h->n));
                *depth -= 1;
                return *depth > 0;
            }
            nee_finish(&acc, L, tail, w, 1.0f);
            return 0;
        }
        dielectric = 1;
    }
    nee_finish(&acc, L, tail, w, sc);
    if (!dielectric) return alive;
    {
        /* trace_dielectric's branches (src/renderer.hpp:1582-1627) */
        float safe = fmaxf(m->ior, 0.01f);
        float eta = h->front ? (1.0f / safe) : safe;
        v3 nd = nrm(ray->d);
        float cos_i = fabsf(dot(nd, h->n));
        float sin_t2 = eta * eta * (1.0f - cos_i * cos_i);
        ray_t refl = {add(h->p, mulf(h->n, P->shadow_bias)), nrm(reflect(nd, h->n))};
        int tir = sin_t2 > 1.0f;
        float kr = 1.0f;
        ray_t refr = refl;
        if (!tir) {
            float cos_t = sqrtf(1.0f - sin_t2);
            refr.o = sub(h->p, mulf(h->n, P->shadow_bias));
            refr.d = nrm(add(mulf(nd, eta), mulf(h->n, eta * cos_i - cos_t)));
            kr = schlick(h->front ? cos_i : cos_t, eta);
        }
        if (tir || rng_unit(rng) < kr) *ray = refl;
        else *ray = refr;
        *T = mulv(*T, albedo);
        *depth -= 1;
        *flags = SPL_WHITTED;
        return *depth > 0;
    }
}

static v3 split_sample(split_t* sp, ray_t r, rng_t* rng) {
    ctx_t* c = sp->c;
    v3 T = mk(1, 1, 1), L = mk(0, 0, 0);
    int depth = c->p->depth;
    unsigned flags = c->p->mode == PGPU_MODE_WHITTED ? SPL_WHITTED : 0u;
    if (c->cnt) c->cnt[ORC_CNT_REFERENCE_RAYS]++;
    int alive = depth > 0;
    while (alive) {
        hitrec h;
        int found = scene_hit(&c->tv, r, 1e-4f, 1e9f, &h);
        alive = split_vertex(sp, &r, &T, &L, rng, &depth, &flags, found, &h);
    }
    return L;
}

typedef struct {
    const orc_scene* s;
    const pgpu_render_params* p;
    float* out;          /* the window's pixels, row-major */
    float* m2;
    int x0, y0, ww, wh;  /* window of the image */
    int row0, stride;    /* window rows row0, row0 + stride, ... */
    const char* area_emitter;
    const float* quad_area;
    int has_quad;
    uint64_t cnt[ORC_CNT_N];
} sjob_t;

static void* split_thread(void* arg) {
    sjob_t* jb = (sjob_t*)arg;
    const pgpu_render_params* p = jb->p;
    ctx_t c;
    c.s = jb->s; c.p = p; c.cnt = jb->cnt; c.tv.s = jb->s; c.tv.cnt = jb->cnt;
    split_t sp = {&c, jb->area_emitter, jb->quad_area, jb->has_quad};
    const int W = p->width, H = p->height, n = p->samples, spp = n * n;
    int G = 1;
    while (G * 2 <= (spp < 32 ? spp : 32)) G *= 2;
    for (int jw = jb->row0; jw < jb->wh; jw += jb->stride) {
        const int j = jb->y0 + jw;
        for (int i = jb->x0; i < jb->x0 + jb->ww; ++i) {
            v3 acc[32], acc2[32];
            for (int g = 0; g < G; ++g) {
                acc[g] = mk(0, 0, 0);
                acc2[g] = mk(0, 0, 0);
                for (int smp = g; smp < spp; smp += G) {
                    rng_t rng = {orc_path_seed(i, j, smp + p->sample_offset, p->seed)};
                    float u = (i + ((smp % n) + 0.5f) / n) / (float)W;
                    float v = 1.0f - (j + ((smp / n) + 0.5f) / n) / (float)H;
                    u += rng_sym(&rng) * (0.5f / (W * n));
                    v += rng_sym(&rng) * (0.5f / (H * n));
                    v3 col = split_sample(&sp, camera_ray(jb->s, u, v), &rng);
                    acc[g] = add(acc[g], col);
                    acc2[g] = add(acc2[g], mulv(col, col));
                }
            }
            for (int off = G >> 1; off > 0; off >>= 1)
                for (int g = 0; g < off; ++g) {
                    acc[g] = add(acc[g], acc[g + off]);
                    acc2[g] = add(acc2[g], acc2[g + off]);
                }
            size_t o = ((size_t)jw * jb->ww + (i - jb->x0)) * 3;
            jb->out[o + 0] = acc[0].x / (float)spp;
            jb->out[o + 1] = acc[0].y / (float)spp;
            jb->out[o + 2] = acc[0].z / (float)spp;
            if (jb->m2) {
                jb->m2[o + 0] = acc2[0].x / (float)spp;
                jb->m2[o + 1] = acc2[0].y / (float)spp;
                jb->m2[o + 2] = acc2[0].z / (float)spp;
            }
        }
    }
    return NULL;
}

int32_t orc_render_split(const orc_scene* s, const pgpu_render_params* p, float* out_rgb,
                         float* out_m2, int32_t n_threads, uint64_t* counters) {
    return orc_render_split_window(s, p, NULL, out_rgb, out_m2, n_threads, counters);
}

int32_t orc_render_split_window(const orc_scene* s, const pgpu_render_params* p,
                                const int32_t* win, float* out_rgb, float* out_m2,
                                int32_t n_threads, uint64_t* counters) {
    if (!s || !p || !out_rgb || p->width <= 0 || p->height <= 0 || p->samples <= 0) return -1;
    int w[4];
    if (window_of(p, win, w)) return -1;
    char* area_emitter = (char*)calloc((size_t)(s->n_materials > 0 ? s->n_materials : 1), 1);
    float* quad_area = (float*)calloc((size_t)(s->n_lights > 0 ? s->n_lights : 1), sizeof(float));
    int has_quad = 0;
    for (int k = 0; k < s->n_lights; ++k) {
        const pgpu_light* l = &s->lights[k];
        if (l->kind != PGPU_LIGHT_QUAD) continue;
        v3 cr = cross(ld3(l->edge_u), ld3(l->edge_v));
        quad_area[k] = sqrtf(cr.x * cr.x + cr.y * cr.y + cr.z * cr.z);
        if (l->material >= 0 && l->material < s->n_materials) area_emitter[l->material] = 1;
        has_quad = 1;
    }
    if (n_threads < 1) n_threads = 1;
    if (n_threads > w[3]) n_threads = w[3];
    sjob_t* jobs = (sjob_t*)calloc((size_t)n_threads, sizeof(sjob_t));
    pthread_t* th = (pthread_t*)calloc((size_t)n_threads, sizeof(pthread_t));
    char* live = (char*)calloc((size_t)n_threads, 1);
    for (int k = 0; k < n_threads; ++k) {
        sjob_t* jb = &jobs[k];
        jb->s = s; jb->p = p; jb->out = out_rgb; jb->m2 = out_m2;
        jb->x0 = w[0]; jb->y0 = w[1]; jb->ww = w[2]; jb->wh = w[3];
        jb->row0 = k; jb->stride = n_threads;
        jb->area_emitter = area_emitter; jb->quad_area = quad_area; jb->has_quad = has_quad;
    }
    for (int k = 1; k < n_threads; ++k)
        live[k] = pthread_create(&th[k], NULL, split_thread, &jobs[k]) == 0;
    split_thread(&jobs[0]);
    for (int k = 1; k < n_threads; ++k) {
        if (live[k]) pthread_join(th[k], NULL);
        else split_thread(&jobs[k]);
    }
    if (counters)
        for (int q = 0; q < ORC_CNT_N; ++q) {
            uint64_t a = 0;
            for (int k = 0; k < n_threads; ++k) a += jobs[k].cnt[q];
            counters[q] = a;
        }
    free(live); free(jobs); free(th); free(area_emitter); free(quad_area);
    return 0;
}

/* ---- FP64 adjoint of the production estimator ---------------------------------
 * Test-only restatement of pencil_b200/csrc/adjoint.cu: each path is replayed
 * with exactly the float32 geometry and decisions of the production
 * estimator (the float throughput drives Russian roulette, as on the GPU);
 * the tape, the backward sweep and every gradient sum are kept in double. */
typedef struct { double x, y, z; } dv3;
static inline dv3 dvk(double x, double y, double z) { dv3 r = {x, y, z}; return r; }
static inline dv3 dvf(v3 a) { return dvk(a.x, a.y, a.z); }
static inline dv3 dvadd(dv3 a, dv3 b) { return dvk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline dv3 dvmul(dv3 a, dv3 b) { return dvk(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline dv3 dvs(dv3 a, double s) { return dvk(a.x * s, a.y * s, a.z * s); }

#define ADJ_MAX_TAPE 16

typedef struct {
    int mat;
    dv3 T, B, g, A;
} tape_t;

typedef struct {
    const orc_scene* s;
    const pgpu_render_params* p;
    const char* area_emitter;
    const float* quad_area;
    int has_quad;
    double* d_albedo;   /* per thread accumulators (3 per material) */
    double* d_emission;
    double* d_light;
    trav_t tv;
} adj_ctx;

/* Replay one path; returns its radiance (double) and adds to the gradients. */
static dv3 adj_path(adj_ctx* a, ray_t r, rng_t* rng, dv3 w) {
    const orc_scene* s = a->s;
    const pgpu_render_params* P = a->p;
    tape_t tape[ADJ_MAX_TAPE];
    int nt = 0;
    v3 Tf = mk(1, 1, 1);               /* float throughput: drives decisions */
    dv3 T = dvk(1, 1, 1), L = dvk(0, 0, 0);
    int depth = P->depth;
    unsigned flags = P->mode == PGPU_MODE_WHITTED ? SPL_WHITTED : 0u;
    int alive = depth > 0;
    while (alive && nt < ADJ_MAX_TAPE) {
        tape_t* tv = &tape[nt++];
        tv->T = T;
        tv->B = dvk(0, 0, 0);
        tv->g = dvk(0, 0, 0);
        hitrec h;
        if (!scene_hit(&a->tv, r, 1e-4f, 1e9f, &h)) {
            tv->mat = -1;
            tv->A = dvf(ld3(s->background));
            L = dvadd(L, dvmul(T, tv->A));
            break;
        }
        const pgpu_material* m = &s->materials[h.mat];
        const v3 albedo = ld3(m->albedo);
        const dv3 ad = dvf(albedo);
        const int metal = m->kind == PGPU_MAT_METAL && m->reflectivity > 0.0f;
        const int glass = m->kind == PGPU_MAT_DIELECTRIC;
        const v3 sorg = add(h.p, mulf(h.n, P->shadow_bias));
        tv->mat = h.mat;
        dv3 e = dvk(0, 0, 0);
        int dielectric = 0;
        alive = 0;
        if (!(flags & SPL_WHITTED)) {
            const int diffuse = !metal && !glass;
            if (!glass && !((flags & SPL_SKIP_AREA) && a->area_emitter[h.mat])) {
                e = dvf(ld3(m->emission));
                double* g = a->d_emission + 3 * h.mat;
                dv3 c = dvmul(w, T);
                g[0] += c.x; g[1] += c.y; g[2] += c.z;
            }
            for (int li = 0; li < s->n_lights; ++li) {
                const pgpu_light* l = &s->lights[li];
                if (l->kind == PGPU_LIGHT_QUAD) continue;
                v3 Ld; float dist;
                light_dir(l, h.p, rng, &Ld, &dist);
                float ndotl = clampf(dot(h.n, Ld), 0.0f, 1.0f);
                ray_t sr = {sorg, Ld};
                int vis = l->is_emissive || !scene_occ(&a->tv, sr, P->shadow_bias, dist - P->shadow_bias);
                if (!vis) continue;
                tv->B = dvadd(tv->B, dvs(dvf(ld3(l->intensity)), ndotl));
                dv3 c = dvs(dvmul(dvmul(w, T), ad), ndotl);
                a->d_light[3 * li] += c.x; a->d_light[3 * li + 1] += c.y; a->d_light[3 * li + 2] += c.z;
            }
            if (a->has_quad && diffuse && depth - 1 > 0) {
                for (int li = 0; li < s->n_lights; ++li) {
                    const pgpu_light* l = &s->lights[li];
                    if (l->kind != PGPU_LIGHT_QUAD) continue;
                    v3 Ld; float tmax, wq;
                    if (!quad_sample(l, a->quad_area[li], h.p, h.n, sorg, P->shadow_bias, rng,
                                     &Ld, &tmax, &wq)) continue;
                    ray_t sr = {sorg, Ld};
                    if (scene_occ(&a->tv, sr, P->shadow_bias, tmax)) continue;
                    tv->B = dvadd(tv->B, dvs(dvf(ld3(l->intensity)), wq));
                    dv3 c = dvs(dvmul(dvmul(w, T), ad), wq);
                    a->d_light[3 * li] += c.x; a->d_light[3 * li + 1] += c.y; a->d_light[3 * li + 2] += c.z;
                }
            }
            tv->B = dvadd(tv->B, dvf(ld3(s->ambient)));
            tv->A = dvadd(e, dvmul(ad, tv->B));
            L = dvadd(L, dvmul(T, tv->A));
            double inv_p = 1.0;
            if (P->depth - depth > 3) {
                float pr = fmaxf(Tf.x, fmaxf(Tf.y, Tf.z));
                if (rng_unit(rng) > pr) break;
                Tf = divf(Tf, pr);
                inv_p = 1.0 / (double)pr;
                T = dvs(T, inv_p);
            }
            if (!glass) {
                v3 nd;
                if (metal) {
                    v3 refl = nrm(reflect(nrm(r.d), h.n));
                    v3 upv = (fabsf(refl.y) < 0.9f) ? mk(0, 1, 0) : mk(1, 0, 0);
                    v3 t1 = nrm(cross(refl, upv));
                    v3 t2 = nrm(cross(refl, t1));
                    float r1 = rng_unit(rng) * 0.1f;
                    float r2 = rng_unit(rng) * 6.28f;
                    nd = nrm(add(add(refl, mulf(t1, r1 * cosf(r2))), mulf(t2, r1 * sinf(r2))));
                    Tf = mulf(mulv(Tf, albedo), m->reflectivity);
                    T = dvs(dvmul(T, ad), m->reflectivity);
                    tv->g = dvs(dvk(inv_p, inv_p, inv_p), m->reflectivity);
                } else {
                    float r1 = rng_unit(rng) * 6.2831853f;
                    float r2 = rng_unit(rng);
                    float r2s = sqrtf(r2);
                    v3 N = h.n;
                    v3 upv = (fabsf(N.y) < 0.9f) ? mk(0, 1, 0) : mk(1, 0, 0);
                    v3 Tn = nrm(cross(upv, N));
                    v3 B = nrm(cross(N, Tn));
                    nd = nrm(add(add(mulf(mulf(Tn, cosf(r1)), r2s), mulf(mulf(B, sinf(r1)), r2s)),
                                 mulf(N, sqrtf(1.0f - r2))));
                    Tf = mulv(Tf, albedo);
                    T = dvmul(T, ad);
                    tv->g = dvk(inv_p, inv_p, inv_p);
                }
                flags = (diffuse && a->has_quad) ? SPL_SKIP_AREA : 0u;
                r.o = sorg;
                r.d = nd;
                depth--;
                alive = depth > 0;
                if (!alive) tv->g = dvk(0, 0, 0);
                continue;
            }
            tv->g = dvk(inv_p, inv_p, inv_p);
            dielectric = 1;
        } else {
            dv3 sum_a = dvk(0, 0, 0), sum_e = dvk(0, 0, 0);
            double sc = 1.0;
            if (!glass) {
                sum_e = dvf(ld3(m->emission));
                sc = metal ? (double)(1.0f - m->reflectivity) : 1.0;
            }
            for (int li = 0; li < s->n_lights; ++li) {
                const pgpu_light* l = &s->lights[li];
                if (l->kind == PGPU_LIGHT_QUAD) continue;
                int ns = (l->radius > 0.0f) ? P->soft_shadow_samples : 1;
                dv3 ca = dvk(0, 0, 0), ce = dvk(0, 0, 0);
                for (int k = 0; k < ns; ++k) {
                    v3 Ld; float dist;
                    light_dir(l, h.p, rng, &Ld, &dist);
                    if (glass) continue;
                    float ndotl = clampf(dot(h.n, Ld), 0.0f, 1.0f);
                    v3 phong = mk(0, 0, 0);
                    if (m->specular > 0.0f && ndotl > 0.0f) {
                        v3 V = neg(nrm(r.d));
                        v3 H = nrm(add(Ld, V));
                        float ndoth = clampf(dot(h.n, H), 0.0f, 1.0f);
                        float spec = powf(ndoth, m->shininess);
                        phong = mulf(ld3(m->specular_color), spec * m->specular);
                    }
                    ray_t sr = {sorg, Ld};
                    if (!l->is_emissive && scene_occ(&a->tv, sr, P->shadow_bias, dist - P->shadow_bias)) continue;
                    ca = dvadd(ca, dvs(dvf(ld3(l->intensity)), ndotl));
                    ce = dvadd(ce, dvmul(dvf(ld3(l->intensity)), dvf(phong)));
                    dv3 c = dvs(dvmul(dvmul(w, T), dvadd(dvs(ad, ndotl), dvf(phong))), sc / ns);
                    a->d_light[3 * li] += c.x; a->d_light[3 * li + 1] += c.y; a->d_light[3 * li + 2] += c.z;
                }
                sum_a = dvadd(sum_a, dvs(ca, 1.0 / ns));
                sum_e = dvadd(sum_e, dvs(ce, 1.0 / ns));
            }
            if (!glass) {
                double* g = a->d_emission + 3 * h.mat;
                dv3 c = dvs(dvmul(w, T), sc);
                g[0] += c.x; g[1] += c.y; g[2] += c.z;
                tv->B = dvs(dvadd(sum_a, dvf(ld3(s->ambient))), sc);
                tv->A = dvadd(dvs(sum_e, sc), dvmul(ad, tv->B));
                L = dvadd(L, dvmul(T, tv->A));
                if (metal) {
                    Tf = mulf(mulv(Tf, albedo), m->reflectivity);
                    T = dvs(dvmul(T, ad), m->reflectivity);
                    tv->g = dvk(m->reflectivity, m->reflectivity, m->reflectivity);
                    r.o = sorg;
                    r.d = nrm(reflect(nrm(r.d), h.n));
                    depth--;
                    alive = depth > 0;
                    if (!alive) tv->g = dvk(0, 0, 0);
                }
                continue;
            }
            tv->A = dvk(0, 0, 0);
            tv->g = dvk(1, 1, 1);
            dielectric = 1;
        }
        if (dielectric) {
            float safe = fmaxf(m->ior, 0.01f);
            float eta = h.front ? (1.0f / safe) : safe;
            v3 ndr = nrm(r.d);
            float cos_i = fabsf(dot(ndr, h.n));
            float sin_t2 = eta * eta * (1.0f - cos_i * cos_i);
            ray_t refl = {add(h.p, mulf(h.n, P->shadow_bias)), nrm(reflect(ndr, h.n))};
            int tir = sin_t2 > 1.0f;
            float kr = 1.0f;
            ray_t refr = refl;
            if (!tir) {
                float cos_t = sqrtf(1.0f - sin_t2);
                refr.o = sub(h.p, mulf(h.n, P->shadow_bias));
                refr.d = nrm(add(mulf(ndr, eta), mulf(h.n, eta * cos_i - cos_t)));
                kr = schlick(h.front ? cos_i : cos_t, eta);
            }
            if (tir || rng_unit(rng) < kr) r = refl;
            else r = refr;
            Tf = mulv(Tf, albedo);
            T = dvmul(T, ad);
            depth--;
            flags = SPL_WHITTED;
            alive = depth > 0;
            if (!alive) tv->g = dvk(0, 0, 0);
        }
    }
    /* backward sweep */
    dv3 R = dvk(0, 0, 0);
    for (int k = nt - 1; k >= 0; --k) {
        tape_t* tv = &tape[k];
        if (tv->mat >= 0) {
            dv3 ad = dvf(ld3(s->materials[tv->mat].albedo));
            dv3 c = dvmul(dvmul(w, tv->T), dvadd(tv->B, dvmul(tv->g, R)));
            double* g = a->d_albedo + 3 * tv->mat;
            g[0] += c.x; g[1] += c.y; g[2] += c.z;
            R = dvadd(tv->A, dvmul(dvmul(ad, tv->g), R));
        } else {
            R = tv->A;
        }
    }
    return L;
}

typedef struct {
    adj_ctx a;
    const float* dl;
    double* img;        /* per-pixel radiance sums (double) */
    int row0, stride;
} ajob_t;

static void* adj_thread(void* arg) {
    ajob_t* jb = (ajob_t*)arg;
    adj_ctx* a = &jb->a;
    const pgpu_render_params* p = a->p;
    const int W = p->width, H = p->height, n = p->samples, spp = n * n;
    for (int j = jb->row0; j < H; j += jb->stride) {
        for (int i = 0; i < W; ++i) {
            size_t o = ((size_t)j * W + i) * 3;
            dv3 w = dvk((double)jb->dl[o] / spp, (double)jb->dl[o + 1] / spp, (double)jb->dl[o + 2] / spp);
            dv3 acc = dvk(0, 0, 0);
            for (int smp = 0; smp < spp; ++smp) {
                rng_t rng = {orc_path_seed(i, j, smp + p->sample_offset, p->seed)};
                float u = (i + ((smp % n) + 0.5f) / n) / (float)W;
                float v = 1.0f - (j + ((smp / n) + 0.5f) / n) / (float)H;
                u += rng_sym(&rng) * (0.5f / (W * n));
                v += rng_sym(&rng) * (0.5f / (H * n));
                acc = dvadd(acc, adj_path(a, camera_ray(a->s, u, v), &rng, w));
            }
            if (jb->img) {
                jb->img[o] = acc.x / spp; jb->img[o + 1] = acc.y / spp; jb->img[o + 2] = acc.z / spp;
            }
        }
    }
    return NULL;
}

int32_t orc_adjoint(const orc_scene* s, const pgpu_render_params* p, const float* dl,
                    double* d_albedo, double* d_emission, double* d_light, double* out_img,
                    int32_t n_threads) {
    if (!s || !p || !dl || !d_albedo || !d_emission) return -1;
    if (p->depth > ADJ_MAX_TAPE) return -1;
    const int nm = s->n_materials, nl = s->n_lights;
    char* area_emitter = (char*)calloc((size_t)(nm > 0 ? nm : 1), 1);
    float* quad_area = (float*)calloc((size_t)(nl > 0 ? nl : 1), sizeof(float));
    int has_quad = 0;
    for (int k = 0; k < nl; ++k) {
        const pgpu_light* l = &s->lights[k];
        if (l->kind != PGPU_LIGHT_QUAD) continue;
        v3 cr = cross(ld3(l->edge_u), ld3(l->edge_v));
        quad_area[k] = sqrtf(cr.x * cr.x + cr.y * cr.y + cr.z * cr.z);
        if (l->material >= 0 && l->material < nm) area_emitter[l->material] = 1;
        has_quad = 1;
    }
    if (n_threads < 1) n_threads = 1;
    if (n_threads > p->height) n_threads = p->height;
    ajob_t* jobs = (ajob_t*)calloc((size_t)n_threads, sizeof(ajob_t));
    pthread_t* th = (pthread_t*)calloc((size_t)n_threads, sizeof(pthread_t));
    char* live = (char*)calloc((size_t)n_threads, 1);
    for (int k = 0; k < n_threads; ++k) {
        ajob_t* jb = &jobs[k];
        jb->a.s = s; jb->a.p = p; jb->a.area_emitter = area_emitter; jb->a.quad_area = quad_area;
        jb->a.has_quad = has_quad;
        jb->a.d_albedo = (double*)calloc((size_t)nm * 3 + 1, sizeof(double));
        jb->a.d_emission = (double*)calloc((size_t)nm * 3 + 1, sizeof(double));
        jb->a.d_light = (double*)calloc((size_t)nl * 3 + 1, sizeof(double));
        jb->a.tv.s = s; jb->a.tv.cnt = NULL;
        jb->dl = dl; jb->img = out_img; jb->row0 = k; jb->stride = n_threads;
    }
    for (int k = 1; k < n_threads; ++k)
        live[k] = pthread_create(&th[k], NULL, adj_thread, &jobs[k]) == 0;
    adj_thread(&jobs[0]);
    for (int k = 1; k < n_threads; ++k) {
        if (live[k]) pthread_join(th[k], NULL);
        else adj_thread(&jobs[k]);
    }
    for (int q = 0; q < nm * 3; ++q) {
        double sa = 0, se = 0;
        for (int k = 0; k < n_threads; ++k) { sa += jobs[k].a.d_albedo[q]; se += jobs[k].a.d_emission[q]; }
        d_albedo[q] = sa; d_emission[q] = se;
    }
    if (d_light)
        for (int q = 0; q < nl * 3; ++q) {
            double sl = 0;
            for (int k = 0; k < n_threads; ++k) sl += jobs[k].a.d_light[q];
            d_light[q] = sl;
        }
    for (int k = 0; k < n_threads; ++k) {
        free(jobs[k].a.d_albedo); free(jobs[k].a.d_emission); free(jobs[k].a.d_light);
    }
    free(jobs); free(th); free(live); free(area_emitter); free(quad_area);
    return 0;
}

/* ---- ray queries ---------------------------------------------------------- */
void orc_trace_rays(const orc_scene* s, const float* rays, int32_t n, int32_t* prim_id,
                    float* t, uint64_t* counters) {
    trav_t tv = {s, counters};
    for (int k = 0; k < n; ++k) {
        ray_t r = {ld3(rays + 6 * k), ld3(rays + 6 * k + 3)};
        hitrec h;
        h.prim = -1;
        if (scene_hit(&tv, r, 1e-4f, 1e9f, &h)) {
            prim_id[k] = h.prim;
            t[k] = h.t;
        } else {
            prim_id[k] = -1;
            t[k] = -1.0f;
        }
    }
}

void orc_camera_rays(const orc_scene* s, const float* uv, int32_t n, float* rays) {
    for (int k = 0; k < n; ++k) {
        ray_t r = camera_ray(s, uv[2 * k], uv[2 * k + 1]);
        rays[6 * k + 0] = r.o.x; rays[6 * k + 1] = r.o.y; rays[6 * k + 2] = r.o.z;
        rays[6 * k + 3] = r.d.x; rays[6 * k + 4] = r.d.y; rays[6 * k + 5] = r.d.z;
    }
}

void orc_primary_hits(const orc_scene* s, const float* uv, int32_t n, int32_t* prim_id, float* t) {
    trav_t tv = {s, NULL};
    for (int k = 0; k < n; ++k) {
        ray_t r = camera_ray(s, uv[2 * k], uv[2 * k + 1]);
        hitrec h;
        if (scene_hit(&tv, r, 1e-4f, 1e9f, &h)) {
            prim_id[k] = h.prim;
            t[k] = h.t;
        } else {
            prim_id[k] = -1;
            t[k] = -1.0f;
        }
    }
}

/* ---- FP64 hit distance recomputation -------------------------------------- */
typedef struct { double x, y, z; } d3;
static inline d3 dk(double x, double y, double z) { d3 r = {x, y, z}; return r; }
static inline d3 dsub(d3 a, d3 b) { return dk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline d3 dadd(d3 a, d3 b) { return dk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline d3 dmul(d3 a, double s) { return dk(a.x * s, a.y * s, a.z * s); }
static inline double ddot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline d3 dcross(d3 a, d3 b) {
    return dk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline d3 dld(const float* p) { return dk(p[0], p[1], p[2]); }
static inline double dcomp(d3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

static int quad_roots(double a, double b, double c, double* t0, double* t1) {
    double disc = b * b - 4.0 * a * c;
    if (disc < 0.0 || a == 0.0) return 0;
    double sq = sqrt(disc);
    *t0 = (-b - sq) / (2.0 * a);
    *t1 = (-b + sq) / (2.0 * a);
    return 1;
}

static double best_of(double cur, double t) {
    if (t < 1e-4 || t > 1e9) return cur;
    if (cur < 0.0 || t < cur) return t;
    return cur;
}

double orc_hit_t_fp64(const pgpu_prim* pr, const float* rayf) {
    d3 o = dld(rayf), d = dld(rayf + 3);
    double best = -1.0;
    switch (pr->type) {
        case PGPU_PRIM_SPHERE: {
            d3 c = dld(pr->p);
            double r = pr->p[3];
            d3 oc = dsub(o, c);
            double t0, t1;
            if (quad_roots(ddot(d, d), 2.0 * ddot(oc, d), ddot(oc, oc) - r * r, &t0, &t1)) {
                best = best_of(best, t0);
                if (best < 0.0) best = best_of(best, t1);
            }
            return best;
        }
        case PGPU_PRIM_TRIANGLE: {
            d3 v0 = dld(pr->p), v1 = dld(pr->p + 3), v2 = dld(pr->p + 6);
            d3 e1 = dsub(v1, v0), e2 = dsub(v2, v0);
            d3 n = dcross(e1, e2);
            double den = ddot(n, d);
            if (den == 0.0) return -1.0;
            double t = ddot(dsub(v0, o), n) / den;
            return best_of(best, t);
        }
        case PGPU_PRIM_PLANE: {
            d3 pt = dld(pr->p), n = dld(pr->p + 3);
            double den = ddot(n, d);
            if (den == 0.0) return -1.0;
            return best_of(best, ddot(dsub(pt, o), n) / den);
        }
        case PGPU_PRIM_CUBE: {
            d3 c = dld(pr->p);
            double h = pr->p[3];
            double tn = -INFINITY, tf = INFINITY;
            for (int a = 0; a < 3; ++a) {
                double da = dcomp(d, a), oa = dcomp(o, a), ca = dcomp(c, a);
                if (da == 0.0) {
                    if (oa < ca - h || oa > ca + h) return -1.0;
                    continue;
                }
                double t0 = (ca - h - oa) / da, t1 = (ca + h - oa) / da;
                if (t0 > t1) { double x = t0; t0 = t1; t1 = x; }
                if (t0 > tn) tn = t0;
                if (t1 < tf) tf = t1;
            }
            if (tf < tn) return -1.0;
            best = best_of(best, tn);
            if (best < 0.0) best = best_of(best, tf);
            return best;
        }
        case PGPU_PRIM_CYLINDER:
        case PGPU_PRIM_CONE: {
            d3 c = dld(pr->p), ax = dld(pr->p + 3);
            double rad = pr->p[6], hp = pr->p[7];
            d3 oc = dsub(o, c);
            double dda = ddot(d, ax), oca = ddot(oc, ax);
            d3 dp = dsub(d, dmul(ax, dda)), op = dsub(oc, dmul(ax, oca));
            double t0, t1, a, b, cc;
            int cyl = pr->type == PGPU_PRIM_CYLINDER;
            double k2 = cyl ? 0.0 : (rad / hp) * (rad / hp);
            a = ddot(dp, dp) - k2 * dda * dda;
            b = 2.0 * (ddot(op, dp) - k2 * dda * oca);
            cc = ddot(op, op) - (cyl ? rad * rad : k2 * oca * oca);
            if (quad_roots(a, b, cc, &t0, &t1)) {
                double ts[2] = {t0, t1};
                for (int q = 0; q < 2; ++q) {
                    double hh = oca + ts[q] * dda;
                    int ok = cyl ? fabs(hh) <= hp : (hh >= 0.0 && hh <= hp);
                    if (ok && ts[q] >= 1e-4 && ts[q] <= 1e9) { best = best_of(best, ts[q]); break; }
                }
            }
            /* caps */
            int ncap = cyl ? 2 : 1;
            for (int q = 0; q < ncap; ++q) {
                double sg = cyl ? (q == 0 ? 1.0 : -1.0) : -1.0;
                d3 cc3 = cyl ? dadd(c, dmul(ax, sg * hp)) : dsub(c, dmul(ax, hp));
                d3 n = dmul(ax, sg);
                double den = ddot(n, d);
                if (den == 0.0) continue;
                double t = ddot(dsub(cc3, o), n) / den;
                d3 pp = dadd(o, dmul(d, t));
                d3 dd = dsub(pp, cc3);
                if (ddot(dd, dd) <= rad * rad) best = best_of(best, t);
            }
            return best;
        }
        default:
            return -1.0;
    }
}

/* ---- write_image's HDR -> 8-bit path (src/image_io.hpp:63-113) ----------- */
static float aces(float x) {
    float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
    float y = (x * (a * x + b)) / (x * (c * x + d) + e);
    return y > 0.0f ? y : 0.0f;
}

void orc_rgb8(const float* hdr, int32_t n_pixels, uint8_t* out, int32_t tonemap, float exposure) {
    float e = powf(2.0f, exposure);
    for (int k = 0; k < n_pixels; ++k) {
        for (int ch = 0; ch < 3; ++ch) {
            float x = hdr[3 * k + ch] * e;
            if (tonemap == 1) x = aces(x);
            else if (tonemap == 2) x = x / (1.0f + x);
            x = clampf(x, 0.0f, 1.0f);
            x = powf(x, 1.0f / 2.2f);
            out[3 * k + ch] = (uint8_t)(x * 255.0f + 0.5f);
        }
    }
}

/* Checks that the 8-bit gamma step of write_image (src/image_io.hpp:88-97),
 * x -> (uint8)(pow(clamp(x, 0, 1), 1/2.2) * 255 + 0.5) with this host's powf,
 * never decreases over all floats in [0, 1] (in bit order). Returns 0, or the
 * bit pattern after which it first decreased. */
uint32_t orc_gamma_monotone(void) {
    uint8_t prev = 0;
    for (uint32_t b = 0; b <= 0x3f800000u; ++b) {
        float x;
        memcpy(&x, &b, 4);
        float g = powf(clampf(x, 0.0f, 1.0f), 1.0f / 2.2f);
        uint8_t q = (uint8_t)(g * 255.0f + 0.5f);
        if (q < prev) return b;
        prev = q;
    }
    return 0;
}
