// harness.cpp - drives the reference Pencil renderer for parity pinning and
// CPU timing. TEST INFRASTRUCTURE ONLY: built by oracle/ref/Makefile from the
// reference's own headers into oracle/_ref/pencil_ref; never shipped.
//
// Commands (all binary files little-endian, formats in scene_io below):
//   dump   <scene.bin> <out.bin>        stored primitive state + DFS BVH
//   render <scene.bin> <out.f32> W H n depth mode bias soft threads repeat
//                                       mode 0 = trace_path, 1 = Whitted,
//                                       2 = trace_path_mis;
//                                       prints {"seconds":[...],"rays":N}
//   hits   <scene.bin> <rays.f32> <out.bin>   closest hit per ray
//   tile   <scene.bin> <out.f32> W H x y w h n depth bias soft
//                                       the distributed worker's tile render
//   parse  <file.pecl> <out_scene.bin>  reference parser -> scene file,
//                                       prints the render block as JSON
//
// Private members of the reference types are read through the usual
// "#define private public" trick, applied only to this translation unit
// after every standard header has been included.
#include <algorithm>
#include <atomic>
#include <cassert>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <random>
#include <set>
#include <sstream>
#include <string>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <utility>
#include <vector>

#define private public
#define protected public
#include "pecl_parser.hpp"
#include "renderer.hpp"
#include "distributed.hpp"
#undef private
#undef protected

#include "../../include/pencil_gpu.h"

using namespace pencil;

namespace {

// ---- scene file -------------------------------------------------------------
// "PGPUSCN1", int32 n_prims, n_materials, n_lights, pgpu_camera,
// float background[3], ambient[3], pgpu_prim[n_prims],
// pgpu_material[n_materials], pgpu_light[n_lights]
struct SceneFile {
    pgpu_camera cam{};
    float bg[3]{}, amb[3]{};
    std::vector<pgpu_prim> prims;
    std::vector<pgpu_material> mats;
    std::vector<pgpu_light> lights;
};

bool read_scene(const char* path, SceneFile& sf) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    char magic[8];
    int32_t n[3];
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "PGPUSCN1", 8) == 0 &&
              std::fread(n, 4, 3, f) == 3 && std::fread(&sf.cam, sizeof(pgpu_camera), 1, f) == 1 &&
              std::fread(sf.bg, 4, 3, f) == 3 && std::fread(sf.amb, 4, 3, f) == 3;
    if (ok) {
        sf.prims.resize(n[0]);
        sf.mats.resize(n[1]);
        sf.lights.resize(n[2]);
        ok = std::fread(sf.prims.data(), sizeof(pgpu_prim), n[0], f) == (size_t)n[0] &&
             std::fread(sf.mats.data(), sizeof(pgpu_material), n[1], f) == (size_t)n[1] &&
             std::fread(sf.lights.data(), sizeof(pgpu_light), n[2], f) == (size_t)n[2];
    }
    std::fclose(f);
    return ok;
}

bool write_scene(const char* path, const SceneFile& sf) {
    FILE* f = std::fopen(path, "wb");
    if (!f) return false;
    int32_t n[3] = {(int32_t)sf.prims.size(), (int32_t)sf.mats.size(), (int32_t)sf.lights.size()};
    std::fwrite("PGPUSCN1", 1, 8, f);
    std::fwrite(n, 4, 3, f);
    std::fwrite(&sf.cam, sizeof(pgpu_camera), 1, f);
    std::fwrite(sf.bg, 4, 3, f);
    std::fwrite(sf.amb, 4, 3, f);
    std::fwrite(sf.prims.data(), sizeof(pgpu_prim), sf.prims.size(), f);
    std::fwrite(sf.mats.data(), sizeof(pgpu_material), sf.mats.size(), f);
    std::fwrite(sf.lights.data(), sizeof(pgpu_light), sf.lights.size(), f);
    std::fclose(f);
    return true;
}

Vec3 v3(const float* p) { return Vec3{p[0], p[1], p[2]}; }
void put3(float* d, const Vec3& v) { d[0] = v.x; d[1] = v.y; d[2] = v.z; }

// ---- pgpu_prim <-> reference primitive objects ------------------------------
// Objects are built through their constructors, then their stored fields are
// set to the file's stored state, so that no re-normalisation changes a bit.
std::shared_ptr<Primitive> make_ref_prim(const pgpu_prim& p) {
    const float* q = p.p;
    switch (p.type) {
        case PGPU_PRIM_SPHERE:
            return std::make_shared<Sphere>(v3(q), q[3], p.material);
        case PGPU_PRIM_TRIANGLE: {
            auto t = std::make_shared<Triangle>(v3(q), v3(q + 3), v3(q + 6), p.material);
            return t;
        }
        case PGPU_PRIM_CUBE:
            return std::make_shared<Cube>(v3(q), q[3], p.material);
        case PGPU_PRIM_PLANE: {
            auto pl = std::make_shared<Plane>(v3(q), v3(q + 3), p.material);
            pl->normal_ = v3(q + 3);
            return pl;
        }
        case PGPU_PRIM_CYLINDER: {
            auto c = std::make_shared<Cylinder>(v3(q), v3(q + 3), q[6], 2.0f * q[7], p.material);
            c->axis_ = v3(q + 3);
            c->half_h_ = q[7];
            return c;
        }
        case PGPU_PRIM_CONE: {
            auto c = std::make_shared<Cone>(v3(q), v3(q + 3), q[6], q[7], p.material);
            c->axis_ = v3(q + 3);
            c->base_center_ = c->apex_ - c->axis_ * c->height_;
            return c;
        }
        default:
            return nullptr;
    }
}

bool prim_state(const Primitive* pr, pgpu_prim& out) {
    std::memset(&out, 0, sizeof(out));
    if (auto s = dynamic_cast<const Sphere*>(pr)) {
        out.type = PGPU_PRIM_SPHERE; out.material = s->material_id_;
        put3(out.p, s->center_); out.p[3] = s->radius_;
    } else if (auto t = dynamic_cast<const Triangle*>(pr)) {
        out.type = PGPU_PRIM_TRIANGLE; out.material = t->material_id_;
        put3(out.p, t->v0_); put3(out.p + 3, t->v1_); put3(out.p + 6, t->v2_);
    } else if (auto c = dynamic_cast<const Cube*>(pr)) {
        out.type = PGPU_PRIM_CUBE; out.material = c->material_id_;
        put3(out.p, c->center_); out.p[3] = c->half_;
    } else if (auto pl = dynamic_cast<const Plane*>(pr)) {
        out.type = PGPU_PRIM_PLANE; out.material = pl->material_id_;
        put3(out.p, pl->point_); put3(out.p + 3, pl->normal_);
    } else if (auto cy = dynamic_cast<const Cylinder*>(pr)) {
        out.type = PGPU_PRIM_CYLINDER; out.material = cy->material_id_;
        put3(out.p, cy->center_); put3(out.p + 3, cy->axis_);
        out.p[6] = cy->radius_; out.p[7] = cy->half_h_;
    } else if (auto co = dynamic_cast<const Cone*>(pr)) {
        out.type = PGPU_PRIM_CONE; out.material = co->material_id_;
        put3(out.p, co->apex_); put3(out.p + 3, co->axis_);
        out.p[6] = co->radius_; out.p[7] = co->height_;
    } else {
        return false;
    }
    return true;
}

Material make_ref_material(const pgpu_material& m) {
    Material r;
    r.kind = (MaterialKind)m.kind;
    r.albedo = v3(m.albedo);
    r.emission = v3(m.emission);
    r.reflectivity = m.reflectivity;
    r.ior = m.ior;
    r.specular = m.specular;
    r.shininess = m.shininess;
    r.specular_color = v3(m.specular_color);
    return r;
}

Light make_ref_light(const pgpu_light& l) {
    Light r;
    r.kind = (LightKind)l.kind;
    r.position_or_direction = v3(l.pos);
    r.intensity = v3(l.intensity);
    r.radius = l.radius;
    r.is_emissive = l.is_emissive != 0;
    return r;
}

// Wrapper that records which primitive produced the last accepted hit, so
// that the reference traversal reports a primitive index.
thread_local int g_last_hit = -1;
class Tagged : public Primitive {
public:
    Tagged(std::shared_ptr<Primitive> p, int id) : inner_(std::move(p)), id_(id) {}
    bool hit(const Ray& r, float t_min, float t_max, HitRecord& out) const override {
        bool ok = inner_->hit(r, t_min, t_max, out);
        if (ok) g_last_hit = id_;
        return ok;
    }
    AABB aabb() const override { return inner_->aabb(); }
    std::shared_ptr<Primitive> inner_;
    int id_;
};

struct Built {
    Scene scene;
    Camera camera;
    std::unordered_map<const Primitive*, int> index;
};

void build_scene(const SceneFile& sf, Built& b, bool tagged) {
    for (const auto& m : sf.mats) b.scene.add_material(make_ref_material(m));
    for (const auto& l : sf.lights) b.scene.add_light(make_ref_light(l));
    for (size_t k = 0; k < sf.prims.size(); ++k) {
        auto p = make_ref_prim(sf.prims[k]);
        if (!p) { std::fprintf(stderr, "bad primitive type at %zu\n", k); std::exit(2); }
        std::shared_ptr<Primitive> q = tagged ? std::make_shared<Tagged>(p, (int)k) : p;
        b.index[q.get()] = (int)k;
        b.scene.add_primitive(q);
    }
    b.scene.background = v3(sf.bg);
    b.scene.ambient = v3(sf.amb);
    b.scene.build_bvh();
    const pgpu_camera& c = sf.cam;
    b.camera = Camera(v3(c.eye), v3(c.look), v3(c.up), c.vfov_deg, c.aspect, c.aperture,
                      c.focus_dist);
}

// ---- BVH dump in DFS pre-order -----------------------------------------------
void dfs(const BVHNode* n, const Built& b, std::vector<pgpu_bvh_node>& out, int depth,
         int& max_depth) {
    max_depth = std::max(max_depth, depth);
    int me = (int)out.size();
    out.push_back(pgpu_bvh_node{});
    put3(out[me].bmin, n->box.min);
    put3(out[me].bmax, n->box.max);
    if (n->is_leaf()) {
        out[me].left = -1;
        out[me].right = b.index.at(n->leaf.get());
        return;
    }
    out[me].left = me + 1;
    dfs(n->left.get(), b, out, depth + 1, max_depth);
    out[me].right = (int)out.size();
    dfs(n->right.get(), b, out, depth + 1, max_depth);
}

int cmd_dump(int argc, char** argv) {
    if (argc < 4) return 2;
    SceneFile sf;
    if (!read_scene(argv[2], sf)) { std::fprintf(stderr, "cannot read scene\n"); return 2; }
    Built b;
    build_scene(sf, b, false);
    std::vector<pgpu_bvh_node> nodes;
    int max_depth = 0;
    if (b.scene.bvh_.root_) dfs(b.scene.bvh_.root_.get(), b, nodes, 1, max_depth);
    FILE* f = std::fopen(argv[3], "wb");
    int32_t hdr[3] = {(int32_t)sf.prims.size(), (int32_t)nodes.size(), max_depth};
    std::fwrite(hdr, 4, 3, f);
    // stored state of every primitive, as the reference objects hold it
    for (const auto& p : b.scene.primitives_) {
        pgpu_prim st;
        prim_state(p.get(), st);
        std::fwrite(&st, sizeof(st), 1, f);
    }
    std::fwrite(nodes.data(), sizeof(pgpu_bvh_node), nodes.size(), f);
    std::fclose(f);
    return 0;
}

int cmd_render(int argc, char** argv) {
    if (argc < 13) return 2;
    SceneFile sf;
    if (!read_scene(argv[2], sf)) { std::fprintf(stderr, "cannot read scene\n"); return 2; }
    Built b;
    build_scene(sf, b, false);
    RenderSettings rs;
    rs.width = std::atoi(argv[4]);
    rs.height = std::atoi(argv[5]);
    rs.samples = std::atoi(argv[6]);
    rs.max_depth = std::atoi(argv[7]);
    // mode: 0 path tracing (trace_path), 1 Whitted (trace), 2 path tracing
    // with multiple importance sampling (trace_path_mis)
    rs.pathtrace = std::atoi(argv[8]) != 1;
    rs.mis = std::atoi(argv[8]) == 2;
    rs.pathtrace_bounces = rs.max_depth;
    rs.shadow_bias = (float)std::atof(argv[9]);
    rs.soft_shadow_samples = std::atoi(argv[10]);
    rs.threads = std::atoi(argv[11]);
    int repeat = std::max(1, std::atoi(argv[12]));
    std::vector<Color> px;
    RenderStats st;
    std::vector<double> secs;
    for (int k = 0; k < repeat; ++k) {
        Renderer r(b.scene, b.camera, rs);
        auto t0 = std::chrono::steady_clock::now();
        r.render(px, &st);
        auto t1 = std::chrono::steady_clock::now();
        secs.push_back(std::chrono::duration<double>(t1 - t0).count());
    }
    if (std::strcmp(argv[3], "-") != 0) {
        FILE* f = std::fopen(argv[3], "wb");
        std::fwrite(px.data(), sizeof(Color), px.size(), f);
        std::fclose(f);
    }
    std::printf("{\"seconds\": [");
    for (size_t k = 0; k < secs.size(); ++k) std::printf("%s%.6f", k ? ", " : "", secs[k]);
    std::printf("], \"rays\": %llu, \"threads\": %d}\n", (unsigned long long)st.rays_traced,
                rs.threads);
    return 0;
}

int cmd_hits(int argc, char** argv) {
    if (argc < 5) return 2;
    SceneFile sf;
    if (!read_scene(argv[2], sf)) { std::fprintf(stderr, "cannot read scene\n"); return 2; }
    Built b;
    build_scene(sf, b, true);
    std::ifstream in(argv[3], std::ios::binary | std::ios::ate);
    size_t bytes = (size_t)in.tellg();
    in.seekg(0);
    std::vector<float> rays(bytes / 4);
    in.read(reinterpret_cast<char*>(rays.data()), (std::streamsize)bytes);
    size_t n = rays.size() / 6;
    std::vector<int32_t> prim(n);
    std::vector<float> tt(n);
    for (size_t k = 0; k < n; ++k) {
        Ray r{v3(&rays[6 * k]), v3(&rays[6 * k + 3])};
        HitRecord h;
        g_last_hit = -1;
        if (b.scene.hit(r, 1e-4f, 1e9f, h)) {
            prim[k] = g_last_hit;
            tt[k] = h.t;
        } else {
            prim[k] = -1;
            tt[k] = -1.0f;
        }
    }
    FILE* f = std::fopen(argv[4], "wb");
    std::fwrite(prim.data(), 4, n, f);
    std::fwrite(tt.data(), 4, n, f);
    std::fclose(f);
    return 0;
}

// The distributed worker's tile render (render_tile, src/distributed.hpp:380-434).
int cmd_tile(int argc, char** argv) {
    if (argc < 14) return 2;
    SceneFile sf;
    if (!read_scene(argv[2], sf)) { std::fprintf(stderr, "cannot read scene\n"); return 2; }
    Built b;
    build_scene(sf, b, false);
    const int W = std::atoi(argv[4]), H = std::atoi(argv[5]);
    const int tx = std::atoi(argv[6]), ty = std::atoi(argv[7]);
    const int tw = std::atoi(argv[8]), th = std::atoi(argv[9]);
    RenderSettings rs;
    rs.width = W;
    rs.height = H;
    rs.samples = std::atoi(argv[10]);
    rs.max_depth = std::atoi(argv[11]);
    rs.shadow_bias = (float)std::atof(argv[12]);
    rs.soft_shadow_samples = std::atoi(argv[13]);
    std::vector<Color> px;
    render_tile(b.scene, b.camera, tx, ty, tw, th, W, H, rs.samples, rs.max_depth, px, &rs);
    FILE* f = std::fopen(argv[3], "wb");
    std::fwrite(px.data(), sizeof(Color), px.size(), f);
    std::fclose(f);
    return 0;
}

int cmd_camrays(int argc, char** argv) {
    // camrays <scene.bin> <uv.f32> <out.f32>: Camera::ray_at(u, v) per point
    if (argc < 5) return 2;
    SceneFile sf;
    if (!read_scene(argv[2], sf)) return 2;
    Built b;
    build_scene(sf, b, false);
    std::ifstream in(argv[3], std::ios::binary | std::ios::ate);
    size_t bytes = (size_t)in.tellg();
    in.seekg(0);
    std::vector<float> uv(bytes / 4);
    in.read(reinterpret_cast<char*>(uv.data()), (std::streamsize)bytes);
    size_t n = uv.size() / 2;
    std::vector<float> out(6 * n);
    for (size_t k = 0; k < n; ++k) {
        Ray r = b.camera.ray_at(uv[2 * k], uv[2 * k + 1]);
        put3(&out[6 * k], r.origin);
        put3(&out[6 * k + 3], r.direction);
    }
    FILE* f = std::fopen(argv[4], "wb");
    std::fwrite(out.data(), 4, out.size(), f);
    std::fclose(f);
    return 0;
}

int cmd_parse(int argc, char** argv) {
    if (argc < 4) return 2;
    ParsedScene ps;
    std::vector<ParseError> errs;
    if (!parse_pecl(argv[2], ps, errs)) {
        for (auto& e : errs) std::fprintf(stderr, "line %d: %s\n", e.line, e.what.c_str());
        return 3;
    }
    SceneFile sf;
    sf.cam.eye[0] = ps.eye.x; sf.cam.eye[1] = ps.eye.y; sf.cam.eye[2] = ps.eye.z;
    sf.cam.look[0] = ps.look.x; sf.cam.look[1] = ps.look.y; sf.cam.look[2] = ps.look.z;
    sf.cam.up[0] = ps.up.x; sf.cam.up[1] = ps.up.y; sf.cam.up[2] = ps.up.z;
    sf.cam.vfov_deg = ps.fov;
    sf.cam.aspect = ps.aspect;
    sf.cam.aperture = ps.aperture;
    sf.cam.focus_dist = ps.focus_dist;
    put3(sf.bg, ps.scene.background);
    put3(sf.amb, ps.scene.ambient);
    for (const auto& p : ps.scene.primitives_) {
        pgpu_prim st;
        if (!prim_state(p.get(), st)) { std::fprintf(stderr, "unsupported primitive\n"); return 4; }
        sf.prims.push_back(st);
    }
    for (const auto& m : ps.scene.materials_) {
        if (m.texture || m.normal_map || m.displacement_map || m.sss > 0.0f || m.refdis ||
            m.kind == MaterialKind::Principled) {
            std::fprintf(stderr, "unsupported material feature\n");
            return 4;
        }
        pgpu_material g{};
        g.kind = (int32_t)m.kind;
        put3(g.albedo, m.albedo);
        put3(g.emission, m.emission);
        g.reflectivity = m.reflectivity;
        g.ior = m.ior;
        g.specular = m.specular;
        g.shininess = m.shininess;
        put3(g.specular_color, m.specular_color);
        sf.mats.push_back(g);
    }
    for (const auto& l : ps.scene.lights_) {
        pgpu_light g{};
        g.kind = (int32_t)l.kind;
        put3(g.pos, l.position_or_direction);
        put3(g.intensity, l.intensity);
        g.radius = l.radius;
        g.is_emissive = l.is_emissive ? 1 : 0;
        sf.lights.push_back(g);
    }
    write_scene(argv[3], sf);
    std::printf("{\"width\": %d, \"height\": %d, \"samples\": %d, \"depth\": %d, "
                "\"pathtrace\": %d, \"skybox\": %d, \"fog\": %d}\n",
                ps.width, ps.height, ps.samples, ps.depth, ps.enable_pathtrace ? 1 : 0,
                ps.scene.skybox ? 1 : 0, ps.scene.fog.enabled ? 1 : 0);
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: pencil_ref dump|render|hits|camrays|parse ...\n");
        return 2;
    }
    std::string c = argv[1];
    if (c == "dump") return cmd_dump(argc, argv);
    if (c == "render") return cmd_render(argc, argv);
    if (c == "hits") return cmd_hits(argc, argv);
    if (c == "camrays") return cmd_camrays(argc, argv);
    if (c == "tile") return cmd_tile(argc, argv);
    if (c == "parse") return cmd_parse(argc, argv);
    std::fprintf(stderr, "unknown command %s\n", argv[1]);
    return 2;
}
