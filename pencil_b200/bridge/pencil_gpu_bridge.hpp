// pencil_gpu_bridge.hpp - Pencil's side of the GPU core: flattens a parsed
// Pencil scene (its primitives, its already-built SAH BVH, materials, lights,
// camera) into the C-ABI of include/pencil_gpu.h and renders it in place of
// pencil::Renderer::render (src/renderer.hpp:198-295).
//
// Include it after Pencil's own headers in pencil.cpp. It reads stored fields
// that Pencil keeps private; Pencil grants access with one line per class,
//     friend struct ::pencil_gpu::Access;
// in Scene, BVH, Sphere, Triangle, Cube, Plane, Cylinder and Cone, after a
// forward declaration `namespace pencil_gpu { struct Access; }`.
#pragma once

#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "pencil_gpu.h"

namespace pencil_gpu {

// Flattened scene: owns the arrays a pgpu_scene points into.
struct SceneTables {
    std::vector<pgpu_prim> prims;
    std::vector<pgpu_bvh_node> nodes;
    std::vector<pgpu_material> materials;
    std::vector<pgpu_light> lights;
    pgpu_scene desc{};
};

struct Access {
    static const std::vector<std::shared_ptr<pencil::Primitive>>& primitives(
        const pencil::Scene& s) {
        return s.primitives_;
    }
    static const pencil::BVHNode* root(const pencil::Scene& s) {
        return s.bvh_built_ ? s.bvh_.root_.get() : nullptr;
    }

    // A primitive's stored state (src/primitives.hpp); false for kinds the
    // GPU core does not implement (ImplicitSurface).
    static bool prim_state(const pencil::Primitive* p, pgpu_prim& out) {
        std::memset(&out, 0, sizeof(out));
        auto put = [](float* d, const pencil::Vec3& v) { d[0] = v.x; d[1] = v.y; d[2] = v.z; };
        if (auto s = dynamic_cast<const pencil::Sphere*>(p)) {
            out.type = PGPU_PRIM_SPHERE; out.material = s->material_id_;
            put(out.p, s->center_); out.p[3] = s->radius_;
        } else if (auto t = dynamic_cast<const pencil::Triangle*>(p)) {
            out.type = PGPU_PRIM_TRIANGLE; out.material = t->material_id_;
            put(out.p, t->v0_); put(out.p + 3, t->v1_); put(out.p + 6, t->v2_);
        } else if (auto c = dynamic_cast<const pencil::Cube*>(p)) {
            out.type = PGPU_PRIM_CUBE; out.material = c->material_id_;
            put(out.p, c->center_); out.p[3] = c->half_;
        } else if (auto pl = dynamic_cast<const pencil::Plane*>(p)) {
            out.type = PGPU_PRIM_PLANE; out.material = pl->material_id_;
            put(out.p, pl->point_); put(out.p + 3, pl->normal_);
        } else if (auto cy = dynamic_cast<const pencil::Cylinder*>(p)) {
            out.type = PGPU_PRIM_CYLINDER; out.material = cy->material_id_;
            put(out.p, cy->center_); put(out.p + 3, cy->axis_);
            out.p[6] = cy->radius_; out.p[7] = cy->half_h_;
        } else if (auto co = dynamic_cast<const pencil::Cone*>(p)) {
            out.type = PGPU_PRIM_CONE; out.material = co->material_id_;
            put(out.p, co->apex_); put(out.p + 3, co->axis_);
            out.p[6] = co->radius_; out.p[7] = co->height_;
        } else {
            return false;
        }
        return true;
    }
};

// Pencil's BVH as the DFS pre-order table the C-ABI takes: the order in
// which BVH::build_range created the nodes (src/bvh.hpp:74-104).
inline void walk(const pencil::BVHNode* n,
                 const std::unordered_map<const pencil::Primitive*, int>& index,
                 std::vector<pgpu_bvh_node>& out) {
    int me = (int)out.size();
    out.push_back(pgpu_bvh_node{});
    pgpu_bvh_node& d = out[me];
    d.bmin[0] = n->box.min.x; d.bmin[1] = n->box.min.y; d.bmin[2] = n->box.min.z;
    d.bmax[0] = n->box.max.x; d.bmax[1] = n->box.max.y; d.bmax[2] = n->box.max.z;
    if (n->is_leaf()) {
        out[me].left = -1;
        out[me].right = index.at(n->leaf.get());
        return;
    }
    out[me].left = me + 1;
    walk(n->left.get(), index, out);
    out[me].right = (int)out.size();
    walk(n->right.get(), index, out);
}

// Flatten `ps` (after ParsedScene::finalize). Returns false with the reason
// when the scene uses something outside the GPU core.
inline bool describe(const pencil::ParsedScene& ps, SceneTables& t, std::string& why) {
    const pencil::Scene& sc = ps.scene;
    if (sc.skybox) { why = "skybox backgrounds are not supported on the GPU"; return false; }
    if (sc.fog.enabled) { why = "fog is not supported on the GPU"; return false; }
    if (ps.aperture > 0.0f) { why = "depth of field is not supported on the GPU"; return false; }
    const auto& prims = Access::primitives(sc);
    std::unordered_map<const pencil::Primitive*, int> index;
    t.prims.resize(prims.size());
    for (size_t k = 0; k < prims.size(); ++k) {
        if (!Access::prim_state(prims[k].get(), t.prims[k])) {
            why = "implicit surfaces are not supported on the GPU";
            return false;
        }
        index[prims[k].get()] = (int)k;
    }
    for (const auto& m : sc.materials()) {
        if (m.texture || m.normal_map || m.displacement_map || m.sss > 0.0f || m.refdis ||
            m.kind == pencil::MaterialKind::Principled) {
            why = "textures, normal/displacement maps, SSS, dispersion and principled "
                  "materials are not supported on the GPU";
            return false;
        }
        pgpu_material g{};
        g.kind = (int32_t)m.kind;
        g.albedo[0] = m.albedo.x; g.albedo[1] = m.albedo.y; g.albedo[2] = m.albedo.z;
        g.emission[0] = m.emission.x; g.emission[1] = m.emission.y; g.emission[2] = m.emission.z;
        g.reflectivity = m.reflectivity;
        g.ior = m.ior;
        g.specular = m.specular;
        g.shininess = m.shininess;
        g.specular_color[0] = m.specular_color.x;
        g.specular_color[1] = m.specular_color.y;
        g.specular_color[2] = m.specular_color.z;
        t.materials.push_back(g);
    }
    for (const auto& l : sc.lights()) {
        pgpu_light g{};
        g.kind = (int32_t)l.kind;
        g.pos[0] = l.position_or_direction.x; g.pos[1] = l.position_or_direction.y;
        g.pos[2] = l.position_or_direction.z;
        g.intensity[0] = l.intensity.x; g.intensity[1] = l.intensity.y;
        g.intensity[2] = l.intensity.z;
        g.radius = l.radius;
        g.is_emissive = l.is_emissive ? 1 : 0;
        t.lights.push_back(g);
    }
    t.nodes.clear();
    if (const pencil::BVHNode* root = Access::root(sc)) walk(root, index, t.nodes);
    pgpu_scene& d = t.desc;
    d = pgpu_scene{};
    d.prims = t.prims.data(); d.n_prims = (int32_t)t.prims.size();
    d.nodes = t.nodes.empty() ? nullptr : t.nodes.data(); d.n_nodes = (int32_t)t.nodes.size();
    d.materials = t.materials.data(); d.n_materials = (int32_t)t.materials.size();
    d.lights = t.lights.data(); d.n_lights = (int32_t)t.lights.size();
    auto cp = [](float* o, const pencil::Vec3& v) { o[0] = v.x; o[1] = v.y; o[2] = v.z; };
    cp(d.camera.eye, ps.eye); cp(d.camera.look, ps.look); cp(d.camera.up, ps.up);
    d.camera.vfov_deg = ps.fov; d.camera.aspect = ps.aspect;
    d.camera.aperture = ps.aperture; d.camera.focus_dist = ps.focus_dist;
    cp(d.background, sc.background);
    cp(d.ambient, sc.ambient);
    return true;
}

// Render settings of the GPU core from Pencil's. PENCIL_GPU_EXACT=1 selects
// the megakernel with Pencil's own per-pixel random stream and both glass
// branches (Pencil's image up to libm's last bits); the default is the
// wavefront engine with the counter RNG (same expectation, faster).
inline bool params_of(const pencil::RenderSettings& rs, pgpu_render_params& p, std::string& why) {
    if (rs.normals_mode || rs.bloom || rs.denoise || rs.bdpt || rs.spectral || rs.volume ||
        rs.sss_enabled || rs.god_rays || rs.motion_blur || rs.adaptive || rs.caustics ||
        rs.ppm) {
        why = "only the path tracer (plain or MIS) and the Whitted tracer run on the GPU";
        return false;
    }
    p = pgpu_render_params{};
    p.width = rs.width;
    p.height = rs.height;
    p.samples = rs.samples;
    p.mode = rs.pathtrace ? PGPU_MODE_PATHTRACE : PGPU_MODE_WHITTED;
    p.depth = rs.pathtrace ? rs.pathtrace_bounces : rs.max_depth;
    p.shadow_bias = rs.shadow_bias;
    p.soft_shadow_samples = rs.soft_shadow_samples;
    if (rs.pathtrace && rs.mis) p.flags |= PGPU_FLAG_MIS;   // trace_path_mis (renderer.hpp:341)
    const char* exact = std::getenv("PENCIL_GPU_EXACT");
    if (exact && exact[0] == '1') {
        p.engine = PGPU_ENGINE_MEGAKERNEL;
        p.rng = PGPU_RNG_PIXEL_SEQUENTIAL;
        p.glass = PGPU_GLASS_BOTH_BRANCHES;
    }
    return true;
}

// Drop-in for `Renderer(ps.scene, ps.camera, rs).render(out, stats)`: same
// output layout; stats->rays_traced gets Pencil's count (one per trace*
// call). Returns 0, or a pgpu_status with `why` set.
inline int render(const pencil::ParsedScene& ps, const pencil::RenderSettings& rs,
                  std::vector<pencil::Color>& out, pencil::RenderStats* stats,
                  std::string& why, int device = 0) {
    SceneTables t;
    if (!describe(ps, t, why)) return PGPU_ERR_UNSUPPORTED;
    pgpu_render_params p;
    if (!params_of(rs, p, why)) return PGPU_ERR_UNSUPPORTED;
    if (stats) p.flags |= PGPU_FLAG_COUNT_RAYS;
    pgpu_ctx* ctx = nullptr;
    int rc = pgpu_create(device, &ctx);
    if (rc) { why = "no usable CUDA device"; return rc; }
    // Scenes with a triangle mesh: the wide traversals walk a tree built on
    // the device over Pencil's leaves (same leaf boxes and leaf order, so
    // the same hits); Pencil's split binning over parent boxes groups a fine
    // mesh inside large walls badly. PENCIL_GPU_TREE=uploaded|lbvh|sah
    // chooses explicitly.
    int tree = t.desc.n_mesh_triangles > 0 ? PGPU_TRAVERSAL_LBVH : PGPU_TRAVERSAL_UPLOADED;
    if (const char* e = std::getenv("PENCIL_GPU_TREE")) {
        const std::string v = e;
        if (v == "uploaded") tree = PGPU_TRAVERSAL_UPLOADED;
        else if (v == "lbvh") tree = PGPU_TRAVERSAL_LBVH;
        else if (v == "sah") tree = PGPU_TRAVERSAL_SAH;
    }
    pgpu_set_traversal_tree(ctx, tree);
    int sid = 0;
    rc = pgpu_upload_scene(ctx, &t.desc, &sid);
    if (rc == PGPU_OK) {
        out.assign((size_t)rs.width * rs.height, pencil::Color{0, 0, 0});
        pgpu_stats st{};
        static_assert(sizeof(pencil::Color) == 3 * sizeof(float), "Color is three floats");
        rc = pgpu_render(ctx, sid, &p, reinterpret_cast<float*>(out.data()), nullptr, &st);
        if (rc == PGPU_OK && stats) stats->rays_traced = st.reference_rays;
        pgpu_free_scene(ctx, sid);
    }
    if (rc) why = pgpu_last_error(ctx);
    pgpu_destroy(ctx);
    return rc;
}

}  // namespace pencil_gpu
