// bvh_build.cpp - host construction of Pencil's SAH BVH, and of primitive
// stored state from constructor arguments.
//
// The tree must be node-for-node the one BVH::build makes
// (src/bvh.hpp:54-192), because Pencil's --gpu mode uploads that tree and the
// library can also be asked to build it. The steps therefore follow the
// reference exactly: box of the range; one primitive -> leaf; longest axis;
// <= 4 primitives -> sort by centroid sum and split at the middle; else 12
// bucket SAH with cost 1 + (nL*SA_L + nR*SA_R)/SA_P, partition by bucket,
// falling back to the median split. std::sort and std::partition are called
// with the same comparisons on a sequence of the same length, so they produce
// the same permutation as the reference's calls on its shared_ptr vector.
// Compiled with -ffp-contract=off so every float operation rounds as the
// reference's do.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/pencil_gpu.h"
#include "host_internal.h"

namespace pgpu {

namespace {

struct Box {
    float mn[3] = {1e30f, 1e30f, 1e30f};
    float mx[3] = {-1e30f, -1e30f, -1e30f};
};

inline Box merge(const Box& a, const Box& b) {
    Box o;
    for (int k = 0; k < 3; ++k) {
        o.mn[k] = std::fmin(a.mn[k], b.mn[k]);
        o.mx[k] = std::fmax(a.mx[k], b.mx[k]);
    }
    return o;
}

inline int longest_axis(const Box& b) {
    float ex = b.mx[0] - b.mn[0], ey = b.mx[1] - b.mn[1], ez = b.mx[2] - b.mn[2];
    if (ex >= ey && ex >= ez) return 0;
    if (ey >= ez) return 1;
    return 2;
}

inline float surface_area(const Box& b) {
    float ex = b.mx[0] - b.mn[0], ey = b.mx[1] - b.mn[1], ez = b.mx[2] - b.mn[2];
    return 2.0f * (ex * ey + ey * ez + ex * ez);
}

// Primitive::aabb for every kind (src/primitives.hpp).
Box prim_box(const pgpu_prim& p) {
    Box b;
    const float* q = p.p;
    switch (p.type) {
        case PGPU_PRIM_SPHERE:
        case PGPU_PRIM_CUBE:
            for (int k = 0; k < 3; ++k) { b.mn[k] = q[k] - q[3]; b.mx[k] = q[k] + q[3]; }
            break;
        case PGPU_PRIM_TRIANGLE:
            for (int k = 0; k < 3; ++k) {
                b.mn[k] = std::fmin(std::fmin(q[k], q[3 + k]), q[6 + k]);
                b.mx[k] = std::fmax(std::fmax(q[k], q[3 + k]), q[6 + k]);
            }
            break;
        case PGPU_PRIM_PLANE:
            for (int k = 0; k < 3; ++k) { b.mn[k] = -1e6f; b.mx[k] = 1e6f; }
            break;
        case PGPU_PRIM_CYLINDER: {
            float r = q[6], hh = q[7];
            for (int k = 0; k < 3; ++k) {
                float ext = std::fabs(q[3 + k] * hh) + r;
                b.mn[k] = q[k] - ext;
                b.mx[k] = q[k] + ext;
            }
            break;
        }
        case PGPU_PRIM_CONE: {
            float r = q[6], h = q[7];
            for (int k = 0; k < 3; ++k) {
                float base = q[k] - q[3 + k] * h;
                b.mn[k] = std::fmin(q[k], base) - r;
                b.mx[k] = std::fmax(q[k], base) + r;
            }
            break;
        }
        default:
            break;
    }
    return b;
}

class Builder {
public:
    explicit Builder(std::vector<Box> boxes) : boxes_(std::move(boxes)) {
        storage_.resize(boxes_.size());
        for (size_t k = 0; k < storage_.size(); ++k) storage_[k] = (int)k;
    }

    void build(std::vector<pgpu_bvh_node>& out, int& depth) {
        out.clear();
        out.reserve(storage_.empty() ? 0 : 2 * storage_.size() - 1);
        depth_ = 0;
        if (!storage_.empty()) build_range(0, (int)storage_.size(), out, 1);
        depth = depth_;
    }

private:
    float key2(int prim, int axis) const {   // centroid sum, as median_split compares
        return boxes_[prim].mn[axis] + boxes_[prim].mx[axis];
    }
    int bucket(int prim, int axis, float lo, float hi) const {
        const Box& pb = boxes_[prim];
        float center = (pb.mn[axis] + pb.mx[axis]) * 0.5f;
        int b = (int)((center - lo) / (hi - lo) * kBuckets);
        if (b < 0) b = 0;
        if (b >= kBuckets) b = kBuckets - 1;
        return b;
    }

    void build_range(int start, int end, std::vector<pgpu_bvh_node>& out, int level) {
        if (level > depth_) depth_ = level;
        Box box;
        for (int i = start; i < end; ++i) box = merge(box, boxes_[storage_[i]]);
        int me = (int)out.size();
        out.push_back(pgpu_bvh_node{});
        std::memcpy(out[me].bmin, box.mn, sizeof(box.mn));
        std::memcpy(out[me].bmax, box.mx, sizeof(box.mx));
        int count = end - start;
        if (count == 1) {
            out[me].left = -1;
            out[me].right = storage_[start];
            return;
        }
        int axis = longest_axis(box);
        if (count <= 4) median_split(start, end, axis);
        else sah_split(start, end, box, axis);
        int split = start + count / 2;
        if (count > 4) split = last_split_;
        out[me].left = me + 1;
        build_range(start, split, out, level + 1);
        out[me].right = (int)out.size();
        build_range(split, end, out, level + 1);
    }

    void median_split(int start, int end, int axis) {
        std::sort(storage_.begin() + start, storage_.begin() + end,
                  [&](int a, int b) { return key2(a, axis) < key2(b, axis); });
        last_split_ = start + (end - start) / 2;
    }

    void sah_split(int start, int end, const Box& parent, int axis) {
        struct Bucket {
            int count = 0;
            Box bounds;
        };
        Bucket buckets[kBuckets];
        float lo = parent.mn[axis];
        float hi = parent.mx[axis];
        if (hi <= lo) { median_split(start, end, axis); return; }
        for (int i = start; i < end; ++i) {
            int b = bucket(storage_[i], axis, lo, hi);
            buckets[b].count++;
            buckets[b].bounds = merge(buckets[b].bounds, boxes_[storage_[i]]);
        }
        Box prefix_b[kBuckets + 1];
        int prefix_c[kBuckets + 1] = {0};
        for (int i = 0; i < kBuckets; ++i) {
            prefix_b[i + 1] = merge(prefix_b[i], buckets[i].bounds);
            prefix_c[i + 1] = prefix_c[i] + buckets[i].count;
        }
        Box suffix_b[kBuckets + 1];
        int suffix_c[kBuckets + 1] = {0};
        for (int i = kBuckets - 1; i >= 0; --i) {
            suffix_b[i] = merge(suffix_b[i + 1], buckets[i].bounds);
            suffix_c[i] = suffix_c[i + 1] + buckets[i].count;
        }
        float best_cost = FLT_MAX;
        int best_bucket = -1;
        float sa_parent = surface_area(parent);
        for (int i = 1; i < kBuckets; ++i) {
            int nL = prefix_c[i], nR = suffix_c[i];
            if (nL == 0 || nR == 0) continue;
            float sa_l = surface_area(prefix_b[i]);
            float sa_r = surface_area(suffix_b[i]);
            float cost = 1.0f + (nL * sa_l + nR * sa_r) / (sa_parent > 0 ? sa_parent : 1.0f);
            if (cost < best_cost) {
                best_cost = cost;
                best_bucket = i;
            }
        }
        if (best_bucket < 0) { median_split(start, end, axis); return; }
        auto pivot = std::partition(storage_.begin() + start, storage_.begin() + end,
                                    [&](int p) { return bucket(p, axis, lo, hi) < best_bucket; });
        last_split_ = (int)(pivot - storage_.begin());
        if (last_split_ <= start || last_split_ >= end) median_split(start, end, axis);
    }

    static constexpr int kBuckets = 12;
    std::vector<Box> boxes_;
    std::vector<int> storage_;
    int last_split_ = 0;
    int depth_ = 0;
};

}  // namespace

// Unified primitive list of a scene: explicit prims, then mesh triangles.
void unified_prims(const pgpu_scene& s, std::vector<pgpu_prim>& out) {
    out.clear();
    out.reserve((size_t)s.n_prims + (size_t)std::max(0, s.n_mesh_triangles));
    for (int k = 0; k < s.n_prims; ++k) out.push_back(s.prims[k]);
    for (int k = 0; k < s.n_mesh_triangles; ++k) {
        pgpu_prim p{};
        p.type = PGPU_PRIM_TRIANGLE;
        p.material = s.mesh_materials ? s.mesh_materials[k] : 0;
        for (int v = 0; v < 3; ++v) {
            int idx = s.mesh_indices[3 * k + v];
            for (int c = 0; c < 3; ++c) p.p[3 * v + c] = s.mesh_vertices[3 * idx + c];
        }
        out.push_back(p);
    }
}

void build_bvh(const std::vector<pgpu_prim>& prims, std::vector<pgpu_bvh_node>& nodes,
               int& depth) {
    std::vector<Box> boxes(prims.size());
    for (size_t k = 0; k < prims.size(); ++k) boxes[k] = prim_box(prims[k]);
    Builder b(std::move(boxes));
    b.build(nodes, depth);
}

// Constructor arithmetic of each primitive (src/primitives.hpp): Vec3::
// normalized is sqrt of (x*x + y*y) + z*z, each component divided by it.
static void normalize3(const float* in, float* out) {
    float len = std::sqrt(in[0] * in[0] + in[1] * in[1] + in[2] * in[2]);
    for (int k = 0; k < 3; ++k) out[k] = (len > 1e-12f) ? in[k] / len : 0.0f;
}

int make_prim(int type, int material, const float* a, const float* b, const float* c, float s0,
              float s1, pgpu_prim* out) {
    std::memset(out, 0, sizeof(*out));
    out->type = type;
    out->material = material;
    float* p = out->p;
    switch (type) {
        case PGPU_PRIM_SPHERE:
        case PGPU_PRIM_CUBE:
            if (!a) return PGPU_ERR_INVALID_ARG;
            std::memcpy(p, a, 12);
            p[3] = s0;
            return PGPU_OK;
        case PGPU_PRIM_TRIANGLE:
            if (!a || !b || !c) return PGPU_ERR_INVALID_ARG;
            std::memcpy(p, a, 12);
            std::memcpy(p + 3, b, 12);
            std::memcpy(p + 6, c, 12);
            return PGPU_OK;
        case PGPU_PRIM_PLANE:
            if (!a || !b) return PGPU_ERR_INVALID_ARG;
            std::memcpy(p, a, 12);
            normalize3(b, p + 3);
            return PGPU_OK;
        case PGPU_PRIM_CYLINDER:
            if (!a || !b) return PGPU_ERR_INVALID_ARG;
            std::memcpy(p, a, 12);
            normalize3(b, p + 3);
            p[6] = s0;
            p[7] = s1 * 0.5f;
            return PGPU_OK;
        case PGPU_PRIM_CONE:
            if (!a || !b) return PGPU_ERR_INVALID_ARG;
            std::memcpy(p, a, 12);
            normalize3(b, p + 3);
            p[6] = s0;
            p[7] = s1;
            return PGPU_OK;
        default:
            return PGPU_ERR_INVALID_ARG;
    }
}

}  // namespace pgpu
