// scene_layout.h - device-resident scene layout shared by the host uploader
// and the kernels.
//
// HBM layout of one uploaded scene (all arrays 16-byte aligned):
//
//   nodes   float4[4 * n_interior]  child-pair BVH: interior node i holds the
//                                   boxes of both children and their refs,
//                                   in the DFS pre-order of Pencil's tree
//                                   (src/bvh.hpp:74-104):
//             [4i+0] = (L.min.x, L.min.y, L.min.z, L.max.x)
//             [4i+1] = (L.max.y, L.max.z, R.min.x, R.min.y)
//             [4i+2] = (R.min.z, R.max.x, R.max.y, R.max.z)
//             [4i+3] = (ref L, ref R, -, -)            (int bits)
//           ref >= 0: interior node index; ref < 0: leaf, ~ref = type<<28 | slot
//   wide    float4[kWideNodeFloat4 * n_wide]
//                                   W-wide nodes (W = kWideWidth, 4 or 8)
//                                   collapsed from the same tree
//                                   (bvh_wide.cpp), used by both engines;
//                                   with G = W / 4 float4 per row of W floats:
//             [(a    )*G + g] = min of axis a (x, y, z) of children 4g..4g+3
//             [(3 + a)*G + g] = max of axis a of the same children
//             [6G + g]        = refs of those children (int bits; a missing
//                               child has an empty box and a leaf ref of type
//                               LEAF_NONE)
//             [7G .. 8G)      = unused
//   geo_a   float4[n_leaves]        leaf geometry in DFS leaf order (slot):
//             sphere   (center.xyz, radius)
//             triangle (v0.xyz, face normal x)
//             cube     (center.xyz, half)
//             plane    (point.xyz, -)
//             cylinder (center.xyz, radius)
//             cone     (apex.xyz, radius)
//   geo_b   float4[n_leaves]        second word where needed (zero elsewhere):
//             triangle (v1 - v0, face normal y)
//             plane    (normal.xyz, -)
//             cylinder (axis.xyz, half_height)
//             cone     (axis.xyz, height)
//   geo_c   float4[n_leaves]        only in scenes with triangles:
//             triangle (v2 - v0, face normal z)
//           (a triangle's first vertex and edges sit in its slot, so its
//            test loads them at once instead of through an index word)
//   leaf_mat  int32[n_leaves]       material id per slot
//   leaf_prim int32[n_leaves]       caller's primitive index per slot
//   mats    DevMaterial[n_materials]
//   lights  DevLight[n_lights]
#pragma once

#include <stdint.h>
#include <vector_types.h>

#ifdef __CUDACC__
#define PGPU_HD __host__ __device__
#else
#define PGPU_HD
#endif

namespace pgpu {

enum LeafType : int {
    LEAF_SPHERE = 0,
    LEAF_TRIANGLE = 1,
    LEAF_CUBE = 2,
    LEAF_PLANE = 3,
    LEAF_CYLINDER = 4,
    LEAF_CONE = 5,
    LEAF_NONE = 7,          // placeholder child of a wide node: never hit
};
constexpr int kLeafNone = LEAF_NONE;
// Children per wide node, fixed at compile time (4 or 8).
#ifndef PGPU_WIDE_WIDTH
#define PGPU_WIDE_WIDTH 4
#endif
constexpr int kWideWidth = PGPU_WIDE_WIDTH;
static_assert(kWideWidth == 4 || kWideWidth == 8, "wide nodes have 4 or 8 children");
constexpr int kWideGroups = kWideWidth / 4;          // float4 per row of child planes
constexpr int kWideNodeFloat4 = 8 * kWideGroups;     // 128 or 256 bytes

constexpr int kLeafTypeShift = 28;
constexpr int kLeafSlotMask = (1 << kLeafTypeShift) - 1;
constexpr int kMaxLeaves = 1 << kLeafTypeShift;

struct alignas(16) DevMaterial {
    float albedo[3];
    int kind;
    float emission[3];
    float reflectivity;
    float ior;
    float specular;
    float shininess;
    int area_emitter;      // 1: material of a quad light's emitter surface
    float specular_color[3];
    int pad;
};

struct alignas(16) DevLight {
    int kind;
    float pos[3];
    float intensity[3];
    float radius;
    int is_emissive;
    float edge_u[3];
    float edge_v[3];
    float area;            // quad: |edge_u x edge_v|
    float normal[3];       // quad: normalized(edge_u x edge_v)
};

// Everything a kernel needs to trace one scene; passed by value for
// single-scene launches and read from global memory for batched ones.
struct SceneView {
    const float4* nodes;
    const float4* wide;    // wide nodes (null when the root is a leaf)
    const float4* geo_a;
    const float4* geo_b;
    const float4* geo_c;   // null in scenes without triangles
    const int* leaf_mat;
    const int* leaf_prim;
    const DevMaterial* mats;
    const DevLight* lights;
    int n_lights;
    int n_leaves;
    int root_ref;          // ref of the root (interior 0, a leaf ref, or kEmpty)
    int has_quad_lights;
    float root_min[3];
    float root_max[3];
    float cam[21];         // origin, lower_left, horizontal, vertical, u, v, w
    float bg[3];
    float amb[3];
};

constexpr int kEmptyRoot = 0x7fffffff;

}  // namespace pgpu
