// bvh_wide.cpp - 4-wide nodes collapsed from Pencil's binary tree.
//
// The wavefront kernels traverse a 4-wide tree made from the uploaded binary
// tree (src/bvh.hpp:54-192 builds it): every wide node lists up to four
// nodes of the binary tree as its children, with their boxes copied bit for
// bit. The boxes a ray is tested against are therefore Pencil's boxes; a
// wide node only skips the boxes of the intermediate binary nodes, and since
// a child's box lies inside its parent's and the slab test's rounding is
// monotone in the plane coordinates, a ray that fails a parent box fails its
// children too: the leaves reached are the same.
//
// Collapse: a wide node starts from the two children of a binary interior
// node and repeatedly replaces its interior child of largest surface area by
// that child's two children, keeping left-to-right order, until it has four
// children or only leaves. Wide nodes are numbered in DFS pre-order.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include <vector_functions.h>

#include "host_internal.h"

namespace pgpu {

namespace {

float area(const pgpu_bvh_node& n) {
    const float dx = n.bmax[0] - n.bmin[0], dy = n.bmax[1] - n.bmin[1], dz = n.bmax[2] - n.bmin[2];
    return 2.0f * (dx * dy + dy * dz + dz * dx);
}

struct Collapser {
    const pgpu_bvh_node* nodes;
    const std::vector<int>& leaf_ref;
    bool expand;
    std::vector<float4>& out;
    int n_wide = 0;

    // Builds the wide node for binary interior node b; returns its index and
    // the stack entries a traversal below it can hold (`need`).
    int build(int b, int& need) {
        const int w = n_wide++;
        int ch[4] = {nodes[b].left, nodes[b].right, -1, -1};
        int n = 2;
        while (expand && n < 4) {
            int pick = -1;
            float best = -1.0f;
            for (int k = 0; k < n; ++k) {
                const pgpu_bvh_node& c = nodes[ch[k]];
                if (c.left >= 0 && area(c) > best) { best = area(c); pick = k; }
            }
            if (pick < 0) break;
            const int l = nodes[ch[pick]].left, r = nodes[ch[pick]].right;
            for (int k = n; k > pick + 1; --k) ch[k] = ch[k - 1];
            ch[pick] = l;
            ch[pick + 1] = r;
            ++n;
        }
        float lo[3][4], hi[3][4];
        int ref[4];
        int interior = 0, deepest = 0;
        for (int k = 0; k < 4; ++k) {
            if (k >= n) {
                // missing child: a box no finite ray enters and a leaf of no type
                for (int a = 0; a < 3; ++a) { lo[a][k] = INFINITY; hi[a][k] = -INFINITY; }
                ref[k] = ~(kLeafNone << kLeafTypeShift);
                continue;
            }
            const pgpu_bvh_node& c = nodes[ch[k]];
            for (int a = 0; a < 3; ++a) { lo[a][k] = c.bmin[a]; hi[a][k] = c.bmax[a]; }
            if (c.left < 0) {
                ref[k] = leaf_ref[ch[k]];
            } else {
                int sub = 0;
                ref[k] = build(ch[k], sub);
                deepest = std::max(deepest, sub);
                ++interior;
            }
        }
        // a step pushes every interior child it enters but the nearest
        need = std::max(0, interior - 1) + deepest;
        float4* q = out.data() + (size_t)w * kWideNodeFloat4;
        q[0] = make_float4(lo[0][0], lo[0][1], lo[0][2], lo[0][3]);
        q[1] = make_float4(lo[1][0], lo[1][1], lo[1][2], lo[1][3]);
        q[2] = make_float4(lo[2][0], lo[2][1], lo[2][2], lo[2][3]);
        q[3] = make_float4(hi[0][0], hi[0][1], hi[0][2], hi[0][3]);
        q[4] = make_float4(hi[1][0], hi[1][1], hi[1][2], hi[1][3]);
        q[5] = make_float4(hi[2][0], hi[2][1], hi[2][2], hi[2][3]);
        static_assert(sizeof(ref) == sizeof(float4), "four refs fill one float4");
        std::memcpy(&q[6], ref, sizeof(ref));
        q[7] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        return w;
    }
};

}  // namespace

int collapse_wide(const pgpu_bvh_node* nodes, int n_nodes, const std::vector<int>& leaf_ref,
                  int max_stack, std::vector<float4>& out, int& stack_need) {
    stack_need = 0;
    if (n_nodes == 0 || nodes[0].left < 0) return 0;
    // greedy collapse; if a pathological tree would need a deeper stack than
    // the kernels hold, two children per node (the binary tree's own bound)
    int n_wide = 0;
    int n_interior = 0;
    for (int k = 0; k < n_nodes; ++k) n_interior += nodes[k].left >= 0;
    // at most one wide node per binary interior node; `out` only grows, so a
    // reused vector is neither reallocated nor cleared
    if (out.size() < (size_t)n_interior * kWideNodeFloat4)
        out.resize((size_t)n_interior * kWideNodeFloat4);
    for (int pass = 0; pass < 2; ++pass) {
        Collapser c{nodes, leaf_ref, pass == 0, out};
        int need = 0;
        c.build(0, need);
        stack_need = need;
        n_wide = c.n_wide;
        if (need <= max_stack) break;
    }
    return n_wide;
}

}  // namespace pgpu
