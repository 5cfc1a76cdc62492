// bvh_wide.cpp - wide nodes collapsed from Pencil's binary tree.
//
// The kernels traverse a wide tree (kWideWidth children per node, 4 or 8)
// made from the uploaded binary tree (src/bvh.hpp:54-192 builds it): every
// wide node lists up to kWideWidth nodes of the binary tree as its children,
// with their boxes copied bit for
// bit. The boxes a ray is tested against are therefore Pencil's boxes; a
// wide node only skips the boxes of the intermediate binary nodes, and since
// a child's box lies inside its parent's and the slab test's rounding is
// monotone in the plane coordinates, a ray that fails a parent box fails its
// children too: the leaves reached are the same.
//
// Collapse: a wide node starts from the two children of a binary interior
// node and repeatedly replaces its interior child of largest surface area by
// that child's two children, keeping left-to-right order, until it has
// kWideWidth children or only leaves. Wide nodes are numbered in DFS
// pre-order.
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

constexpr int W = kWideWidth;
constexpr int G = kWideGroups;

// The node's rows (scene_layout.h): per axis the lo planes of children
// 4g..4g+3 at row a*G + g, the hi planes at (3 + a)*G + g, refs at 6G + g.
void write_node(float4* q, const float (&lo)[3][W], const float (&hi)[3][W], const int (&ref)[W]) {
    for (int a = 0; a < 3; ++a)
        for (int g = 0; g < G; ++g) {
            const int k = 4 * g;
            q[a * G + g] = make_float4(lo[a][k], lo[a][k + 1], lo[a][k + 2], lo[a][k + 3]);
            q[(3 + a) * G + g] = make_float4(hi[a][k], hi[a][k + 1], hi[a][k + 2], hi[a][k + 3]);
        }
    static_assert(sizeof(ref) == G * sizeof(float4), "the refs fill G float4");
    std::memcpy(&q[6 * G], ref, sizeof(ref));
    for (int r = 7 * G; r < 8 * G; ++r) q[r] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

// Expands the children of a wide node rooted at binary interior node b:
// the interior child of largest surface area is replaced by its two
// children while there are fewer than `cap`; returns the child count.
int expand(const pgpu_bvh_node* nodes, int b, int cap, int (&ch)[W]) {
    ch[0] = nodes[b].left;
    ch[1] = nodes[b].right;
    int n = 2;
    while (n < cap) {
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
    return n;
}

// Copies each subtree's block into `out` at base[t], its interior refs
// (local indices) shifted by base[t].
void parallel_relocate(float4* out, const std::vector<std::vector<float4>>& local,
                       const std::vector<int>& count, const std::vector<int>& base) {
    host_run((int)count.size(), [&](int t) {
        const int cnt = count[t];
        float4* dst = out + (size_t)base[t] * kWideNodeFloat4;
        std::copy_n(local[t].begin(), (size_t)cnt * kWideNodeFloat4, dst);
        for (int w = 0; w < cnt; ++w) {
            int* refs = reinterpret_cast<int*>(dst + (size_t)w * kWideNodeFloat4 + 6 * G);
            for (int k = 0; k < W; ++k)
                if (refs[k] >= 0) refs[k] += base[t];
        }
    });
}

struct Collapser {
    const pgpu_bvh_node* nodes;
    const std::vector<int>& leaf_ref;
    int cap;                 // children per node in this collapse
    std::vector<float4>& out;
    int n_wide = 0;

    // Builds the wide node for binary interior node b; returns its index and
    // the stack entries a traversal below it can hold (`need`).
    int build(int b, int& need) {
        const int w = n_wide++;
        if (out.size() < (size_t)n_wide * kWideNodeFloat4)
            out.resize(std::max(out.size() * 2, (size_t)n_wide * kWideNodeFloat4));
        int ch[W];
        const int n = expand(nodes, b, cap, ch);
        float lo[3][W], hi[3][W];
        int ref[W];
        int interior = 0, deepest = 0;
        for (int k = 0; k < W; ++k) {
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
        write_node(out.data() + (size_t)w * kWideNodeFloat4, lo, hi, ref);
        return w;
    }
};

// The top of the tree is collapsed on this thread until there are enough
// independent subtrees; each subtree is then collapsed on its own thread into
// a local array and appended. Wide nodes need no particular numbering (the
// kernels only follow refs), so the top comes first and each subtree's nodes
// follow as one block in DFS pre-order.
int collapse_parallel(const pgpu_bvh_node* nodes, const std::vector<int>& leaf_ref,
                      int cap, int threads, float4* out, WideScratch& scratch,
                      int& stack_need) {
    const int T = threads;
    // top: breadth-first over wide-node roots until enough subtrees wait
    struct Pending { int binary; int parent; int child; };   // ref slot to patch
    std::vector<Pending> todo{{0, -1, -1}};
    std::vector<float4> top;
    size_t head = 0;
    const size_t want = T > 1 ? (size_t)T * 8 : 0;
    std::vector<std::vector<int>> top_kids;  // per top node: its subtrees' todo indices
    int n_top = 0;
    while (head < todo.size() && todo.size() - head < want) {
        const Pending p = todo[head++];
        // collapse one node without recursing into interior children
        int ch[W];
        const int n = expand(nodes, p.binary, cap, ch);
        const int w = n_top++;
        top.resize((size_t)n_top * kWideNodeFloat4);
        top_kids.emplace_back();
        float lo[3][W], hi[3][W];
        int ref[W];
        for (int k = 0; k < W; ++k) {
            if (k >= n) {
                for (int a = 0; a < 3; ++a) { lo[a][k] = INFINITY; hi[a][k] = -INFINITY; }
                ref[k] = ~(kLeafNone << kLeafTypeShift);
                continue;
            }
            const pgpu_bvh_node& c = nodes[ch[k]];
            for (int a = 0; a < 3; ++a) { lo[a][k] = c.bmin[a]; hi[a][k] = c.bmax[a]; }
            if (c.left < 0) {
                ref[k] = leaf_ref[ch[k]];
            } else {
                ref[k] = -1;                 // patched below
                top_kids.back().push_back((int)todo.size());
                todo.push_back({ch[k], w, k});
            }
        }
        write_node(top.data() + (size_t)w * kWideNodeFloat4, lo, hi, ref);
    }
    // remaining subtrees in parallel
    const int n_tasks = (int)(todo.size() - head);
    std::vector<std::vector<float4>>& local = scratch.local;
    if ((int)local.size() < n_tasks) local.resize(n_tasks);
    std::vector<int> local_n(n_tasks, 0), local_need(n_tasks, 0);
    auto run = [&](int t) {
        Collapser c{nodes, leaf_ref, cap, local[t]};
        c.build(todo[head + t].binary, local_need[t]);
        local_n[t] = c.n_wide;
    };
    if (T > 1) {
        host_run(n_tasks, run);
    } else {
        for (int t = 0; t < n_tasks; ++t) run(t);
    }
    // layout: top nodes, then each task's block
    std::vector<int> base(n_tasks);
    int total = n_top;
    for (int t = 0; t < n_tasks; ++t) { base[t] = total; total += local_n[t]; }
    std::copy(top.begin(), top.end(), out);
    // which todo entry is which task: entries [head, end) are tasks; entries
    // before head became top nodes 0, 1, ... in order
    std::vector<int> wide_of_todo(todo.size());
    for (size_t k = 0; k < head; ++k) wide_of_todo[k] = (int)k;
    for (int t = 0; t < n_tasks; ++t) wide_of_todo[head + t] = base[t];
    for (size_t k = 1; k < todo.size(); ++k) {
        const Pending& p = todo[k];
        int* refs = reinterpret_cast<int*>(out + (size_t)p.parent * kWideNodeFloat4 + 6 * G);
        refs[p.child] = wide_of_todo[k];
    }
    parallel_relocate(out, local, local_n, base);
    // stack need: tasks' own, then the top nodes bottom-up (children of a top
    // node come later in todo, so a reverse sweep sees them first)
    std::vector<int> need_of_todo(todo.size(), 0);
    for (int t = 0; t < n_tasks; ++t) need_of_todo[head + t] = local_need[t];
    for (int w = n_top - 1; w >= 0; --w) {
        int interior = 0, deepest = 0;
        for (int k : top_kids[w]) { ++interior; deepest = std::max(deepest, need_of_todo[k]); }
        need_of_todo[w] = std::max(0, interior - 1) + deepest;
    }
    stack_need = need_of_todo[0];
    return total;
}

}  // namespace

int collapse_wide(const pgpu_bvh_node* nodes, int n_nodes, const std::vector<int>& leaf_ref,
                  int max_stack, float4* out, WideScratch& scratch, int& stack_need) {
    stack_need = 0;
    if (n_nodes == 0 || nodes[0].left < 0) return 0;
    // a full binary tree of n_nodes nodes has (n_nodes - 1) / 2 interior ones
    const int n_interior = (n_nodes - 1) / 2;
    // greedy collapse; if a pathological tree would need a deeper stack than
    // the kernels hold, fewer children per node: 4, then two (the binary
    // tree's own bound). Threads only pay off for large trees.
    const int threads = n_interior < 16384 ? 1 : host_threads();
    int n_wide = 0;
    const int caps[3] = {W, 4, 2};
    for (int pass = 0; pass < 3; ++pass) {
        if (pass > 0 && caps[pass] >= caps[pass - 1]) continue;
        n_wide = collapse_parallel(nodes, leaf_ref, caps[pass], threads, out, scratch, stack_need);
        if (stack_need <= max_stack) break;
    }
    return n_wide;
}

}  // namespace pgpu
