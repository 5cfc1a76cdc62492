"""Host-side parallel work of the scene upload (CPU only).

The upload validates, converts and collapses the scene on a persistent pool
of host threads (pencil_b200/csrc/host_pool.cpp) and collapses Pencil's
binary tree to 4-wide nodes on it (bvh_wide.cpp). A small C++ driver built
from those two sources checks that every task runs exactly once, that two
host threads may submit work at the same time, that a forked child gets a
working pool of its own, and that the pooled collapse of a 100k-sphere tree
(large enough to use the threads) gives byte-identical nodes on every call
and a tree in which every wide node is reachable from the root and every
leaf appears exactly once.
"""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
CSRC = ROOT / "pencil_b200" / "csrc"

DRIVER = r"""
#include "host_internal.h"
#include <atomic>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>
#include <sys/wait.h>
#include <unistd.h>
using namespace pgpu;

static int check_cover(int n) {
    std::vector<std::atomic<int>> hits(n);
    for (auto& h : hits) h = 0;
    host_run(n, [&](int t) { hits[t]++; });
    for (int t = 0; t < n; ++t)
        if (hits[t] != 1) return 1;
    return 0;
}

int main(int argc, char** argv) {
    if (host_threads() < 1) return 10;
    for (int n : {0, 1, 2, 7, 64, 1000})
        if (check_cover(n)) return 11;
    // two submitting threads
    std::atomic<int> bad{0};
    auto submit = [&] { for (int r = 0; r < 50; ++r) bad += check_cover(97); };
    std::thread a(submit), b(submit);
    a.join(); b.join();
    if (bad) return 12;
    // a forked child
    fflush(stdout);
    pid_t c = fork();
    if (c == 0) _exit(check_cover(333) ? 1 : 0);
    int st = 0;
    waitpid(c, &st, 0);
    if (!WIFEXITED(st) || WEXITSTATUS(st) != 0) return 13;
    // collapse of a large tree (pooled): two calls byte for byte, then the
    // structure of the result
    FILE* f = fopen(argv[1], "rb");
    if (!f) return 14;
    std::vector<pgpu_bvh_node> nodes;
    pgpu_bvh_node nd;
    while (fread(&nd, sizeof nd, 1, f) == 1) nodes.push_back(nd);
    fclose(f);
    std::vector<int> leaf_ref(nodes.size());
    int nl = 0;
    for (size_t k = 0; k < nodes.size(); ++k) leaf_ref[k] = nodes[k].left < 0 ? ~(nl++) : 0;
    const size_t cap = (nodes.size() / 2 + 1) * kWideNodeFloat4;
    std::vector<float4> o1(cap), o2(cap);
    WideScratch s1, s2;
    int st1 = 0, st2 = 0;
    const int n1 = collapse_wide(nodes.data(), (int)nodes.size(), leaf_ref, 64, o1.data(), s1, st1);
    const int n2 = collapse_wide(nodes.data(), (int)nodes.size(), leaf_ref, 64, o2.data(), s2, st2);
    if (n1 != n2 || st1 != st2) return 15;
    if (std::memcmp(o1.data(), o2.data(), (size_t)n1 * kWideNodeFloat4 * sizeof(float4))) return 16;
    std::vector<int> leaf_seen(nl, 0), node_seen(n1, 0);
    std::vector<int> todo{0};
    while (!todo.empty()) {
        const int w = todo.back();
        todo.pop_back();
        if (w < 0 || w >= n1 || node_seen[w]++) return 17;
        int refs[4];
        std::memcpy(refs, &o1[(size_t)w * kWideNodeFloat4 + 6], sizeof refs);
        for (int r : refs) {
            if (r >= 0) { todo.push_back(r); continue; }
            const int code = ~r;
            if ((code >> kLeafTypeShift) == kLeafNone) continue;
            const int slot = code & kLeafSlotMask;
            if (slot >= nl || leaf_seen[slot]++) return 18;
        }
    }
    for (int v : node_seen) if (v != 1) return 19;
    for (int v : leaf_seen) if (v != 1) return 20;
    printf("%d %d\n", n1, st1);
    return 0;
}
"""


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    if not shutil.which("g++"):
        pytest.skip("g++ not found")
    d = tmp_path_factory.mktemp("pool")
    src = d / "driver.cpp"
    src.write_text(DRIVER)
    exe = d / "driver"
    cmd = ["g++", "-O2", "-std=c++17", "-ffp-contract=off", f"-I{CSRC}",
           "-I/usr/local/cuda/include", str(src), str(CSRC / "host_pool.cpp"),
           str(CSRC / "bvh_wide.cpp"), "-o", str(exe), "-lpthread"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return d, exe


def test_pool_and_pooled_collapse(driver):
    from pencil_b200 import workloads as W
    d, exe = driver
    nodes, _ = W.sphere_cloud().scene.build_bvh()     # 100k spheres: pooled collapse
    path = d / "nodes.bin"
    nodes.tofile(path)
    proc = subprocess.run([str(exe), str(path)], capture_output=True, text=True, timeout=120)
    assert proc.returncode == 0, (proc.returncode, proc.stderr)
    n_wide, stack = (int(x) for x in proc.stdout.split())
    n_int = int((np.asarray(nodes["left"]) >= 0).sum())
    assert (n_int + 2) // 3 <= n_wide <= n_int
    assert 0 < stack <= 64
