// bridge_demo.cpp - Pencil's render path with the --gpu branch, built from the
// reference's own sources plus pencil_b200/bridge/pencil_gpu_bridge.hpp and
// linked against libpencil_gpu.so. TEST INFRASTRUCTURE: it shows the drop-in
// end to end (Pencil's parser -> its BVH -> the bridge -> the GPU core) and
// is built into oracle/_ref by oracle/Makefile.
//
//   pencil_gpu_demo <scene.pecl> <out.f32|-> [--pathtrace] [--width W]
//                   [--height H] [--samples n] [--depth d]
//
// Environment PENCIL_GPU_EXACT=1 selects Pencil's own random stream.
// Private members are opened with "#define private public" in this
// translation unit only, standing in for the one friend declaration per
// class (friend struct ::pencil_gpu::Access) that a Pencil build adds.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#define private public
#define protected public
#include "pecl_parser.hpp"
#include "renderer.hpp"
#undef private
#undef protected

#include "pencil_gpu_bridge.hpp"

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: pencil_gpu_demo scene.pecl out.f32 [options]\n");
        return 2;
    }
    pencil::ParsedScene ps;
    std::vector<pencil::ParseError> errs;
    if (!pencil::parse_pecl(argv[1], ps, errs)) {
        for (auto& e : errs) std::fprintf(stderr, "line %d: %s\n", e.line, e.what.c_str());
        return 3;
    }
    bool pathtrace = ps.enable_pathtrace;
    for (int i = 3; i < argc; ++i) {
        std::string s = argv[i];
        auto next = [&]() { return i + 1 < argc ? std::atoi(argv[++i]) : 0; };
        if (s == "--pathtrace") pathtrace = true;
        else if (s == "--width") { ps.width = next(); ps.aspect = (float)ps.width / ps.height; ps.finalize(); }
        else if (s == "--height") { ps.height = next(); ps.aspect = (float)ps.width / ps.height; ps.finalize(); }
        else if (s == "--samples") ps.samples = next();
        else if (s == "--depth") ps.depth = next();
    }
    pencil::RenderSettings rs;
    rs.width = ps.width;
    rs.height = ps.height;
    rs.samples = ps.samples;
    rs.max_depth = ps.depth;
    rs.pathtrace = pathtrace;
    rs.pathtrace_bounces = ps.depth;
    std::vector<pencil::Color> pixels;
    pencil::RenderStats stats;
    std::string why;
    auto t0 = std::chrono::steady_clock::now();
    int rc = pencil_gpu::render(ps, rs, pixels, &stats, why);
    auto t1 = std::chrono::steady_clock::now();
    if (rc != 0) {
        std::fprintf(stderr, "gpu render failed (%d): %s\n", rc, why.c_str());
        return 5;
    }
    if (std::strcmp(argv[2], "-") != 0) {
        FILE* f = std::fopen(argv[2], "wb");
        std::fwrite(pixels.data(), sizeof(pencil::Color), pixels.size(), f);
        std::fclose(f);
    }
    std::printf("{\"width\": %d, \"height\": %d, \"rays\": %llu, \"seconds\": %.6f}\n", rs.width,
                rs.height, (unsigned long long)stats.rays_traced,
                std::chrono::duration<double>(t1 - t0).count());
    return 0;
}
