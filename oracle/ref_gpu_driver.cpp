// ref_gpu_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Runs the reference's own level-synchronous GPU path, GPU_SIMPLE::rcm
// (src/device/rcm_gpu.cu:400-494, compiled unchanged for sm_100a by
// oracle/Makefile `refgpu`), on a raw CSR from a given start node, so that
// it can be timed on the B200 beside this project's engine.  GPU_SIMPLE
// itself runs 5 warm-up and 20 timed reorders and prints their mean
// ("GPUSimple-RCM duration: X ms", rcm_gpu.cu:475); it orders a parent's
// children by (valence, node id), so its permutation can differ from the
// serial stable order on ties.
//
//   ref_gpu_simple <rp> <ci> <start> <outprefix>
// writes <outprefix>.perm (u32) and prints one line "JSON {...}".
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "Graph.h"
#include "rcm_gpu.h"

namespace {

std::vector<uint32_t> readU32(const char* path)
{
    std::ifstream f(path, std::ios::binary);
    if (!f)
        throw std::runtime_error(std::string("cannot open ") + path);
    f.seekg(0, std::ios::end);
    const size_t bytes = static_cast<size_t>(f.tellg());
    f.seekg(0);
    std::vector<uint32_t> v(bytes / 4);
    f.read(reinterpret_cast<char*>(v.data()), static_cast<std::streamsize>(v.size() * 4));
    return v;
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 5) {
        std::fprintf(stderr, "usage: ref_gpu_simple <rp> <ci> <start> <outprefix>\n");
        return 1;
    }
    try {
        const std::vector<uint32_t> rp = readU32(argv[1]), ci = readU32(argv[2]);
        Graph<float> g;
        const size_t n = rp.size() - 1;
        g.csr.alloc(n, n, ci.size());
        std::memcpy(g.csr.row_offsets.get(), rp.data(), rp.size() * 4);
        std::memcpy(g.csr.col_ids.get(), ci.data(), ci.size() * 4);
        for (size_t i = 0; i < ci.size(); ++i)
            g.csr.data[i] = 1.0f;
        g.alloc(n);
        std::ofstream csv("/dev/null");
        std::vector<unsigned> perm;
        std::stringstream cap;
        auto* old = std::cout.rdbuf(cap.rdbuf());
        GPU_SIMPLE::rcm(g, csv, perm, static_cast<unsigned>(std::atol(argv[3])));
        std::cout.rdbuf(old);
        const std::string s = cap.str();
        const size_t p = s.find("duration: ");
        const double ms = p == std::string::npos ? -1.0 : std::atof(s.c_str() + p + 10);
        std::ofstream o(std::string(argv[4]) + ".perm", std::ios::binary);
        o.write(reinterpret_cast<const char*>(perm.data()), static_cast<std::streamsize>(perm.size() * 4));
        std::printf("JSON {\"n\": %zu, \"nnz\": %zu, \"ms\": %.4f, \"placed\": %zu}\n", n, ci.size(), ms,
                    perm.size());
    } catch (std::exception& e) {
        std::printf("JSON {\"error\": \"%s\"}\n", e.what());
        return 3;
    }
    return 0;
}
