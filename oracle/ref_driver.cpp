// ref_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A small command-line driver that links the reference's own, unmodified CPU
// sources (rcm_cpu.cpp, batchWorker.cpp, simple_peripheral.cpp, CSR.cpp,
// COO.cpp and main.cpp with its main() renamed) so that the oracle and the
// golden fixtures can be pinned on the reference itself, and so that the
// reference's CPU path can be timed as the CPU baseline.  Built by
// oracle/Makefile into oracle/_ref/ (never committed).
//
// Commands (all integers little-endian u32 files):
//   ref_rcm load <file.mtx> <outprefix>
//       Graph<float>::load (Graph.h:266-332; writes its .hicsr caches next to
//       the input, so callers pass a copy in a scratch directory), dumps the
//       loaded CSR to <outprefix>.rp / <outprefix>.ci, then runs `analyze`.
//   ref_rcm csr <rp> <ci> <outprefix> [start]
//       Same analysis on a raw CSR taken as is (no prepareRCM).
//   ref_rcm store64|store32 <rp> <ci> <vals> <out.mtx>
//       CSR<double|float> with the given values -> convert(COO, CSR)
//       (CSR.cpp:210-231) -> storeMTX (COO.cpp:213-251).
//   ref_rcm hicsr32|hicsr64 <file.hicsr> <outprefix>
//       loadCSR<float|double> (CSR.cpp:119-151), dumped to <outprefix>.rp /
//       .ci / .v.
//   ref_rcm time <rp> <ci> <threads> <steps>
//       Times <steps> reorders: findPeripheral + RealCPU::rcm<true> with
//       <threads> workers (1 = the serial rcm_seq path, else CPU_BATCH with
//       batch size 512 as main.cpp:456-483 runs it).
//   ref_rcm timebatch <pack> <threads> <outprefix> [reps]
//       A stream of independent matrices (pack: u64 count, then per matrix
//       u64 n, u64 nnz, row_ptr[n+1], col_idx[nnz]) reordered by <threads>
//       host threads, each taking the next matrix: findPeripheral
//       (simple_peripheral.cpp:92-141, thread-safe: its BFS state is
//       thread_local) + one rcm_seq<true> (rcm_cpu.cpp:57-104, the serial
//       stable path RealCPU::rcm<true> times).  The graphs are filled before
//       the clock starts.  Prints the wall time of the pool; writes per
//       matrix the start node and an FNV-1a hash of the permutation (CM
//       order) to <outprefix>.hash (u32 start, u32 pad, u64 hash) and the
//       permutations themselves, one after the other, to <outprefix>.perm.
//       With [reps], the pool runs that many times over the loaded graphs,
//       one JSON line each; the last repetition's permutations are kept.
// `analyze` = findPeripheral (simple_peripheral.cpp:92) unless a start is
// given, RealCPU::rcm<true>(.., 1, 1) (rcm_cpu.cpp:110), computeBandwidth /
// checkBandwidth / maxValency / checkPermutation (main.cpp:94-226); it writes
// the permutation to <outprefix>.perm and prints one line "JSON {...}".
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "Graph.h"
#include "rcm_cpu.h"
#include "simple_peripheral.h"

// The reference's serial stable pass (rcm_cpu.cpp:57-104); rcm_cpu.cpp
// instantiates it for float (through RealCPU::rcm<true>) as a weak symbol.
namespace RealCPU {
template <bool STABLE, typename T>
void rcm_seq(Graph<T>& graph, std::vector<unsigned>& permutation, unsigned start_node);
}

// main.cpp (compiled with -Dmain=pbrcm_reference_cli_main)
int computeBandwidth(const Graph<float>& graph, std::vector<uint32_t>& permutation);
int checkBandwidth(const Graph<float>& graph);
int maxValency(const Graph<float>& graph);
int checkPermutation(const std::vector<uint32_t>& permutation);

namespace {

struct NullBuf : std::streambuf {
    int overflow(int c) override { return c; }
};

std::vector<uint32_t> readU32(const char* path)
{
    std::ifstream f(path, std::ios::binary);
    if (!f)
        throw std::runtime_error(std::string("cannot open ") + path);
    f.seekg(0, std::ios::end);
    size_t bytes = static_cast<size_t>(f.tellg());
    f.seekg(0);
    std::vector<uint32_t> v(bytes / 4);
    f.read(reinterpret_cast<char*>(v.data()), static_cast<std::streamsize>(v.size() * 4));
    return v;
}

void writeU32(const std::string& path, const uint32_t* p, size_t n)
{
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(p), static_cast<std::streamsize>(n * 4));
}

void fillGraph(Graph<float>& g, const std::vector<uint32_t>& rp, const std::vector<uint32_t>& ci)
{
    size_t n = rp.size() - 1;
    g.csr.alloc(n, n, ci.size());
    std::memcpy(g.csr.row_offsets.get(), rp.data(), rp.size() * 4);
    std::memcpy(g.csr.col_ids.get(), ci.data(), ci.size() * 4);
    for (size_t i = 0; i < ci.size(); ++i)
        g.csr.data[i] = 1.0f;
    g.alloc(n);
}

// Runs findPeripheral with std::cout captured, returning (start, passes, ecc)
// parsed from its "Peripheral<iters, start, end, lastdist>" line
// (simple_peripheral.cpp:132-133).
void peripheral(const Graph<float>& g, uint32_t& start, uint32_t& passes, uint32_t& ecc, double& ms)
{
    NullBuf nb;
    std::ostream null_out(&nb);
    std::stringstream cap;
    auto* old = std::cout.rdbuf(cap.rdbuf());
    auto t0 = std::chrono::high_resolution_clock::now();
    start = SimplePeripheral::findPeripheral(g, null_out, false);
    auto t1 = std::chrono::high_resolution_clock::now();
    std::cout.rdbuf(old);
    ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    std::string s = cap.str();
    size_t p = s.find("Peripheral<");
    passes = ecc = 0;
    if (p != std::string::npos) {
        unsigned a = 0, b = 0, c = 0, d = 0;
        if (std::sscanf(s.c_str() + p, "Peripheral<%u, %u, %u, %u>", &a, &b, &c, &d) == 4) {
            passes = a;
            ecc = d;
        }
    }
}

// Runs RealCPU::rcm with std::cout captured; returns the printed mean (ms) of
// its 25 internal repetitions (rcm_cpu.cpp:138-140).
double rcmTimed(Graph<float>& g, std::vector<unsigned>& perm, uint32_t start, unsigned threads)
{
    NullBuf nb;
    std::ostream null_out(&nb);
    std::stringstream cap;
    auto* old = std::cout.rdbuf(cap.rdbuf());
    if (threads <= 1)
        RealCPU::rcm<true>(g, null_out, perm, start, 1, 1);
    else
        RealCPU::rcm<true>(g, null_out, perm, start, threads, 512);
    std::cout.rdbuf(old);
    std::string s = cap.str();
    size_t p = s.find("duration: ");
    double ms = -1.0;
    if (p != std::string::npos)
        ms = std::atof(s.c_str() + p + 10);
    return ms;
}

// One pass of the thread pool over every graph: findPeripheral + one
// rcm_seq<true> per matrix, each thread taking the next index.  Returns the
// wall time (ms); fills starts / hashes and the threads' summed busy time.
double runPool(std::vector<std::unique_ptr<Graph<float>>>& graphs, unsigned threads, std::vector<uint32_t>& starts,
               std::vector<uint64_t>& hashes, std::vector<std::vector<unsigned>>* keep, double& busy, int& failed)
{
    const uint64_t count = graphs.size();
    std::vector<double> busy_ms(threads, 0.0);
    std::atomic<uint64_t> next{0};
    std::atomic<int> nfail{0};
    // findPeripheral prints one line per call: std::cout goes nowhere while
    // the pool runs (the buffer is swapped before any thread starts)
    NullBuf nb;
    auto* old = std::cout.rdbuf(&nb);
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (unsigned w = 0; w < threads; ++w) {
        pool.emplace_back([&, w] {
            NullBuf nb2;
            std::ostream null_out(&nb2);
            std::vector<unsigned> perm;
            while (true) {
                const uint64_t i = next.fetch_add(1);
                if (i >= count)
                    break;
                auto a = std::chrono::steady_clock::now();
                try {
                    Graph<float>& g = *graphs[i];
                    const uint32_t start = SimplePeripheral::findPeripheral(g, null_out, false);
                    RealCPU::rcm_seq<true>(g, perm, start);
                    uint64_t h = 1469598103934665603ull;
                    for (unsigned v : perm)
                        h = (h ^ v) * 1099511628211ull;
                    starts[i] = start;
                    hashes[i] = h;
                    if (keep)
                        std::swap((*keep)[i], perm);  // no copy; rcm_seq re-reserves
                } catch (...) {
                    nfail.fetch_add(1);
                }
                busy_ms[w] += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - a).count();
            }
        });
    }
    for (auto& t : pool)
        t.join();
    const double wall = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    std::cout.rdbuf(old);
    busy = 0.0;
    for (double b : busy_ms)
        busy += b;
    failed = nfail.load();
    return wall;
}

// timebatch: see the header.
int timeBatch(const char* pack, unsigned threads, const std::string& outprefix, int reps)
{
    std::ifstream f(pack, std::ios::binary);
    if (!f)
        throw std::runtime_error(std::string("cannot open ") + pack);
    uint64_t count = 0;
    f.read(reinterpret_cast<char*>(&count), 8);
    std::vector<std::unique_ptr<Graph<float>>> graphs;
    uint64_t sum_nnz = 0;
    for (uint64_t i = 0; i < count; ++i) {
        uint64_t hdr[2];
        f.read(reinterpret_cast<char*>(hdr), 16);
        std::vector<uint32_t> rp(hdr[0] + 1), ci(hdr[1]);
        f.read(reinterpret_cast<char*>(rp.data()), static_cast<std::streamsize>(rp.size() * 4));
        f.read(reinterpret_cast<char*>(ci.data()), static_cast<std::streamsize>(ci.size() * 4));
        if (!f)
            throw std::runtime_error("truncated pack file");
        graphs.emplace_back(new Graph<float>());
        fillGraph(*graphs.back(), rp, ci);
        sum_nnz += hdr[1];
    }
    threads = std::max(1u, threads);
    std::vector<uint32_t> starts(count, 0);
    std::vector<uint64_t> hashes(count, 0);
    std::vector<std::vector<unsigned>> perms(count);
    int failed_total = 0;
    for (int rep = 0; rep < std::max(1, reps); ++rep) {
        double busy = 0.0;
        int failed = 0;
        // the last repetition keeps its permutations
        const bool last = rep + 1 == std::max(1, reps);
        const double wall = runPool(graphs, threads, starts, hashes, last ? &perms : nullptr, busy, failed);
        failed_total += failed;
        std::printf("JSON {\"rep\": %d, \"count\": %llu, \"sum_nnz\": %llu, \"threads\": %u, \"wall_ms\": %.4f, "
                    "\"busy_ms\": %.4f, \"failed\": %d}\n",
                    rep, (unsigned long long)count, (unsigned long long)sum_nnz, threads, wall, busy, failed);
        std::fflush(stdout);
    }
    std::ofstream o(outprefix + ".hash", std::ios::binary);
    std::ofstream op(outprefix + ".perm", std::ios::binary);
    for (uint64_t i = 0; i < count; ++i) {
        const uint32_t w2[2] = {starts[i], 0u};
        o.write(reinterpret_cast<const char*>(w2), 8);
        o.write(reinterpret_cast<const char*>(&hashes[i]), 8);
        op.write(reinterpret_cast<const char*>(perms[i].data()), static_cast<std::streamsize>(perms[i].size() * 4));
    }
    return failed_total ? 4 : 0;
}

int analyze(Graph<float>& g, const std::string& outprefix, long forced_start)
{
    uint32_t start = 0, passes = 0, ecc = 0;
    double pms = 0.0;
    if (forced_start >= 0)
        start = static_cast<uint32_t>(forced_start);
    else
        peripheral(g, start, passes, ecc, pms);
    std::vector<unsigned> perm;
    double rms = rcmTimed(g, perm, start, 1);
    writeU32(outprefix + ".perm", perm.data(), perm.size());
    std::vector<uint32_t> p32(perm.begin(), perm.end());
    int bw = computeBandwidth(g, p32);
    int bw0 = checkBandwidth(g);
    int mv = maxValency(g);
    int ok = checkPermutation(p32);
    std::printf("JSON {\"n\": %zu, \"nnz\": %zu, \"start\": %u, \"peripheral_passes\": %u, "
                "\"ecc\": %u, \"bandwidth\": %d, \"initial_bandwidth\": %d, \"max_valency\": %d, "
                "\"check_permutation\": %d, \"placed\": %zu, \"peripheral_ms\": %.4f, \"rcm_ms\": %.4f}\n",
                g.csr.rows, g.csr.nnz, start, passes, ecc, bw, bw0, mv, ok, perm.size(), pms, rms);
    return 0;
}

}  // namespace

template <typename T>
int dumpHicsr(const char* file, const std::string& out)
{
    CSR<T> csr = loadCSR<T>(file);
    writeU32(out + ".rp", csr.row_offsets.get(), csr.rows + 1);
    writeU32(out + ".ci", csr.col_ids.get(), csr.nnz);
    std::ofstream fv(out + ".v", std::ios::binary);
    fv.write(reinterpret_cast<const char*>(csr.data.get()), static_cast<std::streamsize>(csr.nnz * sizeof(T)));
    return 0;
}

template <typename T>
int storeAs(const std::vector<uint32_t>& rp, const std::vector<uint32_t>& ci, std::ifstream& fv, const char* out)
{
    const size_t n = rp.size() - 1;
    CSR<T> csr;
    csr.alloc(n, n, ci.size());
    std::memcpy(csr.row_offsets.get(), rp.data(), rp.size() * 4);
    std::memcpy(csr.col_ids.get(), ci.data(), ci.size() * 4);
    fv.read(reinterpret_cast<char*>(csr.data.get()), static_cast<std::streamsize>(ci.size() * sizeof(T)));
    COO<T> coo;
    convert(coo, csr);
    storeMTX(coo, out);
    return 0;
}

int main(int argc, char** argv)
{
    try {
        if (argc >= 4 && std::strcmp(argv[1], "load") == 0) {
            Graph<float> g;
            {
                std::stringstream cap;
                auto* old = std::cout.rdbuf(cap.rdbuf());
                int st = g.load(argv[2]);
                std::cout.rdbuf(old);
                if (st != 0) {
                    std::printf("JSON {\"error\": \"load failed\", \"status\": %d}\n", st);
                    return 2;
                }
            }
            std::string out = argv[3];
            writeU32(out + ".rp", g.csr.row_offsets.get(), g.csr.rows + 1);
            writeU32(out + ".ci", g.csr.col_ids.get(), g.csr.nnz);
            return analyze(g, out, argc >= 5 ? std::atol(argv[4]) : -1);
        }
        if (argc >= 5 && std::strcmp(argv[1], "csr") == 0) {
            Graph<float> g;
            fillGraph(g, readU32(argv[2]), readU32(argv[3]));
            return analyze(g, argv[4], argc >= 6 ? std::atol(argv[5]) : -1);
        }
        if (argc >= 6 && (std::strcmp(argv[1], "store64") == 0 || std::strcmp(argv[1], "store32") == 0)) {
            const std::vector<uint32_t> rp = readU32(argv[2]), ci = readU32(argv[3]);
            std::ifstream fv(argv[4], std::ios::binary);
            if (std::strcmp(argv[1], "store64") == 0)
                return storeAs<double>(rp, ci, fv, argv[5]);
            return storeAs<float>(rp, ci, fv, argv[5]);
        }
        if (argc >= 4 && (std::strcmp(argv[1], "hicsr32") == 0 || std::strcmp(argv[1], "hicsr64") == 0)) {
            if (std::strcmp(argv[1], "hicsr64") == 0)
                return dumpHicsr<double>(argv[2], argv[3]);
            return dumpHicsr<float>(argv[2], argv[3]);
        }
        if (argc >= 6 && std::strcmp(argv[1], "time") == 0) {
            Graph<float> g;
            fillGraph(g, readU32(argv[2]), readU32(argv[3]));
            unsigned threads = static_cast<unsigned>(std::atoi(argv[4]));
            int steps = std::atoi(argv[5]);
            for (int s = 0; s < steps; ++s) {
                uint32_t start, passes, ecc;
                double pms;
                peripheral(g, start, passes, ecc, pms);
                std::vector<unsigned> perm;
                double rms = rcmTimed(g, perm, start, threads);
                std::printf("JSON {\"step\": %d, \"threads\": %u, \"start\": %u, \"peripheral_ms\": %.4f, "
                            "\"rcm_ms\": %.4f, \"reorder_ms\": %.4f}\n",
                            s, threads, start, pms, rms, pms + rms);
                std::fflush(stdout);
            }
            return 0;
        }
        if (argc >= 5 && std::strcmp(argv[1], "timebatch") == 0)
            return timeBatch(argv[2], static_cast<unsigned>(std::atoi(argv[3])), argv[4],
                             argc >= 6 ? std::atoi(argv[5]) : 1);
    } catch (std::exception& e) {
        std::printf("JSON {\"error\": \"%s\"}\n", e.what());
        return 3;
    }
    std::fprintf(stderr, "usage: ref_rcm load <mtx> <outprefix> [start] | csr <rp> <ci> <outprefix> [start] | "
                         "time <rp> <ci> <threads> <steps> | timebatch <pack> <threads> <outprefix> [reps]\n");
    return 1;
}
