// tune.cpp -- the autotuner of the batch and serving shapes (pbrcm_autotune)
// and the tuning cache.
//
// The reference fixes its batch shape at compile time
// (include/rcm_gpu_batch_params.h:36-46: BlockSizePow, MaxElementsPerThreadPow,
// QueueSize, Overalloc).  Here the shape is measured on the device, on a
// calibration batch the caller passes (a sample of its own workload):
//
//   1. the thread-group shape of the batch kernel (kPools 0..3: 1, 2, 4 or 8
//      groups per 512-thread CTA, each reordering its own matrix);
//   2. cluster teams for the biggest matrices: CTAs per cluster and how many
//      matrices get one;
//   3. the entry count from which a matrix may get a cluster team;
//   4. serving: the CTA shape of one-CTA requests (512, 256 or 128 threads) and
//      the cutoff above which a request runs on a cooperative team instead
//      (a replay of the batch through a session, all requests at once,
//      makespan compared).
//
// Coordinate descent: each step keeps the best setting found so far and
// tries its alternatives.  Every run's permutations are compared with the
// first run's; a difference (which would be an engine bug, never a tuning
// effect) stops the tuner with PBRCM_ERR_CHECK.  The result goes into the
// context and, on request, into a small text file keyed by the device's SM
// count and the library version, which pbrcm_context_create reads when the
// environment variable PBRCM_TUNING names it.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/pbrcm.h"
#include "context.h"
#include "kernels.h"
#include "types.h"

using namespace pbrcm;

namespace pbrcm {
extern const char* kVersion;
}

namespace {

constexpr const char* kTuningMagic = "pbrcm-tuning 1";

pbrcm_tuning from_context(const Context& C)
{
    pbrcm_tuning t;
    std::memset(&t, 0, sizeof(t));
    t.batch_pool = (uint32_t)C.batch_pool;
    t.batch_kernel = C.batch_solo_kernel ? 1u : 0u;
    t.cluster_size = (uint32_t)std::max(1, C.cluster_size);
    t.cluster_max = (uint32_t)std::max(0, C.cluster_max);
    t.cluster_nnz = (uint32_t)std::min<uint64_t>(C.cluster_nnz, 0xFFFFFFFFu);
    t.session_cutoff_n = C.session_cutoff_n;
    t.session_pool = (uint32_t)C.session_pool;
    t.session_team_nnz = C.session_team_nnz;
    t.session_cluster_max = (uint32_t)C.session_cluster_max;
    t.sms = (uint32_t)C.sms;
    t.source = C.tuned;
    return t;
}

bool valid(const pbrcm_tuning& t)
{
    return batch_pool_ok((int)t.batch_pool) && t.batch_kernel <= 1 && t.cluster_size >= 1 && t.cluster_size <= 16 && t.cluster_nnz >= 1 &&
           t.session_cutoff_n >= 1 && session_pool_ok((int)t.session_pool) && t.session_team_nnz >= 1 &&
           t.session_cluster_max <= 16 && t.session_cluster_max != 1;
}

void to_context(Context& C, const pbrcm_tuning& t)
{
    C.batch_pool = (int)t.batch_pool;
    C.batch_solo_kernel = t.batch_kernel != 0;
    C.cluster_size = (int)t.cluster_size;
    C.cluster_max = (int)t.cluster_max;
    C.cluster_nnz = t.cluster_nnz;
    C.session_cutoff_n = t.session_cutoff_n;
    C.session_pool = (int)t.session_pool;
    C.session_team_nnz = t.session_team_nnz;
    C.session_cluster_max = (int)t.session_cluster_max;
    // solo bounds of a cluster team follow the pool's CTA shape
    C.cluster_solo_parents = (uint32_t)kPools[C.batch_pool].block;
    C.cluster_solo_edges = (uint32_t)kPools[C.batch_pool].emax;
}

bool write_file(const char* path, const pbrcm_tuning& t)
{
    FILE* f = std::fopen(path, "w");
    if (!f)
        return false;
    std::fprintf(f,
                 "%s\nversion=%s\nsms=%u\nbatch_pool=%u\nbatch_kernel=%u\ncluster_size=%u\ncluster_max=%u\ncluster_nnz=%u\n"
                 "session_cutoff_n=%u\nsession_pool=%u\nsession_team_nnz=%u\nsession_cluster_max=%u\n"
                 "trials=%u\ndefault_ms=%.4f\nbest_ms=%.4f\n"
                 "session_default_ms=%.4f\nsession_best_ms=%.4f\n",
                 kTuningMagic, kVersion, t.sms, t.batch_pool, t.batch_kernel, t.cluster_size, t.cluster_max, t.cluster_nnz,
                 t.session_cutoff_n, t.session_pool, t.session_team_nnz, t.session_cluster_max, t.trials, t.default_ms, t.best_ms, t.session_default_ms,
                 t.session_best_ms);
    return std::fclose(f) == 0;
}

// Permutations of a device batch, copied to the host.
bool fetch_perms(const std::vector<pbrcm_matrix>& dm, std::vector<uint32_t>& out, cudaStream_t st)
{
    size_t total = 0;
    for (const auto& m : dm)
        total += m.n;
    out.resize(total);
    size_t off = 0;
    for (const auto& m : dm) {
        if (cudaMemcpyAsync(out.data() + off, m.perm_out, 4 * (size_t)m.n, cudaMemcpyDeviceToHost, st) != cudaSuccess)
            return false;
        off += m.n;
    }
    return cudaStreamSynchronize(st) == cudaSuccess;
}

}  // namespace

bool pbrcm::load_tuning_file(const char* path, int sms, pbrcm_tuning* out)
{
    FILE* f = path ? std::fopen(path, "r") : nullptr;
    if (!f)
        return false;
    char line[512];
    bool magic = false, version = false;
    pbrcm_tuning t;
    std::memset(&t, 0, sizeof(t));
    t.session_team_nnz = 1u << 20;  // keys a file may lack
    t.session_cluster_max = 16;
    while (std::fgets(line, sizeof(line), f)) {
        std::string s(line);
        while (!s.empty() && (s.back() == '\n' || s.back() == '\r'))
            s.pop_back();
        if (s == kTuningMagic) {
            magic = true;
            continue;
        }
        const size_t eq = s.find('=');
        if (eq == std::string::npos)
            continue;
        const std::string k = s.substr(0, eq), v = s.substr(eq + 1);
        const unsigned long u = std::strtoul(v.c_str(), nullptr, 10);
        if (k == "version")
            version = v == kVersion;
        else if (k == "sms")
            t.sms = (uint32_t)u;
        else if (k == "batch_pool")
            t.batch_pool = (uint32_t)u;
        else if (k == "batch_kernel")
            t.batch_kernel = (uint32_t)u;
        else if (k == "cluster_size")
            t.cluster_size = (uint32_t)u;
        else if (k == "cluster_max")
            t.cluster_max = (uint32_t)u;
        else if (k == "cluster_nnz")
            t.cluster_nnz = (uint32_t)u;
        else if (k == "session_cutoff_n")
            t.session_cutoff_n = (uint32_t)u;
        else if (k == "session_pool")
            t.session_pool = (uint32_t)u;
        else if (k == "session_team_nnz")
            t.session_team_nnz = (uint32_t)u;
        else if (k == "session_cluster_max")
            t.session_cluster_max = (uint32_t)u;
        else if (k == "trials")
            t.trials = (uint32_t)u;
        else if (k == "default_ms")
            t.default_ms = std::strtof(v.c_str(), nullptr);
        else if (k == "best_ms")
            t.best_ms = std::strtof(v.c_str(), nullptr);
        else if (k == "session_default_ms")
            t.session_default_ms = std::strtof(v.c_str(), nullptr);
        else if (k == "session_best_ms")
            t.session_best_ms = std::strtof(v.c_str(), nullptr);
    }
    std::fclose(f);
    if (!magic || !version || (int)t.sms != sms || !valid(t))
        return false;
    t.source = 1;
    *out = t;
    return true;
}

extern "C" {

int32_t pbrcm_tuning_get(pbrcm_context* ctx, pbrcm_tuning* out)
{
    if (!ctx || !out)
        return PBRCM_ERR_ARG;
    std::lock_guard<std::mutex> lk(ctx->ctx.mu);
    *out = from_context(ctx->ctx);
    return PBRCM_OK;
}

int32_t pbrcm_tuning_set(pbrcm_context* ctx, const pbrcm_tuning* t)
{
    if (!ctx || !t || !valid(*t))
        return PBRCM_ERR_ARG;
    std::lock_guard<std::mutex> lk(ctx->ctx.mu);
    to_context(ctx->ctx, *t);
    ctx->ctx.tuned = 2;
    return PBRCM_OK;
}

int32_t pbrcm_tuning_load(pbrcm_context* ctx, const char* path)
{
    if (!ctx || !path)
        return PBRCM_ERR_ARG;
    std::lock_guard<std::mutex> lk(ctx->ctx.mu);
    pbrcm_tuning t;
    if (!load_tuning_file(path, ctx->ctx.sms, &t))
        return PBRCM_ERR_NOT_FOUND;
    to_context(ctx->ctx, t);
    ctx->ctx.tuned = 1;
    return PBRCM_OK;
}

int32_t pbrcm_autotune(pbrcm_context* ctx, const pbrcm_matrix* mats, uint32_t count, const pbrcm_options* opts,
                       const char* cache_path, pbrcm_tuning* out)
{
    using Clock = std::chrono::steady_clock;
    if (!ctx || !mats || count == 0)
        return PBRCM_ERR_ARG;
    for (uint32_t i = 0; i < count; ++i)
        if (!mats[i].row_ptr || (!mats[i].col_idx && mats[i].nnz) || mats[i].n == 0 || mats[i].nnz > kMaxNnz)
            return PBRCM_ERR_ARG;
    std::unique_lock<std::mutex> lk(ctx->ctx.mu);
    Context& C = ctx->ctx;
    cudaSetDevice(C.device);
    cudaStream_t st = C.stream;

    // the calibration batch on the device, once
    size_t bytes = 0;
    for (uint32_t i = 0; i < count; ++i)
        bytes += (4 * ((size_t)mats[i].n + 1) + 4 * (size_t)mats[i].nnz + 4 * (size_t)mats[i].n + 255) & ~(size_t)255;
    unsigned char* D = nullptr;
    if (cudaMalloc(&D, bytes) != cudaSuccess)
        return PBRCM_ERR_OOM;
    std::vector<pbrcm_matrix> dm(count);
    size_t off = 0;
    bool ok = true;
    for (uint32_t i = 0; i < count && ok; ++i) {
        const pbrcm_matrix& m = mats[i];
        dm[i] = m;
        uint32_t* rp = reinterpret_cast<uint32_t*>(D + off);
        uint32_t* ci = rp + (m.n + 1);
        uint32_t* pm = ci + m.nnz;
        ok = cudaMemcpyAsync(rp, m.row_ptr, 4 * ((size_t)m.n + 1), cudaMemcpyHostToDevice, st) == cudaSuccess &&
             (!m.nnz || cudaMemcpyAsync(ci, m.col_idx, 4 * (size_t)m.nnz, cudaMemcpyHostToDevice, st) == cudaSuccess);
        dm[i].row_ptr = rp;
        dm[i].col_idx = ci;
        dm[i].perm_out = pm;
        off += (4 * ((size_t)m.n + 1) + 4 * (size_t)m.nnz + 4 * (size_t)m.n + 255) & ~(size_t)255;
    }
    std::vector<pbrcm_result> res(count);
    std::vector<uint32_t> ref_perms, perms;
    int32_t rc = ok ? PBRCM_OK : PBRCM_ERR_CUDA;
    pbrcm_tuning best = from_context(C);
    uint32_t trials = 0;

    // one setting: one untimed run, then the median of three event-timed
    // runs; the permutations must equal the first run's
    auto measure = [&](const pbrcm_tuning& t, float& ms) -> int32_t {
        to_context(C, t);
        float times[3];
        for (int r = 0; r < 4; ++r) {
            const auto t0 = Clock::now();
            int32_t e = run_batch(C, dm.data(), count, opts, res.data(), st, false);
            if (e != PBRCM_OK)
                return e;
            if (r > 0)
                times[r - 1] = std::chrono::duration<float, std::milli>(Clock::now() - t0).count();
        }
        std::sort(times, times + 3);
        ms = times[1];
        ++trials;
        if (!fetch_perms(dm, perms, st))
            return PBRCM_ERR_CUDA;
        if (ref_perms.empty())
            ref_perms = perms;
        else if (perms != ref_perms)
            return PBRCM_ERR_CHECK;
        return PBRCM_OK;
    };

    float best_ms = 0.f, default_ms = 0.f;
    if (rc == PBRCM_OK)
        rc = measure(best, default_ms);
    best_ms = default_ms;
    auto try_setting = [&](pbrcm_tuning t) {
        if (rc != PBRCM_OK || !valid(t))
            return;
        float ms = 0.f;
        rc = measure(t, ms);
        if (rc == PBRCM_OK && ms < best_ms * 0.985f) {  // keep a setting only for a clear gain
            best_ms = ms;
            best = t;
        }
    };
    // 1. thread-group shape, with the general and (where the shape has
    // one) the solo batch kernel
    {
        const pbrcm_tuning base = best;
        for (uint32_t p = 0; p < (uint32_t)kNumPools; ++p) {
            if (!batch_pool_ok((int)p))
                continue;
            for (uint32_t k = 0; k < 2; ++k) {
                if (k == 1 && solo_max_ctas((int)p, C.sms) <= 0)
                    continue;
                pbrcm_tuning t = best;
                t.batch_pool = p;
                t.batch_kernel = k;
                if (p != base.batch_pool || k != base.batch_kernel)
                    try_setting(t);
            }
        }
    }
    // 2. cluster teams for the biggest matrices: size x count
    {
        const pbrcm_tuning base = best;
        const uint32_t sizes[] = {1, 2, 4};
        const uint32_t counts[] = {8, 16, 32, 64};
        for (uint32_t cs : sizes)
            for (uint32_t cm : counts) {
                if (cs == 1 && cm != counts[0])
                    continue;  // "none" once
                pbrcm_tuning t = base;
                t.cluster_size = cs;
                t.cluster_max = cm;
                if (t.cluster_size != base.cluster_size || t.cluster_max != base.cluster_max)
                    try_setting(t);
            }
    }
    // 3. the entry count from which a matrix may get a cluster team
    if (best.cluster_size > 1) {
        const pbrcm_tuning base = best;
        for (uint32_t sh : {16u, 17u, 18u, 19u, 20u}) {
            pbrcm_tuning t = base;
            t.cluster_nnz = 1u << sh;
            if (t.cluster_nnz != base.cluster_nnz)
                try_setting(t);
        }
    }
    to_context(C, best);
    cudaFree(D);
    lk.unlock();

    // 4. serving cutoff and CTA shape: the batch replayed through a session (host buffers,
    // all requests at once), makespan; results must equal the batch's
    float sdef = 0.f, sbest = 0.f;
    if (rc == PBRCM_OK) {
        auto replay = [&](uint32_t cutoff, uint32_t pool, uint32_t team_nnz, uint32_t cmax, float& ms) -> int32_t {
            {
                std::lock_guard<std::mutex> g(C.mu);
                C.session_cutoff_n = cutoff;
                C.session_pool = (int)pool;
                C.session_team_nnz = team_nnz;
                C.session_cluster_max = (int)cmax;
            }
            pbrcm_session* s = nullptr;
            int32_t e = pbrcm_session_create(ctx, nullptr, &s);
            if (e != PBRCM_OK)
                return e;
            std::vector<uint64_t> tk(count);
            const auto t0 = Clock::now();
            for (uint32_t i = 0; i < count && e == PBRCM_OK; ++i)
                e = pbrcm_session_submit(s, mats[i].row_ptr, mats[i].col_idx, mats[i].n, mats[i].nnz, opts, &tk[i]);
            if (e == PBRCM_OK)
                e = pbrcm_session_drain(s);
            ms = std::chrono::duration<float, std::milli>(Clock::now() - t0).count();
            size_t poff = 0;
            std::vector<uint32_t> p;
            for (uint32_t i = 0; i < count && e == PBRCM_OK; ++i) {
                p.resize(mats[i].n);
                int32_t done = 0;
                e = pbrcm_session_poll(s, tk[i], p.data(), nullptr, &done);
                if (e == PBRCM_OK && (!done || std::memcmp(p.data(), ref_perms.data() + poff, 4 * p.size()) != 0))
                    e = PBRCM_ERR_CHECK;
                poff += mats[i].n;
            }
            pbrcm_session_destroy(s);
            ++trials;
            return e;
        };
        const uint32_t start_cut = best.session_cutoff_n;
        const uint32_t start_pool = best.session_pool;
        const uint32_t tnnz = best.session_team_nnz, cmax = best.session_cluster_max;
        rc = replay(start_cut, start_pool, tnnz, cmax, sdef);
        sbest = sdef;
        for (uint32_t pool : {0u, 4u, 5u, 6u})
            for (uint32_t sh : {16u, 17u, 18u, 19u, 20u}) {
                const uint32_t cut = 1u << sh;
                if (rc != PBRCM_OK || (cut == start_cut && pool == start_pool))
                    continue;
                float ms = 0.f;
                rc = replay(cut, pool, tnnz, cmax, ms);
                if (rc == PBRCM_OK && ms < sbest * 0.97f) {
                    sbest = ms;
                    best.session_cutoff_n = cut;
                    best.session_pool = pool;
                }
            }
        // 5. the teams of big requests: CTAs per entry and the largest
        // thread-block-cluster team
        for (uint32_t cm : {0u, 8u, 16u})
            for (uint32_t sh : {19u, 20u, 21u}) {
                const uint32_t tn = 1u << sh;
                if (rc != PBRCM_OK || (tn == tnnz && cm == cmax))
                    continue;
                float ms = 0.f;
                rc = replay(best.session_cutoff_n, best.session_pool, tn, cm, ms);
                if (rc == PBRCM_OK && ms < sbest * 0.97f) {
                    sbest = ms;
                    best.session_team_nnz = tn;
                    best.session_cluster_max = cm;
                }
            }
        std::lock_guard<std::mutex> g(C.mu);
        C.session_cutoff_n = best.session_cutoff_n;
        C.session_pool = (int)best.session_pool;
        C.session_team_nnz = best.session_team_nnz;
        C.session_cluster_max = (int)best.session_cluster_max;
    }
    if (rc != PBRCM_OK)
        return rc;
    std::lock_guard<std::mutex> g(C.mu);
    C.tuned = 2;
    best.sms = (uint32_t)C.sms;
    best.trials = trials;
    best.source = 2;
    best.default_ms = default_ms;
    best.best_ms = best_ms;
    best.session_default_ms = sdef;
    best.session_best_ms = sbest;
    if (cache_path && !write_file(cache_path, best))
        rc = PBRCM_ERR_IO;
    if (out)
        *out = best;
    return rc;
}

}  // extern "C"
