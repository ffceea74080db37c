// batch.cpp -- many independent matrices in one persistent launch
// (pbrcm_reorder_batch / pbrcm_reorder_batch_device).
//
// Layout: one device arena per call holds, per matrix, its CSR (host-input
// form only), its node table node[n], rec[n] and perm[n] (host-input form
// only), each 16-byte aligned.  Jobs are ordered by nnz, biggest first.  The
// biggest (nnz >= cluster_nnz, at most cluster_max of them) are reordered by
// thread-block-cluster teams of whole CTAs; every other job takes one slot
// of the work list, which the CTAs' thread groups (several per CTA, the
// context's pool shape) hand out with an atomic counter, so that several
// matrices are in flight on every SM.  (With PBRCM_BATCH_TEAM_MAX > 1 a big
// job instead gets a team of K groups with its own zeroed barrier words and
// K consecutive slots, in a cooperative launch.)  Every group of a job runs
// the whole reorder of that matrix (start search, CM pass, reverse,
// bandwidth).
#include <algorithm>
#include <chrono>
#include <cstring>
#include <numeric>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/pbrcm.h"
#include "context.h"
#include "kernels.h"
#include "types.h"

using namespace pbrcm;

namespace {

inline size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }
inline size_t align128(size_t x) { return (x + 127) & ~(size_t)127; }

struct Slot {
    size_t rp, ci, node, rec, perm, e2, gvis;  // arena offsets (rp/ci/perm unused for device input;
                                               // e2 / gvis 0: none)
};

int env_int(const char* name, int dflt)
{
    const char* v = std::getenv(name);
    return v && *v ? std::atoi(v) : dflt;
}

template <typename T>
bool grow_dev(T*& p, size_t& cap, size_t need)
{
    if (need <= cap && p)
        return true;
    if (p)
        cudaFree(p);
    p = nullptr;
    cap = 0;
    if (cudaMalloc(&p, sizeof(T) * std::max<size_t>(need, 1)) != cudaSuccess)
        return false;
    cap = std::max<size_t>(need, 1);
    return true;
}

// Team size of a job: one CTA up to min_nnz entries, then one CTA per
// nnz_per_cta entries, at most max_team.
uint32_t team_size(uint64_t nnz, uint64_t min_nnz, uint64_t nnz_per_cta, uint32_t max_team)
{
    if (nnz < min_nnz || max_team < 2)
        return 1;
    const uint64_t k = (nnz + nnz_per_cta - 1) / nnz_per_cta;
    return (uint32_t)std::max<uint64_t>(2, std::min<uint64_t>(k, max_team));
}

}  // namespace

namespace {

template <typename T>
bool grow_pinned(T*& p, size_t& cap, size_t need)
{
    if (need <= cap && p)
        return true;
    if (p)
        cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    if (cudaMallocHost(&p, sizeof(T) * std::max<size_t>(need, 1)) != cudaSuccess)
        return false;
    cap = std::max<size_t>(need, 1);
    return true;
}

bool is_pinned(const void* p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

inline void mix(uint64_t& h, uint64_t v)
{
    h ^= v + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
}

// Everything a captured batch depends on: the matrices' buffers and sizes,
// the options, the shape settings and the context's device buffers.
uint64_t batch_key(const Context& C, const pbrcm_matrix* mats, uint32_t count, const Options& opt, bool host)
{
    uint64_t h = 0x5EED;
    mix(h, count);
    mix(h, host ? 1 : 2);
    for (uint32_t j = 0; j < count; ++j) {
        mix(h, (uint64_t)(uintptr_t)mats[j].row_ptr);
        mix(h, (uint64_t)(uintptr_t)mats[j].col_idx);
        mix(h, (uint64_t)(uintptr_t)mats[j].perm_out);
        mix(h, ((uint64_t)mats[j].n << 32) ^ mats[j].nnz);
    }
    for (uint64_t v : {(uint64_t)opt.start, (uint64_t)opt.reverse, (uint64_t)opt.want_bw, (uint64_t)opt.outnodes,
                       (uint64_t)opt.wait_ns, (uint64_t)opt.phantom, (uint64_t)C.batch_pool,
                       (uint64_t)C.cluster_size, (uint64_t)C.cluster_max, (uint64_t)C.cluster_nnz,
                       (uint64_t)C.solo, (uint64_t)C.batch_solo_kernel, (uint64_t)(uintptr_t)C.d_arena, (uint64_t)(uintptr_t)C.d_jobs,
                       (uint64_t)(uintptr_t)C.d_slots, (uint64_t)(uintptr_t)C.d_bres,
                       (uint64_t)(uintptr_t)C.d_ready, (uint64_t)(uintptr_t)C.d_counter,
                       (uint64_t)(uintptr_t)C.h_bres})
        mix(h, v);
    return h;
}

}  // namespace

// Shared driver; `host` selects whether mats[] point to host or device memory.
//
// 1. prepare (host): job order, team / cluster decisions, arena layout,
//    copy waves, the job list in pinned staging;
// 2. enqueue: zero the per-call words, upload the job list, launch the batch
//    kernel, then (host buffers) the CSR copies wave by wave on the copy
//    stream, and the results and permutations back behind the kernel.  A
//    batch on device buffers, or on host buffers that are all pinned, is
//    captured as a CUDA graph on its first call and replayed on later calls
//    with the same buffers, sizes, options and shape (step 1 is then
//    skipped);
// 3. finish: wait, rerun matrices with a hub row on the team path, fill the
//    results.
int32_t pbrcm::run_batch(Context& C, const pbrcm_matrix* mats, uint32_t count, const pbrcm_options* opts,
                         pbrcm_result* results, cudaStream_t st, bool host)
{
    auto t0 = std::chrono::steady_clock::now();
    Options opt = make_options(opts, kModeFull);
    const int v = C.batch_pool;
    opt.solo_parents = 2 * kPools[v].group;
    opt.solo_edges = 2 * kPools[v].gemax;
    opt.barrier = 0;
    for (uint32_t j = 0; j < count; ++j) {
        const pbrcm_matrix& m = mats[j];
        if (!m.row_ptr || (!m.col_idx && m.nnz) || !m.perm_out || m.n == 0 || m.n == 0xFFFFFFFFu ||
            m.nnz > kMaxNnz)
            return PBRCM_ERR_ARG;
    }
    const int maxc = batch_max_ctas(v, C.sms);
    if (maxc <= 0)
        return PBRCM_ERR_CUDA;
    // host buffers: a permutation buffer in pinned memory is written by the
    // kernel itself (its device-side address; no copy back after the
    // kernel), and a matrix whose col_idx follows its row_ptr in memory
    // comes in with one copy instead of two
    std::vector<uint32_t*> pdirect(host ? count : 0, nullptr);
    for (uint32_t j = 0; j < count && host; ++j) {
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, mats[j].perm_out) == cudaSuccess && a.type == cudaMemoryTypeHost &&
            a.devicePointer)
            pdirect[j] = static_cast<uint32_t*>(a.devicePointer);
        else
            cudaGetLastError();
    }
    auto joined = [&](uint32_t j) {
        return mats[j].nnz && reinterpret_cast<const char*>(mats[j].col_idx) ==
                                  reinterpret_cast<const char*>(mats[j].row_ptr) + 4 * ((size_t)mats[j].n + 1);
    };
    // graph capture: device buffers, or host buffers that are all pinned (a
    // copy from pageable memory cannot be captured)
    bool use_graph = C.batch_graphs;
    for (uint32_t j = 0; j < count && use_graph && host; ++j)
        use_graph = is_pinned(mats[j].row_ptr) && (!mats[j].nnz || is_pinned(mats[j].col_idx)) && pdirect[j];
    // the wait for a wave is bounded; the bound grows with the bytes to copy
    // (at least 1 GB/s)
    size_t in_bytes = 0;
    if (host)
        for (uint32_t j = 0; j < count; ++j)
            in_bytes += 4 * ((size_t)mats[j].n + 1) + 4 * (size_t)mats[j].nnz;
    opt.data_wait_ns = opt.wait_ns + (unsigned long long)in_bytes;
    float dms = 0.f;
    bool replayed = false;
    if (use_graph && C.bgraph.exec && C.bgraph.key == batch_key(C, mats, count, opt, host) &&
        C.bgraph.order.size() == count) {
        if (cudaGraphLaunch(C.bgraph.exec, st) != cudaSuccess)
            return PBRCM_ERR_CUDA;
        replayed = true;
        ++C.bgraph.replays;
    }
    std::vector<uint32_t> order_local;
    std::vector<BatchJob> jobs_local;
    std::vector<uint32_t>& order = replayed ? C.bgraph.order : order_local;
    std::vector<BatchJob>& jobs = replayed ? C.bgraph.jobs : jobs_local;
    if (!replayed) {
        // job order (biggest first) and team sizes
        const uint64_t min_nnz = (uint64_t)env_int("PBRCM_BATCH_TEAM_MIN_NNZ", 1 << 19);
        const uint64_t per_cta = (uint64_t)std::max(1, env_int("PBRCM_BATCH_TEAM_NNZ", 1 << 18));
        // teams are off by default: on mixed batches the total work, not the
        // biggest matrix, bounds the makespan, and team members of a matrix
        // whose levels are small idle at the gate (PBRCM_BATCH_TEAM_MAX
        // enables them)
        const uint32_t max_team = (uint32_t)std::max(1, std::min(env_int("PBRCM_BATCH_TEAM_MAX", 1), maxc));
        order.resize(count);
        std::iota(order.begin(), order.end(), 0u);
        std::stable_sort(order.begin(), order.end(),
                         [&](uint32_t a, uint32_t b) { return mats[a].nnz > mats[b].nnz; });
        // Without group teams, the biggest matrices (nnz >= cluster_nnz) go to
        // thread-block-cluster teams: on one group they would set the
        // makespan.  The launch is then in clusters: they take the big
        // matrices first, then their CTAs' groups take the rest one by one.
        uint32_t nbig = 0;
        int ncl = 0;
        if (max_team == 1 && C.cluster_size > 1) {
            while (nbig < count && mats[order[nbig]].nnz >= C.cluster_nnz)
                ++nbig;
            ncl = nbig ? cluster_max_active(v, C.cluster_size) : 0;
            // one round at most: a team of CTAs spends more CTA-time on a
            // matrix than one group, so only the matrices that would set the
            // tail get one
            nbig = std::min<uint32_t>(
                nbig, (uint32_t)std::max(0, C.cluster_max > 0 ? std::min(C.cluster_max, ncl) : ncl));
            if (ncl <= 0)
                nbig = 0;
        }
        std::vector<uint32_t> team(count);
        size_t nslots = 0, teamws = 0;
        for (uint32_t q = nbig; q < count; ++q) {
            team[q] = team_size(mats[order[q]].nnz, min_nnz, per_cta, max_team);
            nslots += team[q];
            if (team[q] > 1)
                teamws = align128(teamws + sizeof(GridSync)) + align128(team_words_bytes((int)team[q]));
        }
        const bool cooperative = nslots > count - nbig;
        use_graph = use_graph && !cooperative;
        // arena layout, in job order (biggest first); every CSR on a 128-byte
        // boundary so that no cache line holds two matrices' data (a
        // host-buffer batch's CSRs arrive while other matrices are already
        // being read)
        std::vector<Slot> slot(count);
        size_t off = 0;
        for (uint32_t q = 0; q < count; ++q) {
            const uint32_t j = order[q];
            const pbrcm_matrix& m = mats[j];
            if (host) {
                slot[j].rp = off;
                if (joined(j)) {  // the host layout, so that one copy brings both
                    slot[j].ci = off + 4 * ((size_t)m.n + 1);
                    off = align128(slot[j].ci + 4 * (size_t)m.nnz);
                } else {
                    off = align128(off + 4 * ((size_t)m.n + 1));
                    slot[j].ci = off;
                    off = align128(off + 4 * (size_t)m.nnz);
                }
            }
            slot[j].node = off;
            off = align16(off + 16 * (size_t)m.n);
            slot[j].rec = off;
            off = align16(off + 16 * (size_t)m.n);
            slot[j].perm = 0;
            if (host && !pdirect[j]) {
                slot[j].perm = off;
                off = align16(off + 4 * (size_t)m.n);
            }
            // the one-group engine's edge records (16 bytes per entry) for a
            // matrix a single group will take (and its visited bitmap when
            // that does not fit shared memory); it uses the node table's room
            // for its inverse permutation
            slot[j].e2 = 0;
            slot[j].gvis = 0;
            if (C.solo && q >= nbig && team[q] == 1 && m.nnz > 0 && m.n <= kSoloMaxNodes) {
                off = align16(off);
                slot[j].e2 = off;
                off += 8 * (size_t)m.nnz;
                if (m.n > kSoloMaxN) {  // the visited bitmap does not fit shared memory
                    slot[j].gvis = off;
                    off = align16(off + 4 * (((size_t)m.n + 31) / 32));
                }
            }
            off = align128(off);
        }
        const size_t team_off = align128(off);
        off = team_off + teamws;
        // host buffers: the CSRs go in waves of about in_bytes / kWaves in
        // job order, each wave followed by its ready word, while the kernel
        // runs
        constexpr size_t kWaves = 48;
        const size_t wave_bytes = std::max<size_t>(in_bytes / kWaves, (size_t)4 << 20);
        std::vector<uint32_t> wave(count, 0);
        uint32_t nwaves = 0;
        if (host) {
            size_t cum = 0;
            for (uint32_t q = 0; q < count; ++q) {
                const pbrcm_matrix& m = mats[order[q]];
                wave[q] = nwaves;
                cum += 4 * ((size_t)m.n + 1) + 4 * (size_t)m.nnz;
                if (cum >= wave_bytes || q + 1 == count) {
                    ++nwaves;
                    cum = 0;
                }
            }
        }
        if (!grow_dev(C.d_arena, C.cap_arena, off) || !grow_dev(C.d_jobs, C.cap_jobs, count) ||
            !grow_dev(C.d_bres, C.cap_bres, count) || !grow_dev(C.d_slots, C.cap_slots, nslots) ||
            !grow_dev(C.d_counter, C.cap_counter, 8) || (nwaves && !grow_dev(C.d_ready, C.cap_ready, nwaves)) ||
            !grow_pinned(C.h_jobs, C.cap_hjobs, count) || !grow_pinned(C.h_slots, C.cap_hslots, nslots) ||
            !grow_pinned(C.h_bres, C.cap_hbres, count))
            return PBRCM_ERR_OOM;
        unsigned char* A = C.d_arena;
        jobs.assign(count, BatchJob{});
        size_t tw = team_off, ns = 0;
        for (uint32_t q = 0; q < count; ++q) {
            const uint32_t j = order[q];
            const pbrcm_matrix& m = mats[j];
            BatchJob& J = jobs[q];
            std::memset(&J, 0, sizeof(J));
            J.M.rp = host ? reinterpret_cast<const uint32_t*>(A + slot[j].rp) : m.row_ptr;
            J.M.ci = host ? reinterpret_cast<const uint32_t*>(A + slot[j].ci) : m.col_idx;
            J.M.n = m.n;
            J.M.nnz = (uint32_t)m.nnz;
            J.M.node = reinterpret_cast<NodeEntry*>(A + slot[j].node);
            J.M.rec = reinterpret_cast<PosRec*>(A + slot[j].rec);
            J.M.perm = !host ? m.perm_out : pdirect[j] ? pdirect[j] : reinterpret_cast<uint32_t*>(A + slot[j].perm);
            J.M.hub = nullptr;
            J.M.res = C.d_bres + q;
            J.team = q < nbig ? 1 : team[q];
            J.ready = host ? C.d_ready + wave[q] : nullptr;
            J.e2 = slot[j].e2 ? reinterpret_cast<uint2*>(A + slot[j].e2) : nullptr;
            J.gvis = slot[j].gvis ? reinterpret_cast<uint32_t*>(A + slot[j].gvis) : nullptr;
            J.inv = reinterpret_cast<uint32_t*>(A + slot[j].node);
            if (team[q] > 1) {
                J.gs = reinterpret_cast<GridSync*>(A + tw);
                tw = align128(tw + sizeof(GridSync));
                J.words = reinterpret_cast<unsigned long long*>(A + tw);
                tw = align128(tw + team_words_bytes((int)team[q]));
            }
            for (uint32_t r = 0; r < team[q]; ++r)
                C.h_slots[ns++] = BatchSlot{q, r};
        }
        std::memcpy(C.h_jobs, jobs.data(), sizeof(BatchJob) * count);

        // ---- enqueue (captured as a graph when use_graph) ----------------
        // (not on the legacy default stream, nor on a stream the caller is
        // capturing; a capture that cannot start falls back to plain launches)
        const BatchJob* src_jobs = C.h_jobs;
        const BatchSlot* src_slots = C.h_slots;
        if (use_graph) {
            // the graph uploads its job list from pinned buffers of its own
            // (the context's staging is rewritten by every batch that is not
            // a replay); the graph they belonged to goes first
            if (C.bgraph.exec) {
                cudaGraphExecDestroy(C.bgraph.exec);
                C.bgraph.exec = nullptr;
            }
            if (!grow_pinned(C.bgraph.h_jobs, C.bgraph.cap_jobs, count) ||
                !grow_pinned(C.bgraph.h_slots, C.bgraph.cap_slots, nslots))
                return PBRCM_ERR_OOM;
            std::memcpy(C.bgraph.h_jobs, C.h_jobs, sizeof(BatchJob) * count);
            std::memcpy(C.bgraph.h_slots, C.h_slots, sizeof(BatchSlot) * nslots);
            src_jobs = C.bgraph.h_jobs;
            src_slots = C.bgraph.h_slots;
            cudaStreamCaptureStatus cs_status = cudaStreamCaptureStatusNone;
            if (st == nullptr || st == cudaStreamLegacy || st == cudaStreamPerThread ||
                cudaStreamIsCapturing(st, &cs_status) != cudaSuccess || cs_status != cudaStreamCaptureStatusNone ||
                cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
                cudaGetLastError();
                use_graph = false;
            }
        }
        bool ok = cudaMemcpyAsync(C.d_jobs, src_jobs, sizeof(BatchJob) * count, cudaMemcpyHostToDevice, st) ==
                      cudaSuccess &&
                  cudaMemcpyAsync(C.d_slots, src_slots, sizeof(BatchSlot) * nslots, cudaMemcpyHostToDevice, st) ==
                      cudaSuccess &&
                  (!teamws || cudaMemsetAsync(A + team_off, 0, teamws, st) == cudaSuccess) &&
                  (!nwaves || cudaMemsetAsync(C.d_ready, 0, sizeof(uint32_t) * nwaves, st) == cudaSuccess) &&
                  cudaMemsetAsync(C.d_bres, 0, sizeof(DevResult) * count, st) == cudaSuccess &&
                  cudaMemsetAsync(C.d_counter, 0, 2 * sizeof(uint32_t), st) == cudaSuccess;
        // the copy stream starts once the ready words are zeroed (fork)
        if (ok && host)
            ok = cudaEventRecord(C.ev_fork, st) == cudaSuccess &&
                 cudaStreamWaitEvent(C.copy_stream, C.ev_fork, 0) == cudaSuccess;
        if (ok && !use_graph)
            ok = cudaEventRecord(C.ev0, st) == cudaSuccess;
        if (ok && nbig) {
            Options copt = opt;
            copt.solo_parents = C.cluster_solo_parents;
            copt.solo_edges = C.cluster_solo_edges;
            ok = launch_cluster(v, C.d_jobs, nbig, C.d_slots, (uint32_t)nslots, C.d_counter, copt, opt,
                                C.cluster_size, ncl, st) == cudaSuccess;
        } else if (ok) {
            // every job one group's: the solo batch kernel where the shape
            // has one, else the general kernel
            const uint32_t per = (uint32_t)(kPools[v].block / kPools[v].group);
            const int smaxc = C.solo && C.batch_solo_kernel && !cooperative ? solo_max_ctas(v, C.sms) : 0;
            const int ctas = std::max(1, std::min<int>(smaxc > 0 ? smaxc : maxc, (int)((nslots + per - 1) / per)));
            ok = (smaxc > 0 ? launch_solo(v, C.d_jobs, C.d_slots, (uint32_t)nslots, C.d_counter, opt, ctas, st)
                            : launch_batch(v, C.d_jobs, C.d_slots, (uint32_t)nslots, C.d_counter, opt, ctas,
                                           cooperative, st)) == cudaSuccess;
        }
        if (ok && host) {
            // the inputs, wave by wave, each wave's ready word after its CSRs
            // (copies on one stream complete in order); the kernel above
            // waits for each matrix's wave
            cudaStream_t cs = C.copy_stream;
            uint32_t q = 0;
            for (uint32_t w = 0; w < nwaves && ok; ++w) {
                for (; q < count && wave[q] == w && ok; ++q) {
                    const pbrcm_matrix& m = mats[order[q]];
                    const Slot& sl = slot[order[q]];
                    if (joined(order[q]))
                        ok = cudaMemcpyAsync(A + sl.rp, m.row_ptr, 4 * ((size_t)m.n + 1 + m.nnz),
                                             cudaMemcpyHostToDevice, cs) == cudaSuccess;
                    else
                        ok = cudaMemcpyAsync(A + sl.rp, m.row_ptr, 4 * ((size_t)m.n + 1), cudaMemcpyHostToDevice,
                                             cs) == cudaSuccess &&
                             (!m.nnz || cudaMemcpyAsync(A + sl.ci, m.col_idx, 4 * (size_t)m.nnz,
                                                        cudaMemcpyHostToDevice, cs) == cudaSuccess);
                }
                ok = ok && cudaMemcpyAsync(C.d_ready + w, C.h_one, sizeof(uint32_t), cudaMemcpyHostToDevice, cs) ==
                               cudaSuccess;
            }
            // join: nothing after the kernel runs before the copies are done
            ok = ok && cudaEventRecord(C.ev_join, cs) == cudaSuccess &&
                 cudaStreamWaitEvent(st, C.ev_join, 0) == cudaSuccess;
        }
        if (ok && !use_graph)
            ok = cudaEventRecord(C.ev1, st) == cudaSuccess;
        ok = ok && cudaMemcpyAsync(C.h_bres, C.d_bres, sizeof(DevResult) * count, cudaMemcpyDeviceToHost, st) ==
                       cudaSuccess;
        // every permutation not written in place straight behind the kernel
        // (issued while it runs); a matrix that fails leaves its perm_out
        // unspecified
        for (uint32_t q = 0; q < count && ok && host; ++q)
            if (!pdirect[order[q]])
                ok = cudaMemcpyAsync(mats[order[q]].perm_out, jobs[q].M.perm, 4 * (size_t)mats[order[q]].n,
                                     cudaMemcpyDeviceToHost, st) == cudaSuccess;
        if (use_graph) {
            cudaGraph_t g = nullptr;
            const bool ended = cudaStreamEndCapture(st, &g) == cudaSuccess;
            cudaGraphExec_t exec = nullptr;
            ok = ok && ended && g && cudaGraphInstantiate(&exec, g, 0) == cudaSuccess;
            if (g)
                cudaGraphDestroy(g);
            if (ok) {
                C.bgraph.exec = exec;
                C.bgraph.key = batch_key(C, mats, count, opt, host);
                C.bgraph.order = order;
                C.bgraph.jobs = jobs;
                C.bgraph.replays = 0;
                ok = cudaGraphLaunch(exec, st) == cudaSuccess;
            } else if (exec) {
                cudaGraphExecDestroy(exec);
            }
        }
        if (!ok)
            return PBRCM_ERR_CUDA;
    }
    // ---- finish -------------------------------------------------------------
    if (cudaStreamSynchronize(st) != cudaSuccess)
        return PBRCM_ERR_CUDA;
    if (!replayed && !use_graph)
        cudaEventElapsedTime(&dms, C.ev0, C.ev1);
    std::vector<DevResult> res(C.h_bres, C.h_bres + count);
    // matrices with a hub row rerun on the team path with hub scratch
    Options topt = make_options(opts, kModeFull);
    apply_team_shape(C, topt);
    for (uint32_t q = 0; q < count; ++q) {
        if (res[q].status != kNeedHub)
            continue;
        const MatrixView& M = jobs[q].M;
        if (!C.ensure_hub(M.nnz))
            return PBRCM_ERR_OOM;
        MatrixView H = M;
        H.hub = C.d_hub;
        if (cudaMemsetAsync(M.res, 0, sizeof(DevResult), st) != cudaSuccess ||
            cudaMemsetAsync(C.d_gs, 0, sizeof(GridSync), st) != cudaSuccess ||
            cudaMemsetAsync(C.d_agg, 0, team_words_bytes(C.team_ctas), st) != cudaSuccess ||
            launch_validate(M.rp, M.ci, M.n, M.nnz, M.res, C.sms, st) != cudaSuccess ||
            launch_team(C.team_variant, H, topt, C.d_gs, C.d_agg, C.team_ctas, st) != cudaSuccess ||
            cudaMemcpyAsync(&res[q], M.res, sizeof(DevResult), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            (host && !pdirect[order[q]] &&
             cudaMemcpyAsync(mats[order[q]].perm_out, M.perm, 4 * (size_t)M.n, cudaMemcpyDeviceToHost, st) !=
                 cudaSuccess) ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return PBRCM_ERR_CUDA;
    }
    // per-matrix latency inside the batch: from the first matrix taken to
    // this one's result (device %globaltimer)
    unsigned long long tmin = ~0ull;
    for (uint32_t q = 0; q < count; ++q)
        if (res[q].t_begin)
            tmin = std::min(tmin, res[q].t_begin);
    int32_t worst = PBRCM_OK;
    for (uint32_t q = 0; q < count; ++q) {
        const uint32_t j = order[q];
        if (results) {
            fill_result(res[q], opt, &results[j]);
            results[j].device_ms = res[q].t_end >= tmin && tmin != ~0ull ? (float)((res[q].t_end - tmin) * 1e-6)
                                                                          : dms;
        }
        if (res[q].status != kOk && worst == PBRCM_OK)
            worst = map_status(res[q].status);
    }
    if (results) {
        const float tms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
        for (uint32_t j = 0; j < count; ++j)
            results[j].total_ms = tms;
    }
    return worst;
}

extern "C" {

int32_t pbrcm_reorder_batch(pbrcm_context* ctx, const pbrcm_matrix* mats, uint32_t count, const pbrcm_options* opts,
                            pbrcm_result* results)
{
    if (!mats && count)
        return PBRCM_ERR_ARG;
    if (count == 0)
        return PBRCM_OK;
    pbrcm_context* ctx_local = nullptr;
    if (!ctx) {
        int32_t rc = pbrcm_context_create(-1, &ctx_local);
        if (rc != PBRCM_OK)
            return rc;
        ctx = ctx_local;
    }
    int32_t rc;
    {
        std::lock_guard<std::mutex> lk(ctx->ctx.mu);
        cudaSetDevice(ctx->ctx.device);
        rc = run_batch(ctx->ctx, mats, count, opts, results, ctx->ctx.stream, true);
    }
    if (ctx_local)
        pbrcm_context_destroy(ctx_local);
    return rc;
}

int32_t pbrcm_reorder_batch_device(pbrcm_context* ctx, const pbrcm_matrix* mats, uint32_t count,
                                   const pbrcm_options* opts, pbrcm_result* results, void* stream)
{
    if (!mats && count)
        return PBRCM_ERR_ARG;
    if (count == 0)
        return PBRCM_OK;
    pbrcm_context* ctx_local = nullptr;
    if (!ctx) {
        int32_t rc = pbrcm_context_create(-1, &ctx_local);
        if (rc != PBRCM_OK)
            return rc;
        ctx = ctx_local;
    }
    int32_t rc;
    {
        std::lock_guard<std::mutex> lk(ctx->ctx.mu);
        cudaSetDevice(ctx->ctx.device);
        rc = run_batch(ctx->ctx, mats, count, opts, results, stream ? (cudaStream_t)stream : ctx->ctx.stream,
                       false);
    }
    if (ctx_local)
        pbrcm_context_destroy(ctx_local);
    return rc;
}

}  // extern "C"
