// session.cpp -- serving session: continuous batching of reorder requests.
//
// submit() copies a request's CSR into pinned staging and queues it.  A
// worker thread admits queued requests in arrival order whenever the device
// bytes in flight stay under the cap, the CTAs they hold fit the GPU and a
// stream is free, and launches each one at once on that stream (no request
// waits behind another in a stream): stream-ordered device allocation, H2D,
// validation, the reorder kernel (one CTA for small matrices, a cooperative
// team for large ones or ones with hub rows), D2H of the permutation and the
// result, an event.  Requests that arrive while others run are launched
// immediately, so their kernels overlap on the device.  The worker retires
// finished requests by polling their events, frees their memory and records
// submit->completion latency.  The reference has no serving mode; each result
// equals the single-matrix result for the same input.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/pbrcm.h"
#include "context.h"
#include "kernels.h"
#include "types.h"

using namespace pbrcm;

namespace {

using Clock = std::chrono::steady_clock;

inline size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

// Pinned host memory for the sessions' staging: slabs from cudaHostAlloc,
// carved first-fit into blocks that coalesce again when freed.  One pool per
// context, shared by its sessions (a session finds the staging earlier ones
// left behind); its own lock.  Pinning costs milliseconds per call, so the
// pool grows in slabs of at least its current size and never shrinks: a
// burst of requests that fit before fits again.
class PinnedPool {
public:
    ~PinnedPool()
    {
        for (const Slab& sl : slabs_)
            cudaFreeHost(sl.base);
    }
    void* get(size_t bytes, size_t& cap)
    {
        std::lock_guard<std::mutex> lk(mu_);
        bytes = (std::max<size_t>(bytes, 1) + 4095) & ~(size_t)4095;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second.size < bytes)
                continue;
            unsigned char* p = it->first;
            const Block b = it->second;
            free_.erase(it);
            if (b.size > bytes)
                free_.emplace(p + bytes, Block{b.size - bytes, b.slab});
            cap = bytes;
            return p;
        }
        const size_t sz = std::max(bytes, std::max(total_, (size_t)64 << 20));
        void* raw = nullptr;
        if (cudaHostAlloc(&raw, sz, cudaHostAllocDefault) != cudaSuccess)
            return nullptr;
        auto* base = static_cast<unsigned char*>(raw);
        slabs_.push_back(Slab{base, sz});
        total_ += sz;
        if (sz > bytes)
            free_.emplace(base + bytes, Block{sz - bytes, slabs_.size() - 1});
        cap = bytes;
        return base;
    }
    void put(void* ptr, size_t cap)
    {
        if (!ptr)
            return;
        std::lock_guard<std::mutex> lk(mu_);
        auto* p = static_cast<unsigned char*>(ptr);
        size_t slab = 0;
        while (slab < slabs_.size() && !(p >= slabs_[slab].base && p < slabs_[slab].base + slabs_[slab].size))
            ++slab;
        Block b{cap, slab};
        // coalesce with the blocks on either side (same slab only)
        auto next = free_.lower_bound(p);
        if (next != free_.end() && next->first == p + b.size && next->second.slab == slab) {
            b.size += next->second.size;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second.size == p && prev->second.slab == slab) {
                prev->second.size += b.size;
                return;
            }
        }
        free_.emplace(p, b);
    }
    size_t pinned_bytes() const { return total_; }

private:
    struct Slab {
        unsigned char* base;
        size_t size;
    };
    struct Block {
        size_t size;
        size_t slab;
    };
    std::mutex mu_;
    std::vector<Slab> slabs_;
    std::map<unsigned char*, Block> free_;  // free blocks by address
    size_t total_ = 0;
};

// Host threads for the submit-time copy of a CSR into pinned staging: one
// thread copies pageable memory at a few GB/s, so a request of millions of
// entries would spend milliseconds in submit and a burst of them would
// throttle the whole stream.  run(parts, f) runs f(0) .. f(parts - 1) on the
// pool's threads and the caller and returns when all are done; concurrent
// callers take turns.
class CopyPool {
public:
    explicit CopyPool(int threads)
    {
        for (int i = 0; i < threads; ++i)
            th_.emplace_back([this] { loop(); });
    }
    ~CopyPool()
    {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (std::thread& t : th_)
            t.join();
    }
    int threads() const { return (int)th_.size(); }
    void run(int parts, const std::function<void(int)>& f)
    {
        std::lock_guard<std::mutex> turn(run_mu_);
        auto job = std::make_shared<Job>();
        job->f = &f;
        job->parts = parts;
        {
            std::lock_guard<std::mutex> lk(mu_);
            job_ = job;
            ++gen_;
        }
        cv_.notify_all();
        work(*job);
        std::unique_lock<std::mutex> lk(mu_);
        cv_done_.wait(lk, [&] { return job->done == job->parts; });
        job_.reset();
    }

private:
    struct Job {
        const std::function<void(int)>* f = nullptr;
        int parts = 0;
        std::atomic<int> next{0};
        int done = 0;  // under mu_
    };
    void work(Job& job)
    {
        // f stays valid while a part is left: run() returns only after the
        // last part is done
        while (true) {
            const int p = job.next.fetch_add(1);
            if (p >= job.parts)
                return;
            (*job.f)(p);
            std::lock_guard<std::mutex> lk(mu_);
            if (++job.done == job.parts)
                cv_done_.notify_all();
        }
    }
    void loop()
    {
        uint64_t seen = 0;
        std::unique_lock<std::mutex> lk(mu_);
        while (true) {
            cv_.wait(lk, [&] { return stop_ || (gen_ != seen && job_); });
            if (stop_)
                return;
            seen = gen_;
            std::shared_ptr<Job> job = job_;
            lk.unlock();
            work(*job);
            lk.lock();
        }
    }
    std::vector<std::thread> th_;
    std::mutex mu_, run_mu_;
    std::condition_variable cv_, cv_done_;
    std::shared_ptr<Job> job_;
    uint64_t gen_ = 0;
    bool stop_ = false;
};

struct Request {
    uint64_t ticket = 0;
    uint32_t n = 0;
    uint64_t nnz = 0;
    uint32_t maxdeg = 0;
    Options opt{};
    size_t dev_bytes = 0;
    // pinned staging: [rp | ci | view | perm_out | result]
    unsigned char* host = nullptr;
    size_t host_cap = 0;
    size_t off_rp = 0, off_ci = 0, off_view = 0, off_perm = 0, off_res = 0;
    // device block: [rp | ci | node | rec | perm | res | gs | counter + view | agg | hub? | edge records?]
    unsigned char* dev = nullptr;
    size_t d_rp = 0, d_ci = 0, d_node = 0, d_rec = 0, d_perm = 0, d_res = 0, d_gs = 0, d_cnt = 0, d_agg = 0,
           d_hub = 0, d_e2 = 0, d_gvis = 0;
    bool big = false;      // above the team cutoff (or a row longer than a one-CTA chunk)
    bool solo_able = false;  // the solo engine can take it (rows fit its chunk)
    bool team = false;     // decided at admission: a cooperative team of CTAs
    bool solo = false;     // decided at admission: one CTA running the solo engine
    bool cluster = false;  // team as one thread-block cluster (no hub row)
    int ctas = 1;       // CTAs of its launch (team size, or 1)
    int units = 1;      // share of the GPU it holds (see pbrcm_session::units_per_sm)
    int stream = 0;
    cudaEvent_t ev = nullptr;     // the result is back in the staging
    cudaEvent_t ev_in = nullptr;  // the CSR is in device memory
    bool copied = false;          // ev_in seen complete (the worker's own flag)
    int state = 0;  // 0 queued, 1 copying in or running, 2 done
    bool launched = false;
    int32_t rc = PBRCM_OK;
    // once done: the result and permutation, moved out of the pinned staging
    // (which goes back to the pool at once, for the next submissions)
    DevResult res_done{};
    std::vector<uint32_t> perm_done;
    Clock::time_point t_submit, t_copy, t_launch, t_done;
    float stage_ms = 0.f;  // host time of the submit-time staging copy
    float get_ms = 0.f;    // ... of taking the staging and events (the session lock included)
};

}  // namespace

struct pbrcm_session {
    Context* C = nullptr;
    uint64_t cap_bytes = 0;
    uint32_t max_inflight = 0;
    std::vector<cudaStream_t> streams;
    std::vector<int> stream_busy;  // requests in flight per stream
    int small_pool = 0;            // shape of one-CTA requests (kPools 0, 4 or 5: 512, 128 or 256 threads)
    uint32_t team_cutoff_n = 1u << 18;
    int max_ctas = 0;              // largest team (co-resident CTAs of the team kernel)
    // GPU share in units: an SM holds units_per_sm one-CTA requests, or one
    // CTA of a team (which takes a whole SM)
    int units_per_sm = 1;
    int cap_ctas = 0;              // units the running requests may hold together
    int ctas_in_use = 0;           // units held
    int team_min = 2, team_max = 64;
    int idle_team = 0;             // team of a large request that finds the GPU idle (0 = no boost)
    // largest cluster team (0: cooperative teams only).  A big request whose
    // rows fit a CTA's chunk runs as one thread-block cluster of up to this
    // many CTAs (hardware cluster barrier, all-gather in distributed shared
    // memory; a plain launch beside the others): on the Poisson mix all at
    // once, 884 / 840 reorders/s with clusters of up to 16 / 8 CTAs against
    // 726 with cooperative teams only
    int cluster_max = 16;
    // entries per team CTA (measured on the Poisson mix all at once: 2^20
    // with teams of at least 2 CTAs served 630-692 reorders/s, 2^19 with at
    // least 4 served 630-661, 2^21 served 551)
    uint64_t team_nnz = 1ull << 20;
    uint32_t light_team_n = 1u << 14;  // under light load, requests above this many nodes get a team
    bool big_solo = false;  // under load, big requests run as one solo CTA too (PBRCM_SESSION_BIG_SOLO)
    bool solo_kernel = false;  // one-CTA solo requests launch the solo batch kernel

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> queued;
    std::vector<Request*> copying;  // device memory held, CSR on its way in (arrival order)
    std::vector<Request*> running;  // kernel launched
    size_t admitting = 0;  // being started by the worker (in no list)
    std::unordered_map<uint64_t, Request*> all;
    uint64_t next_ticket = 1;
    uint64_t bytes_in_flight = 0, peak_bytes = 0;
    uint64_t submitted = 0, completed = 0;
    std::vector<double> lat_ms;
    Clock::time_point t_first{}, t_last{};
    bool have_first = false;
    std::shared_ptr<PinnedPool> pinned_pool = std::make_shared<PinnedPool>();  // the context's (see PinnedPool)
    std::unique_ptr<CopyPool> copy_pool;  // submit-time staging copies (PBRCM_SESSION_COPY_THREADS, 0: none)
    std::vector<cudaEvent_t> free_events;  // events of retired requests, for reuse
    std::atomic<bool> stop{false};
    std::thread worker;
    // PBRCM_SESSION_TRACE=<path>: one CSV line per request (written when the
    // session is destroyed): size, how it ran, and its host-clock times
    std::string trace_path;
    std::vector<std::string> trace;
    cudaMemPool_t pool = nullptr;

    void run();
    bool start_copy(Request* r);
    bool launch(Request* r);
    void fail(Request* r);
    void collect(Request* r);
    void retire(Request* r);
    void decide_mode(Request* r) const;
    int choose_ctas(const Request* r) const;
};

namespace {

size_t device_bytes(uint32_t n, uint64_t nnz, bool hub, bool solo, int team_ctas, size_t* offs)
{
    // room for either way a request may run (decided at admission): team
    // words and hub scratch for a team, edge records (and a global visited
    // bitmap over kSoloMaxN nodes) for the solo engine
    size_t o = 0;
    offs[0] = o;  // rp
    o = align16(o + 4 * ((size_t)n + 1));
    offs[1] = o;  // ci
    o = align16(o + 4 * (size_t)nnz);
    offs[2] = o;  // node table
    o = align16(o + 16 * (size_t)n);
    offs[3] = o;  // rec
    o = align16(o + 16 * (size_t)n);
    offs[4] = o;  // perm
    o = align16(o + 4 * (size_t)n);
    offs[5] = o;  // res
    o = align16(o + sizeof(DevResult));
    offs[6] = (o + 127) & ~(size_t)127;  // gs
    o = offs[6] + sizeof(GridSync);
    offs[7] = o;  // counter, then one BatchJob and one BatchSlot
    o = align16(o + 16 + sizeof(BatchJob) + sizeof(BatchSlot));
    offs[8] = o;  // agg (2 words per team CTA)
    o = align16(o + team_words_bytes(team_ctas));
    offs[9] = o;  // hub
    if (hub)
        o = align16(o + 16 * std::max<uint64_t>(nnz, 1));
    offs[10] = o;  // the solo engine's edge records
    if (solo)
        o = align16(o + 8 * std::max<uint64_t>(nnz, 1));
    offs[11] = o;  // its visited bitmap, when it does not fit shared memory
    if (solo && n > kSoloMaxN)
        o = align16(o + 4 * (((size_t)n + 31) / 32));
    return o;
}

}  // namespace

// Copies a CSR into its staging (rp_out, ci_out) and returns its longest
// row; requests of 4 MB or more are cut into slices of about 1 MB (rows of
// row_ptr with their valences, entries of col_idx) for the copy threads.
static uint32_t copy_csr(pbrcm_session* s, const uint32_t* row_ptr, const uint32_t* col_idx, uint32_t n, uint64_t nnz,
                  uint32_t* rp_out, uint32_t* ci_out)
{
    const size_t bytes = 4 * ((size_t)n + 1 + nnz);
    const int parts = s->copy_pool && bytes >= ((size_t)4 << 20)
                          ? (int)std::min<size_t>((size_t)s->copy_pool->threads() + 1, bytes >> 20)
                          : 1;
    std::vector<uint32_t> md((size_t)parts, 0u);
    auto slice = [&](int p) {
        const uint64_t a = (uint64_t)n * p / parts, b = (uint64_t)n * (p + 1) / parts;
        uint32_t m = 0;
        for (uint64_t i = a; i < b; ++i)
            m = std::max(m, row_ptr[i + 1] - row_ptr[i]);
        md[(size_t)p] = m;
        std::memcpy(rp_out + a, row_ptr + a, 4 * (size_t)(b - a + (p == parts - 1 ? 1 : 0)));
        const uint64_t c = nnz * p / parts, d = nnz * (p + 1) / parts;
        if (d > c)
            std::memcpy(ci_out + c, col_idx + c, 4 * (size_t)(d - c));
    };
    if (parts == 1)
        slice(0);
    else
        s->copy_pool->run(parts, slice);
    return *std::max_element(md.begin(), md.end());
}

// Stage 1 of a request (admitted by device memory): its device block and
// the CSR's copy in, on its own stream; ev_in marks the copy done.  It holds
// no CTAs yet, so that copies queued behind the copy engines never keep SMs
// idle.
bool pbrcm_session::start_copy(Request* r)
{
    cudaStream_t st = streams[r->stream];
    if (cudaMallocFromPoolAsync(reinterpret_cast<void**>(&r->dev), r->dev_bytes, pool, st) != cudaSuccess)
        return false;
    unsigned char* D = r->dev;
    bool ok = cudaMemcpyAsync(D + r->d_rp, r->host + r->off_rp, 4 * ((size_t)r->n + 1), cudaMemcpyHostToDevice,
                              st) == cudaSuccess;
    if (r->nnz)
        ok = ok && cudaMemcpyAsync(D + r->d_ci, r->host + r->off_ci, 4 * (size_t)r->nnz, cudaMemcpyHostToDevice,
                                   st) == cudaSuccess;
    ok = ok && cudaEventRecord(r->ev_in, st) == cudaSuccess;
    return ok;
}

// Stage 2 (admitted by CTAs once its CSR is in): the kernel in the mode
// decide_mode chose, then the permutation and result back to the staging;
// ev marks them there.
bool pbrcm_session::launch(Request* r)
{
    cudaStream_t st = streams[r->stream];
    Context& c = *C;
    unsigned char* D = r->dev;
    MatrixView M{};
    M.rp = reinterpret_cast<const uint32_t*>(D + r->d_rp);
    M.ci = reinterpret_cast<const uint32_t*>(D + r->d_ci);
    M.n = r->n;
    M.nnz = (uint32_t)r->nnz;
    M.node = reinterpret_cast<NodeEntry*>(D + r->d_node);
    M.rec = reinterpret_cast<PosRec*>(D + r->d_rec);
    M.perm = reinterpret_cast<uint32_t*>(D + r->d_perm);
    M.hub = r->team && r->maxdeg > (uint32_t)kVariants[c.team_variant].emax
                ? reinterpret_cast<uint32_t*>(D + r->d_hub)
                : nullptr;
    M.res = reinterpret_cast<DevResult*>(D + r->d_res);
    BatchJob J{};
    J.M = M;
    J.team = 1;
    if (r->solo) {
        J.e2 = reinterpret_cast<uint2*>(D + r->d_e2);
        J.inv = reinterpret_cast<uint32_t*>(D + r->d_node);
        J.gvis = r->n > kSoloMaxN ? reinterpret_cast<uint32_t*>(D + r->d_gvis) : nullptr;
    }
    const BatchSlot one{0, 0};
    std::memcpy(r->host + r->off_view, &J, sizeof(J));
    std::memcpy(r->host + r->off_view + sizeof(J), &one, sizeof(one));
    BatchJob* d_job = reinterpret_cast<BatchJob*>(D + r->d_cnt + 16);
    BatchSlot* d_slot = reinterpret_cast<BatchSlot*>(D + r->d_cnt + 16 + sizeof(BatchJob));
    uint32_t* d_counter = reinterpret_cast<uint32_t*>(D + r->d_cnt);
    bool ok = cudaMemsetAsync(D + r->d_res, 0, sizeof(DevResult), st) == cudaSuccess;
    ok = ok && cudaMemsetAsync(D + r->d_gs, 0, sizeof(GridSync), st) == cudaSuccess;
    if (r->team)
        ok = ok && cudaMemsetAsync(D + r->d_agg, 0, team_words_bytes(r->ctas), st) == cudaSuccess;
    ok = ok && cudaMemsetAsync(d_counter, 0, 16, st) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(d_job, r->host + r->off_view, sizeof(BatchJob) + sizeof(BatchSlot),
                               cudaMemcpyHostToDevice, st) == cudaSuccess;
    // the batch and cluster kernels check the CSR themselves; the team
    // kernel needs the separate check first
    if (r->team && !r->cluster)
        ok = ok && launch_validate(M.rp, M.ci, M.n, M.nnz, M.res, c.sms, st) == cudaSuccess;
    if (r->cluster) {
        // one thread-block cluster: no cooperative launch, so it runs beside
        // the other requests' kernels
        Options copt = r->opt;
        copt.solo_parents = c.cluster_solo_parents;
        copt.solo_edges = c.cluster_solo_edges;
        ok = ok && launch_cluster(small_pool, d_job, 1, d_slot, 0, d_counter, copt, r->opt, r->ctas, 1, st) ==
                       cudaSuccess;
    } else if (r->team)
        ok = ok && launch_team(c.team_variant, M, r->opt, reinterpret_cast<GridSync*>(D + r->d_gs),
                               reinterpret_cast<unsigned long long*>(D + r->d_agg), r->ctas, st) == cudaSuccess;
    else if (r->solo && solo_kernel)
        ok = ok && launch_solo(small_pool, d_job, d_slot, 1, d_counter, r->opt, 1, st) == cudaSuccess;
    else
        ok = ok && launch_batch(small_pool, d_job, d_slot, 1, d_counter, r->opt, 1, false, st) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(r->host + r->off_perm, M.perm, 4 * (size_t)r->n, cudaMemcpyDeviceToHost, st) ==
                   cudaSuccess;
    ok = ok && cudaMemcpyAsync(r->host + r->off_res, M.res, sizeof(DevResult), cudaMemcpyDeviceToHost, st) ==
                   cudaSuccess;
    ok = ok && cudaFreeAsync(r->dev, st) == cudaSuccess;
    ok = ok && cudaEventRecord(r->ev, st) == cudaSuccess;
    return ok;
}

// A request whose copy or launch could not be issued: done with
// PBRCM_ERR_CUDA, its share released (under the session lock).
void pbrcm_session::fail(Request* r)
{
    r->rc = PBRCM_ERR_CUDA;
    r->state = 2;
    r->t_done = Clock::now();
    bytes_in_flight -= r->dev_bytes;
    ctas_in_use -= r->units;
    r->units = 0;
    stream_busy[r->stream] -= 1;
    ++completed;
}

// A finished request's result and permutation out of its pinned staging
// (the worker calls this without the session lock: nothing else touches a
// running request's staging).
void pbrcm_session::collect(Request* r)
{
    r->t_done = Clock::now();
    DevResult& res = r->res_done;
    std::memcpy(&res, r->host + r->off_res, sizeof(res));
    r->rc = map_status(res.status);
    if (r->rc == PBRCM_OK)
        r->perm_done.assign(reinterpret_cast<const uint32_t*>(r->host + r->off_perm),
                            reinterpret_cast<const uint32_t*>(r->host + r->off_perm) + r->n);
}

// Bookkeeping of a collected request (under the session lock): staging and
// event back to their pools, the GPU share it held released.
void pbrcm_session::retire(Request* r)
{
    const DevResult& res = r->res_done;
    pinned_pool->put(r->host, r->host_cap);
    r->host = nullptr;
    free_events.push_back(r->ev);
    free_events.push_back(r->ev_in);
    r->ev = nullptr;
    r->ev_in = nullptr;
    r->state = 2;
    if (!trace_path.empty()) {
        auto ms = [&](Clock::time_point t) { return std::chrono::duration<double, std::milli>(t - t_first).count(); };
        char line[256];
        std::snprintf(line, sizeof(line), "%u,%llu,%s,%d,%.3f,%.3f,%.3f,%.3f,%.3f,%.3f,%.3f", r->n,
                      (unsigned long long)r->nnz,
                      r->cluster ? "cluster" : r->team ? "team" : r->solo ? "solo" : "cta", r->ctas, ms(r->t_submit),
                      ms(r->t_copy), ms(r->t_launch), ms(r->t_done),
                      res.t_end > res.t_begin ? (double)(res.t_end - res.t_begin) * 1e-6 : -1.0, (double)r->stage_ms,
                      (double)r->get_ms);
        trace.emplace_back(line);
    }
    bytes_in_flight -= r->dev_bytes;
    ctas_in_use -= r->units;
    stream_busy[r->stream] -= 1;
    ++completed;
    lat_ms.push_back(std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count());
    t_last = std::max(t_last, r->t_done);
}

// How a request runs, decided when it is admitted.  A request above the
// cutoff (or with a row longer than a one-CTA chunk) gets a cooperative team:
// on one CTA its thousands of BFS levels would set the p99 (measured: the
// Poisson mix served 125 reorders/s with them on single CTAs, 220-260 with
// teams).  A mid-size request that finds the GPU lightly loaded also gets a
// team, for latency; under load it runs on one CTA (the solo engine where it
// applies), which spends far fewer SM-seconds per request.
void pbrcm_session::decide_mode(Request* r) const
{
    const bool light = ctas_in_use * 4 < cap_ctas && queued.size() <= 2;
    r->team = (r->big && (!r->solo_able || !big_solo || light)) || (light && r->n > light_team_n);
    r->solo = !r->team && r->solo_able;
    r->cluster = r->team && cluster_max >= 2 && r->maxdeg <= (uint32_t)kPools[small_pool].gemax;
}

// CTAs of a request: 1 for a small matrix; for a large one a team that grows
// with its nnz (team_min..team_max) -- small teams spend far fewer CTA-seconds
// per BFS level than the whole GPU -- or, if idle_team is set and nothing else
// is running or waiting, idle_team CTAs for a lower latency.
int pbrcm_session::choose_ctas(const Request* r) const
{
    if (!r->team)
        return 1;
    if (r->cluster) {
        // a power of two up to cluster_max, growing with nnz like a team
        const uint64_t k = (r->nnz + team_nnz - 1) / team_nnz;
        const int t = (int)std::max<uint64_t>((uint64_t)team_min, std::min<uint64_t>(k, (uint64_t)cluster_max));
        int c = 2;
        while (c * 2 <= t)
            c *= 2;
        return c;
    }
    if (idle_team > 0 && running.empty() && queued.size() <= 1)
        return std::max(1, std::min(std::min(idle_team, max_ctas), cap_ctas));
    const uint64_t k = (r->nnz + team_nnz - 1) / team_nnz;
    const int t = (int)std::max<uint64_t>((uint64_t)team_min, std::min<uint64_t>(k, (uint64_t)team_max));
    return std::max(1, std::min(t, max_ctas));
}

// The worker, in two stages per request: a queued request is admitted by
// device memory (start_copy: its CSR goes in on its own stream), then, once
// the copy is done, by CTAs (launch: decide_mode picks how it runs).  It
// retires finished requests.  The CUDA calls (event queries, copies and
// launches) and the result copies run without the session lock, so that
// submit() and poll() from other threads never wait behind them.
void pbrcm_session::run()
{
    cudaSetDevice(C->device);
    std::vector<Request*> snap_run, snap_copy, fin, to_copy, to_launch;
    std::unique_lock<std::mutex> lk(mu);
    while (!stop.load()) {
        snap_run.assign(running.begin(), running.end());
        snap_copy.assign(copying.begin(), copying.end());
        lk.unlock();
        fin.clear();
        for (Request* r : snap_run)
            if (cudaEventQuery(r->ev) == cudaSuccess)
                fin.push_back(r);
        bool newly_copied = false;
        for (Request* r : snap_copy)
            if (!r->copied && cudaEventQuery(r->ev_in) == cudaSuccess) {
                r->copied = true;
                newly_copied = true;
            }
        for (Request* r : fin)
            collect(r);
        lk.lock();
        for (Request* r : fin) {
            retire(r);
            running.erase(std::find(running.begin(), running.end(), r));
        }
        // stage 1, by device memory, in arrival order
        to_copy.clear();
        while (!queued.empty() && copying.size() + running.size() + to_copy.size() < max_inflight) {
            Request* r = queued.front();
            const bool idle = running.empty() && copying.empty() && to_copy.empty();
            if (bytes_in_flight + r->dev_bytes > cap_bytes && !idle)
                break;
            int free_stream = -1;
            for (size_t k = 0; k < stream_busy.size(); ++k)
                if (stream_busy[k] == 0) {
                    free_stream = (int)k;
                    break;
                }
            if (free_stream < 0)
                break;
            queued.pop_front();
            r->stream = free_stream;
            r->units = 0;
            stream_busy[free_stream] += 1;
            bytes_in_flight += r->dev_bytes;
            peak_bytes = std::max(peak_bytes, bytes_in_flight);
            r->state = 1;
            to_copy.push_back(r);
        }
        // stage 2, by CTAs: the copied requests in arrival order, until one
        // does not fit (capping the team requests that run at once, to spare
        // L2, measured 217-381 reorders/s against 694 on the Poisson mix)
        to_launch.clear();
        for (Request* r : copying) {
            if (!r->copied)
                continue;
            decide_mode(r);
            const int need = choose_ctas(r);
            const int units = r->team && !r->cluster ? need * units_per_sm : need;
            if (ctas_in_use + units > cap_ctas && !(running.empty() && to_launch.empty()))
                break;
            r->ctas = need;
            r->units = units;
            ctas_in_use += units;
            to_launch.push_back(r);
        }
        for (Request* r : to_launch)
            copying.erase(std::find(copying.begin(), copying.end(), r));
        if (!to_copy.empty() || !to_launch.empty()) {
            admitting = to_copy.size() + to_launch.size();
            lk.unlock();
            for (Request* r : to_copy) {
                r->t_copy = Clock::now();
                r->launched = start_copy(r);
            }
            for (Request* r : to_launch) {
                r->t_launch = Clock::now();
                r->launched = launch(r);
            }
            lk.lock();
            admitting = 0;
            for (Request* r : to_copy) {
                if (r->launched)
                    copying.push_back(r);
                else
                    fail(r);
            }
            for (Request* r : to_launch) {
                if (r->launched)
                    running.push_back(r);
                else
                    fail(r);
            }
        }
        const bool progress = !fin.empty() || !to_copy.empty() || !to_launch.empty() || newly_copied;
        if (progress)
            cv_done.notify_all();
        if (running.empty() && copying.empty() && queued.empty())
            cv_work.wait(lk, [&] { return stop.load() || !queued.empty(); });
        else if (!progress) {
            lk.unlock();
            std::this_thread::sleep_for(std::chrono::microseconds(20));
            lk.lock();
        }
    }
}

extern "C" {

int32_t pbrcm_session_create(pbrcm_context* ctx, const pbrcm_session_config* cfg, pbrcm_session** out)
{
    if (!ctx || !out)
        return PBRCM_ERR_ARG;
    *out = nullptr;
    auto* s = new (std::nothrow) pbrcm_session();
    if (!s)
        return PBRCM_ERR_OOM;
    s->C = &ctx->ctx;
    cudaSetDevice(s->C->device);
    {
        std::lock_guard<std::mutex> lk(s->C->mu);
        if (s->C->session_pinned)
            s->pinned_pool = std::static_pointer_cast<PinnedPool>(s->C->session_pinned);
        else
            s->C->session_pinned = s->pinned_pool;
    }
    s->cap_bytes = cfg && cfg->memory_cap_bytes ? cfg->memory_cap_bytes : 120ull * 1000 * 1000 * 1000;
    s->max_inflight = cfg && cfg->max_inflight ? cfg->max_inflight : 4096;
    const uint32_t ns = cfg && cfg->streams ? std::min<uint32_t>(cfg->streams, 128) : 64;
    for (uint32_t i = 0; i < ns; ++i) {
        cudaStream_t st;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
            delete s;
            return PBRCM_ERR_CUDA;
        }
        s->streams.push_back(st);
    }
    s->small_pool = s->C->session_pool;
    s->team_cutoff_n = s->C->session_cutoff_n;
    s->max_ctas = std::max(1, team_max_ctas(s->C->team_variant, s->C->sms));
    // one-CTA requests on the solo batch kernel where the shape has one (it
    // may fit more CTAs on an SM than the general kernel)
    const int solo_cap = s->C->solo && s->C->batch_solo_kernel ? solo_max_ctas(s->small_pool, s->C->sms) : 0;
    s->solo_kernel = solo_cap > 0;
    s->cap_ctas = std::max(1, s->solo_kernel ? solo_cap : batch_max_ctas(s->small_pool, s->C->sms));
    s->units_per_sm = std::max(1, s->cap_ctas / std::max(1, s->C->sms));
    s->stream_busy.assign(s->streams.size(), 0);
    s->team_nnz = std::max<uint64_t>(1, s->C->session_team_nnz);  // context: tuned, or PBRCM_SESSION_TEAM_NNZ
    s->cluster_max = s->C->session_cluster_max;                    // ... or PBRCM_SESSION_CLUSTER_MAX
    if (const char* e = std::getenv("PBRCM_SESSION_TEAM_MIN"))
        s->team_min = std::max(1, std::atoi(e));
    if (const char* e = std::getenv("PBRCM_SESSION_TEAM_MAX"))
        s->team_max = std::max(s->team_min, std::atoi(e));
    if (const char* e = std::getenv("PBRCM_SESSION_IDLE_TEAM"))
        s->idle_team = std::max(0, std::atoi(e));
    if (const char* e = std::getenv("PBRCM_SESSION_BIG_SOLO"))
        s->big_solo = std::atoi(e) != 0;
    if (const char* e = std::getenv("PBRCM_SESSION_LIGHT_TEAM_N"))
        s->light_team_n = (uint32_t)std::max(1L, std::atol(e));
    {
        const unsigned hc = std::thread::hardware_concurrency();
        int ct = (int)std::min(8u, std::max(1u, hc / 2)) - 1;  // the submitting thread copies too
        if (const char* e = std::getenv("PBRCM_SESSION_COPY_THREADS"))
            ct = std::max(0, std::min(64, std::atoi(e)));
        if (ct > 0)
            s->copy_pool.reset(new (std::nothrow) CopyPool(ct));
    }
    if (const char* e = std::getenv("PBRCM_SESSION_TRACE"))
        s->trace_path = e;
    if (cudaDeviceGetDefaultMemPool(&s->pool, s->C->device) != cudaSuccess) {
        delete s;
        return PBRCM_ERR_CUDA;
    }
    uint64_t thr = ~0ull;
    cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &thr);
    s->worker = std::thread([s] { s->run(); });
    *out = s;
    return PBRCM_OK;
}

void pbrcm_session_destroy(pbrcm_session* s)
{
    if (!s)
        return;
    pbrcm_session_drain(s);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable())
        s->worker.join();
    cudaSetDevice(s->C->device);
    for (auto& kv : s->all) {
        Request* r = kv.second;
        if (r->ev)
            cudaEventDestroy(r->ev);
        if (r->ev_in)
            cudaEventDestroy(r->ev_in);
        if (r->host)
            s->pinned_pool->put(r->host, r->host_cap);
        delete r;
    }
    for (cudaEvent_t e : s->free_events)
        cudaEventDestroy(e);
    if (!s->trace_path.empty()) {
        if (FILE* f = std::fopen(s->trace_path.c_str(), "w")) {
            std::fprintf(f, "n,nnz,mode,ctas,submit_ms,copy_ms,launch_ms,done_ms,device_ms,stage_ms,get_ms\n");
            for (const std::string& l : s->trace)
                std::fprintf(f, "%s\n", l.c_str());
            std::fclose(f);
        }
    }
    for (cudaStream_t st : s->streams) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    delete s;
}

int32_t pbrcm_session_submit(pbrcm_session* s, const uint32_t* row_ptr, const uint32_t* col_idx, uint32_t n,
                             uint64_t nnz, const pbrcm_options* opts, uint64_t* ticket)
{
    if (!s || !row_ptr || (!col_idx && nnz) || !ticket || n == 0 || n == 0xFFFFFFFFu || nnz > kMaxNnz)
        return PBRCM_ERR_ARG;
    auto* r = new (std::nothrow) Request();
    if (!r)
        return PBRCM_ERR_OOM;
    r->n = n;
    r->nnz = nnz;
    r->opt = make_options(opts, kModeFull);
    apply_team_shape(*s->C, r->opt);
    r->opt.phantom = 0;
    // pinned staging: [rp | ci | view | perm_out | result]
    size_t o = 0;
    r->off_rp = o;
    o = align16(o + 4 * ((size_t)n + 1));
    r->off_ci = o;
    o = align16(o + 4 * (size_t)nnz);
    r->off_view = o;
    o = align16(o + sizeof(BatchJob) + sizeof(BatchSlot));
    r->off_perm = o;
    o = align16(o + 4 * (size_t)n);
    r->off_res = o;
    o = align16(o + sizeof(DevResult));
    const Clock::time_point t_get = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        cudaSetDevice(s->C->device);
        r->host = static_cast<unsigned char*>(s->pinned_pool->get(o, r->host_cap));
        for (cudaEvent_t* e : {&r->ev, &r->ev_in}) {
            if (!s->free_events.empty()) {
                *e = s->free_events.back();
                s->free_events.pop_back();
            } else if (cudaEventCreateWithFlags(e, cudaEventDisableTiming) != cudaSuccess) {
                *e = nullptr;
            }
        }
        if (!r->host || !r->ev || !r->ev_in) {
            s->pinned_pool->put(r->host, r->host_cap);
            for (cudaEvent_t e : {r->ev, r->ev_in})
                if (e)
                    s->free_events.push_back(e);
            delete r;
            return PBRCM_ERR_OOM;
        }
    }
    // the CSR into the staging and its longest row, in slices on the copy
    // threads when it is large
    const Clock::time_point t_stage = Clock::now();
    r->get_ms = (float)std::chrono::duration<double, std::milli>(t_stage - t_get).count();
    r->maxdeg = copy_csr(s, row_ptr, col_idx, n, nnz, reinterpret_cast<uint32_t*>(r->host + r->off_rp),
                         reinterpret_cast<uint32_t*>(r->host + r->off_ci));
    r->stage_ms = (float)std::chrono::duration<double, std::milli>(Clock::now() - t_stage).count();
    const uint32_t maxdeg = r->maxdeg;
    const int emax_small = kPools[s->small_pool].gemax;
    r->big = n > s->team_cutoff_n || maxdeg > (uint32_t)emax_small;
    r->solo_able = s->C->solo && nnz > 0 && maxdeg <= (uint32_t)emax_small && n <= kSoloMaxNodes;
    size_t offs[12];
    // any request may get a team at admission: room for its words (and hub
    // scratch for a row longer than the team kernel's chunk)
    r->dev_bytes = device_bytes(n, nnz, maxdeg > (uint32_t)kVariants[s->C->team_variant].emax, r->solo_able,
                                s->max_ctas, offs);
    r->d_rp = offs[0];
    r->d_ci = offs[1];
    r->d_node = offs[2];
    r->d_rec = offs[3];
    r->d_perm = offs[4];
    r->d_res = offs[5];
    r->d_gs = offs[6];
    r->d_cnt = offs[7];
    r->d_agg = offs[8];
    r->d_hub = offs[9];
    r->d_e2 = offs[10];
    r->d_gvis = offs[11];
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (r->dev_bytes > s->cap_bytes) {
            s->pinned_pool->put(r->host, r->host_cap);
            s->free_events.push_back(r->ev);
            s->free_events.push_back(r->ev_in);
            delete r;
            return PBRCM_ERR_BUSY;
        }
        r->ticket = s->next_ticket++;
        r->t_submit = Clock::now();
        if (!s->have_first) {
            s->t_first = r->t_submit;
            s->have_first = true;
        }
        s->all[r->ticket] = r;
        s->queued.push_back(r);
        ++s->submitted;
        *ticket = r->ticket;
    }
    s->cv_work.notify_all();
    return PBRCM_OK;
}

int32_t pbrcm_session_poll(pbrcm_session* s, uint64_t ticket, uint32_t* perm_out, pbrcm_result* result,
                           int32_t* done)
{
    if (!s || !done)
        return PBRCM_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(ticket);
    if (it == s->all.end())
        return PBRCM_ERR_NOT_FOUND;
    Request* r = it->second;
    if (r->state != 2) {
        *done = 0;
        return PBRCM_OK;
    }
    *done = 1;
    const DevResult& res = r->res_done;
    if (perm_out && r->rc == PBRCM_OK)
        std::memcpy(perm_out, r->perm_done.data(), 4 * (size_t)r->n);
    if (result) {
        fill_result(res, r->opt, result);
        result->total_ms = (float)std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
        // the kernel's own %globaltimer stamps
        result->device_ms = res.t_end > res.t_begin ? (float)((res.t_end - res.t_begin) * 1e-6) : 0.f;
    }
    int32_t rc = r->rc;
    s->all.erase(it);
    delete r;
    return rc;
}

int32_t pbrcm_session_drain(pbrcm_session* s)
{
    if (!s)
        return PBRCM_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_done.wait(lk, [&] {
        return s->queued.empty() && s->copying.empty() && s->running.empty() && s->admitting == 0;
    });
    return PBRCM_OK;
}

int32_t pbrcm_session_stats_get(pbrcm_session* s, pbrcm_session_stats* st)
{
    if (!s || !st)
        return PBRCM_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(st, 0, sizeof(*st));
    st->submitted = s->submitted;
    st->completed = s->completed;
    st->bytes_in_flight = s->bytes_in_flight;
    st->peak_bytes_in_flight = s->peak_bytes;
    if (!s->lat_ms.empty()) {
        std::vector<double> v = s->lat_ms;
        std::sort(v.begin(), v.end());
        auto q = [&](double f) { return v[std::min(v.size() - 1, (size_t)(f * (double)(v.size() - 1) + 0.5))]; };
        st->p50_ms = q(0.50);
        st->p99_ms = q(0.99);
        st->max_ms = v.back();
    }
    if (s->have_first && s->completed)
        st->busy_s = std::chrono::duration<double>(s->t_last - s->t_first).count();
    return PBRCM_OK;
}

}  // extern "C"
