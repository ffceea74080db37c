// engine.cuh -- device core of the B200 Cuthill-McKee engine (sm_100a).
//
// What it computes
//   The serial stable Cuthill-McKee order of the reference
//   (src/rcm_cpu.cpp:57-104): FIFO over positions; the parent at position i
//   appends its still-unvisited neighbours, stable-sorted by valence (row
//   length).  The reference's GPU_BATCH reaches it with a chain of
//   speculative batches (include/device/batchWorker.cuh); this engine reaches
//   it level by level, every CTA of a team working on one BFS level at a time.
//
// The claim key
//   Within one BFS pass the edges are numbered in queue order: edge (position
//   i, slot k) has id ebase(i) + k, where ebase(i) = sum of the valences at
//   positions < i.  Pass p owns the key range [p*kspan, p*kspan + nnz + 1]
//   (kspan = nnz + 2); edge id e maps to key base_p - 1 - e with
//   base_p = p*kspan + nnz + 1 (the start node takes base_p itself).  Every
//   frontier edge does atomicMax(node[child].claim, key).  Once a level's
//   claims are done, a node's claim is the key of the FIRST edge that reaches
//   it in queue order -- exactly the (parent, slot) that discovers it in the
//   serial algorithm, duplicate entries included -- so an edge is a child
//   edge iff node[col].claim == its key: a purely local test.  Keys of later
//   levels are smaller, so claiming for the next level never disturbs a node
//   already placed, and keys of a later pass are larger than every key of an
//   earlier one, so passes need no reset.  The key is an order-preserving
//   (parent position, slot) code; the reference's batch code
//   (batchId << 11 | offset, batchWorker.cuh:574-586) plays the same role for
//   its batches.
//
// One level (frontier = positions [a, b), edge ids [Ka, Kb))
//   collect: each CTA takes a contiguous range of parents, splits it into
//            chunks (<= B parents, <= EMAX edges), reads one node entry per
//            edge (claim + row start + valence in one 16-byte load), keeps
//            the child edges in (parent, slot) order and ranks every
//            parent's children by (valence, slot).
//   place:   children get positions b + (children of earlier parents) + rank
//            and edge bases Kb + (valences of earlier children): records to
//            rec[], the node to perm[].
//   claim:   the placed children claim their own edges for the next level.
//   A grid team publishes per-CTA (children, valence) totals with a
//   level-tagged all-gather, places, and meets at a barrier.  Levels with a
//   small frontier run on CTA 0 alone ("solo") with block barriers only; the
//   other CTAs park at a gate until CTA 0 hands a large level back.  Parents
//   with more than EMAX edges ("hubs") are collected and radix-sorted in
//   global scratch by one CTA.
//
// Every wait is bounded by %globaltimer and reports PBRCM_ERR_TIMEOUT.
// With PBRCM_CHECKS defined, every global index is range-checked and a
// failure records PBRCM_ERR_CHECK and skips the access.
#pragma once

#include <cstdint>
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "types.h"

namespace pbrcm {

// ---------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long globaltimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p)
{
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long* p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_relaxed64(unsigned long long* p, unsigned long long v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void st_release(unsigned int* p, unsigned int v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void red_release_add(unsigned int* p, unsigned int v)
{
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ uint32_t ld_ro(const uint32_t* p) { return __ldg(p); }

__device__ __forceinline__ uint4 ld_node(const NodeEntry* p) { return __ldcg(reinterpret_cast<const uint4*>(p)); }

// The claim word a pass uses: NodeEntry::claim (M.cf == 0) or, for the
// speculative ordered pass that runs beside a start-search pass, the word
// NodeEntry::inv (M.cf == 3; inv is only used after the last pass).
__device__ __forceinline__ uint32_t* claim_ptr(const MatrixView& M, uint32_t v)
{
    return reinterpret_cast<uint32_t*>(M.node + v) + M.cf;
}
__device__ __forceinline__ uint32_t claim_of(const MatrixView& M, const uint4& nd) { return M.cf ? nd.w : nd.x; }

__device__ __forceinline__ void set_status(DevResult* r, uint32_t code, uint32_t where)
{
    if (atomicCAS(&r->status, 0u, code) == 0u)
        r->where = where;
}

__device__ __forceinline__ uint32_t read_status(const DevResult* r)
{
    return *reinterpret_cast<const volatile uint32_t*>(&r->status);
}

#ifdef PBRCM_CHECKS
#define PB_CHECK(res, cond, where) ((cond) ? true : (set_status((res), kErrCheck, (where)), false))
#else
#define PB_CHECK(res, cond, where) true
#endif

// ---------------------------------------------------------------------------
// Thread groups.  One engine instance runs on a group of B consecutive
// threads of a CTA: the whole CTA, or one of blockDim.x / B equal slices, so
// that one CTA can reorder several matrices at once.  Group g synchronises on
// named barrier 1 + g (barrier 0 stays the CTA-wide __syncthreads); every
// engine barrier is reached by all B threads of the group, never by a
// diverged subset.
// ---------------------------------------------------------------------------
template <int B>
__device__ __forceinline__ uint32_t gtid()
{
    static_assert(B >= 32 && B <= 1024 && (B & (B - 1)) == 0, "groups are a power-of-two number of warps");
    return threadIdx.x & (B - 1);
}

template <int B>
__device__ __forceinline__ uint32_t gbar_id()
{
    return 1u + threadIdx.x / B;
}

template <int B>
__device__ __forceinline__ void gsync()
{
    asm volatile("bar.sync %0, %1;" ::"r"(gbar_id<B>()), "n"(B) : "memory");
}

// Group barrier that also counts the threads whose predicate holds.
template <int B>
__device__ __forceinline__ int gsync_count(bool pred)
{
    int r;
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.popc.u32 %0, %2, %3, p;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)pred), "r"(gbar_id<B>()), "n"(B)
        : "memory");
    return r;
}

// Barrier of a group given at run time (id, threads).
__device__ __forceinline__ void gsync_n(uint32_t id, uint32_t nthr)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthr) : "memory");
}

// Block-wide exclusive scan of one value per thread (T = uint32_t or
// unsigned long long).  `tmp` holds B/32 + 1 entries.  Ends with a barrier,
// so `tmp` can be reused right away.
template <int B, typename T>
__device__ __forceinline__ T block_exclusive_scan(T v, T& total, T* tmp)
{
    constexpr int W = B / 32;
    const int lane = threadIdx.x & 31, w = gtid<B>() >> 5;
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(kFull, x, o);
        if (lane >= o)
            x += y;
    }
    if (lane == 31)
        tmp[w] = x;
    gsync<B>();
    if (w == 0) {
        T s = lane < W ? tmp[lane] : T(0);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T y = __shfl_up_sync(kFull, s, o);
            if (lane >= o)
                s += y;
        }
        if (lane < W)
            tmp[lane] = s;
    }
    gsync<B>();
    T r = (w ? tmp[w - 1] : T(0)) + x - v;
    total = tmp[W - 1];
    gsync<B>();
    return r;
}

// Block-wide exclusive scan with a single barrier.  `buf` (B/32 entries) must
// belong to this call site alone: it is read after the barrier and not
// cleared, so the next write to it must come after another block barrier.
template <int B>
__device__ __forceinline__ uint32_t block_scan1(uint32_t v, uint32_t& total, uint32_t* buf)
{
    constexpr int W = B / 32;
    const int lane = threadIdx.x & 31, w = gtid<B>() >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, x, o);
        if (lane >= o)
            x += y;
    }
    if (lane == 31)
        buf[w] = x;
    gsync<B>();
    uint32_t before = 0, all = 0;
#pragma unroll
    for (int i = 0; i < W; ++i) {
        const uint32_t b = buf[i];
        before += i < w ? b : 0u;
        all += b;
    }
    total = all;
    return before + x - v;
}

template <int B, typename T>
__device__ __forceinline__ T block_reduce_max(T v, T* tmp)
{
    constexpr int W = B / 32;
    const int lane = threadIdx.x & 31, w = gtid<B>() >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        T y = __shfl_xor_sync(kFull, v, o);
        v = v > y ? v : y;
    }
    if (lane == 0)
        tmp[w] = v;
    gsync<B>();
    T r = tmp[0];
    for (int i = 1; i < W; ++i)
        r = r > tmp[i] ? r : tmp[i];
    gsync<B>();
    return r;
}

template <int B, typename T>
__device__ __forceinline__ T block_reduce_sum(T v, T* tmp)
{
    constexpr int W = B / 32;
    const int lane = threadIdx.x & 31, w = gtid<B>() >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(kFull, v, o);
    if (lane == 0)
        tmp[w] = v;
    gsync<B>();
    T r = 0;
    for (int i = 0; i < W; ++i)
        r += tmp[i];
    gsync<B>();
    return r;
}

// Two sums at once (tmp holds 2 * (B/32) entries).
template <int B>
__device__ __forceinline__ void block_reduce_sum2(unsigned long long& a, unsigned long long& b,
                                                  unsigned long long* tmp)
{
    constexpr int W = B / 32;
    const int lane = threadIdx.x & 31, w = gtid<B>() >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(kFull, a, o);
        b += __shfl_xor_sync(kFull, b, o);
    }
    if (lane == 0) {
        tmp[w] = a;
        tmp[W + w] = b;
    }
    gsync<B>();
    unsigned long long ra = 0, rb = 0;
    for (int i = 0; i < W; ++i) {
        ra += tmp[i];
        rb += tmp[W + i];
    }
    a = ra;
    b = rb;
    gsync<B>();
}

// Level state of one pass, the same in every CTA of a team.
constexpr int kTeamShared = 12;  // group-shared ints a team needs (Team::sh)

struct LevelState {
    uint32_t a, b;     // frontier positions [a, b)
    uint32_t Ka, Kb;   // edge ids of the frontier [Ka, Kb)
    uint32_t L;        // level index of the frontier
    uint32_t last_start;
};

// ---------------------------------------------------------------------------
// Team: one CTA, or all CTAs of a cooperative launch (global-memory
// barriers, all-gather and gate, every wait bounded by wait_ns).
// ---------------------------------------------------------------------------
struct Team {
    static constexpr bool kGrid = true;
    GridSync* gs;        // nullptr for a one-CTA team
    unsigned int* flags; // one barrier flag word per CTA (+ phantom), zeroed per launch
    uint32_t size;       // CTAs in the team
    uint32_t rank;       // this CTA
    uint32_t expected;   // CTAs a barrier waits for (size + phantom)
    uint32_t target;     // barriers passed so far
    uint32_t mode;       // barrier implementation (see sync)
    uint32_t epoch;      // gate epochs seen
    unsigned long long wait_ns;
    DevResult* res;
    // the thread group running this CTA's part (see gtid): its thread 0 is
    // tid == 0, its barrier is (bar, nthr); sh holds kTeamShared ints of
    // group-shared scratch, one slot per function so that one function's
    // result can still be read while the next one writes its own
    uint32_t tid, bar, nthr;
    int* sh;

    __device__ __forceinline__ void gbar() const { gsync_n(bar, nthr); }

    // Group-uniform "keep going?" after a group barrier.
    __device__ bool block_ok()
    {
        gbar();
        if (tid == 0)
            sh[0] = read_status(res) == 0;
        gbar();
        return sh[0] != 0;
    }

    // Team barrier, two implementations (Options::barrier):
    //  0  monotonic counter: one release-add per CTA on gs->count, thread 0
    //     acquire-polls until it reaches (barriers so far) x (team size);
    //  1  flag array: every CTA release-stores the barrier's sequence number
    //     into its own flag word; threads i < expected poll flag i with
    //     relaxed loads, then fence (acquire pattern).
    // Returns false if the team must stop (an error anywhere, or the wait
    // ran out).
    __device__ bool sync(uint32_t where)
    {
        if (gs == nullptr)
            return block_ok();
        target += 1;
        // this barrier's verdict, in one of two slots by parity (the next
        // barrier resets the other one, so no thread reading this one meets
        // the reset and no barrier is needed after the read)
        int& s_ok = sh[(target & 1u) ? 1 : 10];
        if (tid == 0)
            s_ok = 1;
        gbar();
        if (mode == 0) {
            if (tid == 0) {
                red_release_add(&gs->count, 1u);
                // the status read goes out with the polls, not after them:
                // an error posted before this CTA arrived is seen here, one
                // posted later at the next barrier or bounded wait (each
                // checks the status)
                const uint32_t st0 = read_status(res);
                const uint32_t goal = target * expected;
                unsigned long long t0 = 0;
                uint32_t spins = 0;
                while ((int)(ld_acquire(&gs->count) - goal) < 0) {
                    if ((++spins & 31u) == 0 && !wait_check(t0, where)) {
                        s_ok = 0;
                        break;
                    }
                    if (spins > 2048)
                        __nanosleep(128);
                }
                if (st0 != 0)
                    s_ok = 0;
            }
            gbar();
            return s_ok != 0;
        } else {
            if (tid == 0)
                st_release(flags + rank, target);
            for (uint32_t i = tid; i < expected; i += nthr) {
                unsigned long long t0 = 0;
                uint32_t spins = 0;
                while ((int)(*reinterpret_cast<volatile unsigned int*>(flags + i) - target) < 0) {
                    if ((++spins & 31u) == 0 && !wait_check(t0, where)) {
                        s_ok = 0;
                        break;
                    }
                    if (spins > 256)
                        __nanosleep(64);
                }
                __threadfence();
            }
        }
        gbar();
        const int ok = s_ok && read_status(res) == 0;
        gbar();
        return ok != 0;
    }

    // Shared by every bounded wait: false once an error is posted or the
    // wait has run longer than wait_ns (then it posts PBRCM_ERR_TIMEOUT).
    __device__ __forceinline__ bool wait_check(unsigned long long& t0, uint32_t where)
    {
        if (read_status(res) != 0)
            return false;
        const unsigned long long now = globaltimer();
        if (t0 == 0) {
            t0 = now;
        } else if (now - t0 > wait_ns) {
            set_status(res, kErrTimeout, where);
            return false;
        }
        return true;
    }

    // Heartbeat of CTA 0's solo run (keeps the gate waiters' bound fresh).
    __device__ __forceinline__ void beat()
    {
        if (gs != nullptr && tid == 0)
            atomicAdd(&gs->heartbeat, 1u);
    }

    // Bounded wait at the gate for CTA 0 to hand a solo run back.  Thread 0
    // polls; the wait only runs out if CTA 0's heartbeat stops for wait_ns.
    __device__ bool gate_wait(LevelState& st)
    {
        int& s_ok = sh[2];
        int* s_st = sh + 3;  // 6 slots
        gbar();
        if (tid == 0) {
            int ok = 1;
            const uint32_t want = epoch + 1;
            unsigned long long t0 = globaltimer();
            uint32_t hb = *reinterpret_cast<volatile uint32_t*>(&gs->heartbeat);
            uint32_t spins = 0;
            while ((int)(ld_acquire(&gs->epoch) - want) < 0) {
                if ((++spins & 63u) == 0) {
                    if (read_status(res) != 0) {
                        ok = 0;
                        break;
                    }
                    const uint32_t h = *reinterpret_cast<volatile uint32_t*>(&gs->heartbeat);
                    const unsigned long long now = globaltimer();
                    if (h != hb) {
                        hb = h;
                        t0 = now;
                    } else if (now - t0 > wait_ns) {
                        set_status(res, kErrTimeout, 50);
                        ok = 0;
                        break;
                    }
                }
                if (spins > 1024)
                    __nanosleep(256);
            }
            if (ok)
                for (int i = 0; i < 6; ++i)
                    s_st[i] = (int)__ldcg(&gs->st[i]);
            s_ok = ok && read_status(res) == 0;
        }
        gbar();
        epoch += 1;
        if (s_ok) {
            st.a = s_st[0];
            st.b = s_st[1];
            st.Ka = s_st[2];
            st.Kb = s_st[3];
            st.L = s_st[4];
            st.last_start = s_st[5];
        }
        return s_ok != 0;
    }

    // CTA 0 publishes the state and opens the gate.  Returns whether the
    // team goes on (the waiters read the error status themselves).
    __device__ bool gate_open(const LevelState& st, bool ok)
    {
        gbar();
        if (tid == 0) {
            gs->st[0] = st.a;
            gs->st[1] = st.b;
            gs->st[2] = st.Ka;
            gs->st[3] = st.Kb;
            gs->st[4] = st.L;
            gs->st[5] = st.last_start;
            __threadfence();
            st_release(&gs->epoch, epoch + 1);
        }
        gbar();
        epoch += 1;
        return ok;
    }

    // Level all-gather, first half: this CTA's (children, edges), tagged
    // with the level's step number.
    __device__ __forceinline__ void ag_publish(uint32_t cnt, uint32_t esum, uint32_t step, unsigned long long* agg)
    {
        if (tid == 0) {
            st_relaxed64(agg + 2 * rank, ((unsigned long long)step << 32) | cnt);
            st_relaxed64(agg + 2 * rank + 1, ((unsigned long long)step << 32) | esum);
        }
    }

    // Second half: the sums over the CTAs before this one (pre) and over
    // all (all), children in the low and edges in the high 32 bits.
    template <int B>
    __device__ bool ag_collect(uint32_t step, const unsigned long long* agg, unsigned long long& pre,
                               unsigned long long& all, unsigned long long* red)
    {
        int& s_ok = sh[9];
        const uint32_t t = tid;
        pre = 0;
        all = 0;
        if (t == 0)
            s_ok = 1;
        gbar();
        for (uint32_t i = t; i < size; i += B) {
            unsigned long long vc, ve;
            unsigned long long t0 = 0;
            uint32_t spins = 0;
            while (true) {
                vc = ld_relaxed64(agg + 2 * i);
                ve = ld_relaxed64(agg + 2 * i + 1);
                if ((uint32_t)(vc >> 32) == step && (uint32_t)(ve >> 32) == step)
                    break;
                if ((++spins & 31u) == 0 && !wait_check(t0, 4)) {
                    s_ok = 0;
                    break;
                }
                if (spins > 2048)
                    __nanosleep(128);
            }
            const unsigned long long v = ((ve & 0xFFFFFFFFull) << 32) | (vc & 0xFFFFFFFFull);
            all += v;
            if (i < rank)
                pre += v;
        }
        block_reduce_sum2<B>(pre, all, red);
        return s_ok != 0;
    }
};

// ---------------------------------------------------------------------------
// ClusterTeam: the CTAs of one thread-block cluster.  The hardware cluster
// barrier (release / acquire at cluster scope) replaces the global-memory
// barrier, and the all-gather and the gate hand-over read the peers' shared
// memory (DSMEM).  A hardware barrier has no time bound, so every CTA of the
// cluster must reach every barrier: the engine takes each "stop" decision
// uniformly (from flags all CTAs read after the same barrier) and returns
// only through such decisions.
// ---------------------------------------------------------------------------
struct ClusterShared {
    unsigned long long ag[2][2];  // all-gather words by barrier phase: children, edges
    uint32_t ok[2];               // "no error seen" flag at a barrier, by phase
    uint32_t st[6];               // CTA 0: level state handed over at the gate
    uint32_t job;                 // CTA 0: the job the cluster works on
    uint32_t all_ok;              // this CTA's AND of the peers' flags
    uint32_t job_ok;              // this CTA's verdict on the job (CSR arrived and valid, no hub)
};

__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }

struct ClusterTeam {
    static constexpr bool kGrid = false;
    ClusterShared* cs;  // this CTA's
    uint32_t size;      // CTAs in the cluster
    uint32_t rank;      // this CTA's rank in the cluster
    uint32_t phase;     // cluster barriers passed (slot parity)
    DevResult* res;
    // the CTA's thread group (a cluster team always spans whole CTAs) and
    // its group-shared scratch, as in Team
    uint32_t tid, bar, nthr;
    int* sh;

    __device__ __forceinline__ void gbar() const { gsync_n(bar, nthr); }

    __device__ __forceinline__ ClusterShared* peer(uint32_t r) const
    {
        return cooperative_groups::this_cluster().map_shared_rank(cs, r);
    }

    __device__ bool block_ok()
    {
        gbar();
        if (tid == 0)
            sh[0] = read_status(res) == 0;
        gbar();
        return sh[0] != 0;
    }

    // Cluster barrier; true iff no CTA had seen an error when it arrived.
    __device__ bool sync(uint32_t)
    {
        if (size == 1)
            return block_ok();
        const uint32_t ph = phase & 1u;
        gbar();
        if (tid == 0)
            cs->ok[ph] = read_status(res) == 0 ? 1u : 0u;
        cluster_arrive();
        cluster_wait();
        if (tid == 0) {
            uint32_t a = 1;
            for (uint32_t r = 0; r < size; ++r)
                a &= peer(r)->ok[ph];
            cs->all_ok = a;
        }
        gbar();
        ++phase;
        return cs->all_ok != 0;
    }

    __device__ __forceinline__ void beat() {}

    // Every CTA but 0: wait (hardware barrier) for CTA 0 to end its solo run,
    // then take its level state and its go / stop decision.
    __device__ bool gate_wait(LevelState& st)
    {
        const uint32_t ph = phase & 1u;
        gbar();
        cluster_arrive();
        cluster_wait();
        if (tid == 0) {
            const ClusterShared* p0 = peer(0);
            cs->st[0] = p0->st[0];
            cs->st[1] = p0->st[1];
            cs->st[2] = p0->st[2];
            cs->st[3] = p0->st[3];
            cs->st[4] = p0->st[4];
            cs->st[5] = p0->st[5];
            cs->all_ok = p0->ok[ph];
        }
        gbar();
        ++phase;
        st.a = cs->st[0];
        st.b = cs->st[1];
        st.Ka = cs->st[2];
        st.Kb = cs->st[3];
        st.L = cs->st[4];
        st.last_start = cs->st[5];
        return cs->all_ok != 0;
    }

    // CTA 0: hand the state over; the decision is CTA 0's alone.
    __device__ bool gate_open(const LevelState& st, bool ok)
    {
        const uint32_t ph = phase & 1u;
        gbar();
        if (tid == 0) {
            cs->st[0] = st.a;
            cs->st[1] = st.b;
            cs->st[2] = st.Ka;
            cs->st[3] = st.Kb;
            cs->st[4] = st.L;
            cs->st[5] = st.last_start;
            cs->ok[ph] = ok && read_status(res) == 0 ? 1u : 0u;
        }
        cluster_arrive();
        cluster_wait();
        ++phase;
        return cs->ok[ph] != 0;
    }

    // All-gather, first half: publish and arrive (the caller may work before
    // ag_collect waits).
    __device__ __forceinline__ void ag_publish(uint32_t cnt, uint32_t esum, uint32_t, unsigned long long*)
    {
        const uint32_t ph = phase & 1u;
        gbar();
        if (tid == 0) {
            cs->ag[ph][0] = cnt;
            cs->ag[ph][1] = esum;
            cs->ok[ph] = read_status(res) == 0 ? 1u : 0u;
        }
        cluster_arrive();
    }

    template <int B>
    __device__ bool ag_collect(uint32_t, const unsigned long long*, unsigned long long& pre, unsigned long long& all,
                               unsigned long long* red)
    {
        const uint32_t ph = phase & 1u;
        cluster_wait();
        const uint32_t t = tid;
        pre = 0;
        all = 0;
        if (t == 0)
            cs->all_ok = 1;
        gbar();
        for (uint32_t i = t; i < size; i += B) {
            const ClusterShared* pi = peer(i);
            const unsigned long long v = (pi->ag[ph][1] << 32) | (pi->ag[ph][0] & 0xFFFFFFFFull);
            if (!pi->ok[ph])
                atomicAnd(&cs->all_ok, 0u);
            all += v;
            if (i < rank)
                pre += v;
        }
        block_reduce_sum2<B>(pre, all, red);
        ++phase;
        return cs->all_ok != 0;
    }
};

// ---------------------------------------------------------------------------
// Shared memory of one thread group (one engine instance).
// ---------------------------------------------------------------------------
template <int B, int EMAX>
struct Smem {
    static constexpr int W = B / 32;
    static constexpr int PREMAX = 4 * EMAX;  // prefetched child adjacency
    // parents of the current chunk
    uint32_t pn[B], prs[B], pdeg[B], peb[B];
    uint32_t soff[B + 1];   // edge offset of parent j inside the chunk
    uint32_t cs[B], cc[B];  // first child index / child count of parent j
    // children of the current chunk (compacted in (parent, slot) order);
    // the hub radix sort reuses this space for its per-warp digit counts
    static_assert(4 * EMAX >= W * 256, "EMAX too small for the hub counters");
    union {
        struct {
            uint32_t ch_node[EMAX], ch_deg[EMAX], ch_rs[EMAX], ch_par[EMAX];
        };
        uint32_t hcnt[W * 256];
    };
    uint32_t so_idx[EMAX];       // ranked position -> compacted index
    uint32_t so_eoff[EMAX + 1];  // edge offset of the child at ranked position
    uint32_t pre[PREMAX];        // children's adjacency loaded ahead of the all-gather
    uint32_t tmp32[W + 1];
    unsigned long long tmp64[2 * W + 2];
    unsigned long long gat64[2 * W + 2];  // all-gather reduction (its own buffer)
    uint32_t scanbuf[5][W];               // one per block_scan1 call site
    uint32_t wq[EMAX / B][W];             // collect: child edges per (round, warp)
    uint32_t hist[256];
    // chunk scalars
    uint32_t m, Ec, Q, Qdeg, hub, npre;
    uint32_t bcast[8];
    int gsh[kTeamShared];  // the team's group-shared slots (Team::sh)
};

// Wires a team to the calling thread group (B threads) and its shared memory.
template <int B, int EMAX, class TeamT>
__device__ __forceinline__ void bind_group(TeamT& tm, Smem<B, EMAX>& s)
{
    tm.tid = gtid<B>();
    tm.bar = gbar_id<B>();
    tm.nthr = B;
    tm.sh = s.gsh;
}

// Counts of one collected unit (chunk or hub).
struct Agg {
    uint32_t cnt;   // children
    uint32_t esum;  // sum of their valences
};

// ---------------------------------------------------------------------------
// Chunk machinery
// ---------------------------------------------------------------------------
template <int B, int EMAX>
struct Chunk {
    static constexpr int MAXEPT = EMAX / B;
    static_assert(EMAX % B == 0, "EMAX must be a multiple of B");
    Smem<B, EMAX>& s;
    const MatrixView& M;
    uint32_t base;  // key of the pass: edge id e has key base - 1 - e
    // queue record of position pf_base + (group thread), loaded by the previous
    // form() for the chunk that follows it (its latency hides behind that
    // chunk's work); pf_base == kUnvisited: none
    uint32_t pf_base = kUnvisited;
    uint4 pf = make_uint4(0u, 0u, 0u, 0u);

    // Loads up to B parents starting at position p (< pend) and forms the
    // next chunk: the longest run with <= EMAX edges.  Sets s.m (0 = the
    // first parent is a hub; s.hub = 1 then) and s.Ec.  Returns the number of
    // parents consumed (the hub counts as 1).
    __device__ uint32_t form(uint32_t p, uint32_t pend)
    {
        const uint32_t t = gtid<B>();
        uint32_t deg = 0;
        const bool have = p + t < pend;
        if (have) {
            const uint32_t pos = p + t;
            if (PB_CHECK(M.res, pos < M.n, 101)) {
                const uint4 r = p == pf_base ? pf : __ldcg(reinterpret_cast<const uint4*>(M.rec) + pos);
                s.pn[t] = r.x;
                s.prs[t] = r.y;
                s.pdeg[t] = r.z;
                s.peb[t] = r.w;
                deg = r.z;
            }
        }
        s.cc[t] = 0;
        uint32_t total;
        const uint32_t excl = block_scan1<B>(deg, total, s.scanbuf[0]);
        const uint32_t incl = excl + deg;
        // incl is monotone in t, so the fitting parents are a prefix
        const int fits = have && incl <= (uint32_t)EMAX;
        const int m = gsync_count<B>(fits);
        if (fits)
            s.soff[t] = excl;
        if (m > 0 && t == (uint32_t)(m - 1))
            s.soff[m] = incl;
        if (t == 0) {
            s.m = (uint32_t)m;
            s.hub = (m == 0 && p < pend) ? 1u : 0u;
            if (m == 0)
                s.soff[0] = 0;
        }
        // the next chunk starts where this one ends: load its records now
        const uint32_t used = m > 0 ? (uint32_t)m : (p < pend ? 1u : 0u);
        const uint32_t nb = p + used;
        pf_base = kUnvisited;
        if (nb < pend) {
            pf_base = nb;
            if (nb + t < pend && PB_CHECK(M.res, nb + t < M.n, 109))
                pf = __ldcg(reinterpret_cast<const uint4*>(M.rec) + nb + t);
        }
        gsync<B>();
        if (t == 0)
            s.Ec = m > 0 ? s.soff[m] : 0;
        gsync<B>();
        return used;
    }

    // Makes the ranked children of the previous chunk (still in shared memory,
    // with their adjacency in s.pre) the parents of this one: no global load.
    // Needs Q <= B and Qdeg <= EMAX; K0prev is the edge base they were placed
    // with.
    __device__ void form_from_children(uint32_t K0prev)
    {
        const uint32_t t = gtid<B>();
        const uint32_t F = s.Q, E = s.Qdeg;
        if (t < F) {
            const uint32_t x = s.so_idx[t];
            s.pn[t] = s.ch_node[x];
            s.prs[t] = s.ch_rs[x];
            s.pdeg[t] = s.ch_deg[x];
            s.peb[t] = K0prev + s.so_eoff[t];
            s.soff[t] = s.so_eoff[t];
        }
        s.cc[t] = 0;
        if (t == 0) {
            s.soff[F] = E;
            s.m = F;
            s.Ec = E;
            s.hub = 0;
        }
        gsync<B>();
    }

    // Finds the child edges of the chunk, compacts them, ranks every
    // parent's children (sorted = by valence, stable; else slot order) and
    // computes the edge offsets of the ranked children.
    __device__ Agg collect(bool sorted, bool from_pre = false)
    {
        const uint32_t t = gtid<B>(), lane = t & 31u, w = t >> 5;
        const uint32_t m = s.m, Ec = s.Ec;
        // thread t takes the edges e = t + B r: a warp loads consecutive
        // entries of the parents' rows (coalesced), and edge order is
        // (round r, warp, lane), the order the compaction below keeps
        uint32_t c[MAXEPT], jj[MAXEPT], key[MAXEPT], kk[MAXEPT];
#pragma unroll
        for (int r = 0; r < MAXEPT; ++r) {
            const uint32_t e = t + (uint32_t)B * r;
            c[r] = kUnvisited;
            jj[r] = 0;
            kk[r] = 1;
            if (e < Ec) {
                // the edge's parent: the last j < m with soff[j] <= e (a
                // parent of valence 0 owns no edge)
                uint32_t j = 0;
#pragma unroll
                for (uint32_t d = (uint32_t)B / 2u; d > 0; d >>= 1) {
                    const uint32_t mid = j + d;
                    if (mid < m && s.soff[mid] <= e)
                        j = mid;
                }
                const uint32_t k = e - s.soff[j];
                const uint32_t idx = s.prs[j] + k;
                jj[r] = j;
                kk[r] = k;
                key[r] = base - 1u - (s.peb[j] + k);
                if (from_pre)
                    c[r] = s.pre[e];  // the parents' adjacency, loaded when they were placed
                else if (PB_CHECK(M.res, idx < M.nnz, 102))
                    c[r] = ld_ro(M.ci + idx);
            }
        }
        uint4 nd[MAXEPT];
#pragma unroll
        for (int r = 0; r < MAXEPT; ++r) {
            nd[r] = make_uint4(0, 0, 0, 0);
            if (c[r] != kUnvisited && PB_CHECK(M.res, c[r] < M.n, 103))
                nd[r] = ld_node(M.node + c[r]);
        }
        // the child edges (claimed by this edge's key) compacted in edge
        // order: a ballot per warp and round, then the (round, warp) counts
        uint32_t pos[MAXEPT];
#pragma unroll
        for (int r = 0; r < MAXEPT; ++r) {
            if (!(c[r] != kUnvisited && c[r] < M.n && claim_of(M, nd[r]) == key[r]))
                c[r] = kUnvisited;
            const uint32_t bal = __ballot_sync(kFull, c[r] != kUnvisited);
            pos[r] = __popc(bal & ((1u << lane) - 1u));
            if (lane == 0)
                s.wq[r][w] = __popc(bal);
        }
        gsync<B>();
        uint32_t Q = 0;
#pragma unroll
        for (int r = 0; r < MAXEPT; ++r) {
#pragma unroll
            for (int i = 0; i < Smem<B, EMAX>::W; ++i) {
                const uint32_t n_ = s.wq[r][i];
                pos[r] += (uint32_t)i < w ? n_ : 0u;
                Q += n_;
            }
            // the rounds before this one
            if (r + 1 < MAXEPT)
                pos[r + 1] += Q;
        }
#pragma unroll
        for (int r = 0; r < MAXEPT; ++r) {
            const uint32_t e = t + (uint32_t)B * r;
            if (e < Ec) {
                const uint32_t q = pos[r];
                if (kk[r] == 0)
                    s.cs[jj[r]] = q;
                if (c[r] != kUnvisited && PB_CHECK(M.res, q < (uint32_t)EMAX, 104)) {
                    s.ch_node[q] = c[r];
                    s.ch_rs[q] = nd[r].y;
                    s.ch_deg[q] = nd[r].z;
                    s.ch_par[q] = jj[r];
                    atomicAdd(&s.cc[jj[r]], 1u);
                }
            }
        }
        gsync<B>();
        // rank every child inside its parent's run
        for (uint32_t x = t; x < Q; x += B) {
            const uint32_t jp = s.ch_par[x];
            const uint32_t st = s.cs[jp], len = s.cc[jp];
            uint32_t rank = x - st;
            if (sorted && len > 1) {
                const uint32_t dx = s.ch_deg[x];
                rank = 0;
                for (uint32_t y = st; y < st + len; ++y) {
                    const uint32_t dy = s.ch_deg[y];
                    rank += (dy < dx) || (dy == dx && y < x);
                }
            }
            s.so_idx[st + rank] = x;
        }
        gsync<B>();
        // edge offsets in ranked order (blocked exclusive scan)
        const uint32_t per = (Q + B - 1) / B;
        const uint32_t i0 = min(t * per, Q), i1 = min(i0 + per, Q);
        uint32_t loc = 0;
        for (uint32_t i = i0; i < i1; ++i)
            loc += s.ch_deg[s.so_idx[i]];
        uint32_t Qdeg;
        uint32_t off = block_scan1<B>(loc, Qdeg, s.scanbuf[2]);
        for (uint32_t i = i0; i < i1; ++i) {
            s.so_eoff[i] = off;
            off += s.ch_deg[s.so_idx[i]];
        }
        if (t == 0) {
            s.so_eoff[Q] = Qdeg;
            s.Q = Q;
            s.Qdeg = Qdeg;
            s.npre = 0;
        }
        gsync<B>();
        return Agg{Q, Qdeg};
    }

    // The ranked child owning edge offset f: so_eoff[lo] <= f < so_eoff[lo+1].
    __device__ __forceinline__ uint32_t child_of(uint32_t f) const
    {
        uint32_t lo = 0, hi = s.Q;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (s.so_eoff[mid] <= f)
                lo = mid;
            else
                hi = mid;
        }
        return lo;
    }

    // Walks the ranked children's edges in blocks of consecutive edge offsets
    // (one search per thread, then a forward walk), calling
    // fn(f, col_index) for each.
    template <typename Fn>
    __device__ __forceinline__ void for_child_edges(Fn fn) const
    {
        const uint32_t Qdeg = s.Qdeg;
        const uint32_t per = (Qdeg + B - 1) / B;
        const uint32_t f0 = gtid<B>() * per, f1 = min(f0 + per, Qdeg);
        if (f0 >= f1)
            return;
        uint32_t lo = child_of(f0);
        uint32_t beg = s.so_eoff[lo], nxt = s.so_eoff[lo + 1];
        uint32_t rs = s.ch_rs[s.so_idx[lo]];
        for (uint32_t f = f0; f < f1; ++f) {
            while (f >= nxt) {
                ++lo;
                beg = nxt;
                nxt = s.so_eoff[lo + 1];
                rs = s.ch_rs[s.so_idx[lo]];
            }
            fn(f, rs + (f - beg));
        }
    }

    // Loads the ranked children's adjacency into s.pre (when it fits) so that
    // the claims after the all-gather issue no dependent load.
    __device__ void prefetch()
    {
        const uint32_t Qdeg = s.Qdeg;
        if (Qdeg > (uint32_t)Smem<B, EMAX>::PREMAX)
            return;
        for_child_edges([&](uint32_t f, uint32_t idx) {
            s.pre[f] = PB_CHECK(M.res, idx < M.nnz, 108) ? ld_ro(M.ci + idx) : 0u;
        });
        gsync<B>();
        if (gtid<B>() == 0)
            s.npre = Qdeg;
        gsync<B>();
    }

    // Writes the ranked children of the chunk at positions P0.. and edge
    // bases K0.., then claims their edges for the next level.
    __device__ void place_and_claim(uint32_t P0, uint32_t K0, bool write_perm, bool reverse)
    {
        const uint32_t t = gtid<B>();
        const uint32_t Q = s.Q, Qdeg = s.Qdeg;
        const bool have_pre = s.npre == Qdeg && Qdeg > 0;
        for (uint32_t i = t; i < Q; i += B) {
            const uint32_t x = s.so_idx[i];
            const uint32_t pos = P0 + i;
            if (PB_CHECK(M.res, pos < M.n, 105)) {
                const uint4 r = make_uint4(s.ch_node[x], s.ch_rs[x], s.ch_deg[x], K0 + s.so_eoff[i]);
                __stcg(reinterpret_cast<uint4*>(M.rec) + pos, r);
                if (write_perm)
                    M.perm[reverse ? M.n - 1 - pos : pos] = r.x;
            }
        }
        const uint32_t kb = base - 1u - K0;
        if (have_pre) {
            for (uint32_t f = t; f < Qdeg; f += B) {
                const uint32_t d = s.pre[f];
                if (PB_CHECK(M.res, d < M.n, 107))
                    atomicMax(claim_ptr(M, d), kb - f);
            }
        } else {
            for_child_edges([&](uint32_t f, uint32_t idx) {
                if (PB_CHECK(M.res, idx < M.nnz, 106)) {
                    const uint32_t d = ld_ro(M.ci + idx);
                    if (PB_CHECK(M.res, d < M.n, 107))
                        atomicMax(claim_ptr(M, d), kb - f);
                }
            });
        }
    }

    // Writes the ranked children of the chunk to M.stage[at..]: node, row
    // start, valence and the child-edge offset eoff0 + so_eoff[i].
    __device__ void stage_children(uint32_t at, uint32_t eoff0)
    {
        const uint32_t Q = s.Q;
        for (uint32_t i = gtid<B>(); i < Q; i += B) {
            const uint32_t x = s.so_idx[i];
            if (PB_CHECK(M.res, (uint64_t)at + i < M.nnz, 130))
                __stcg(reinterpret_cast<uint4*>(M.stage) + at + i,
                       make_uint4(s.ch_node[x], s.ch_rs[x], s.ch_deg[x], eoff0 + s.so_eoff[i]));
        }
    }

    // Places the `count` children staged at M.stage[at..] (in order) at
    // positions P0.. with edge ids K0 + their child-edge offsets, and claims
    // their edges, in tiles of up to EMAX children.
    __device__ void place_staged(uint32_t at, uint32_t count, uint32_t P0, uint32_t K0, bool write_perm,
                                 bool reverse)
    {
        uint32_t done = 0, kdone = 0;
        while (done < count) {
            const uint32_t cnt = min((uint32_t)EMAX, count - done);
            for (uint32_t i = gtid<B>(); i < cnt; i += B) {
                uint4 r = make_uint4(0u, 0u, 0u, kdone);
                if (PB_CHECK(M.res, (uint64_t)at + done + i < M.nnz, 131))
                    r = __ldcg(reinterpret_cast<const uint4*>(M.stage) + at + done + i);
                s.ch_node[i] = r.x;
                s.ch_rs[i] = r.y;
                s.ch_deg[i] = r.z;
                s.so_idx[i] = i;
                s.so_eoff[i] = r.w - kdone;
                if (i == cnt - 1) {
                    s.so_eoff[cnt] = r.w + r.z - kdone;
                    s.Q = cnt;
                    s.Qdeg = r.w + r.z - kdone;
                    s.npre = 0;
                }
            }
            gsync<B>();
            const uint32_t qdeg = s.Qdeg;
            place_and_claim(P0 + done, K0 + kdone, write_perm, reverse);
            gsync<B>();
            done += cnt;
            kdone += qdeg;
        }
    }

    // ---- hubs: one parent with more than EMAX edges -----------------------
    // Scratch layout (4 arrays of nnz words): key0 | val0 | key1 | val1.  A
    // hub at level-relative edge offset r0 owns [r0, r0 + deg) of each.
    __device__ uint32_t* hk0() const { return M.hub; }
    __device__ uint32_t* hv0() const { return M.hub + M.nnz; }
    __device__ uint32_t* hk1() const { return M.hub + 2ull * M.nnz; }
    __device__ uint32_t* hv1() const { return M.hub + 3ull * M.nnz; }

    // Collects the hub's children (valence, slot) in slot order and sorts
    // them stably by valence (sorted == true) into key0/val0.  The counts
    // are also left in key1[r0], key1[r0+1] for a later placement.
    __device__ Agg hub_collect(uint32_t r0, bool sorted)
    {
        const uint32_t t = gtid<B>();
        const uint32_t rs = s.prs[0], D = s.pdeg[0], eb = s.peb[0];
        if (M.hub == nullptr) {
            set_status(M.res, kErrCheck, 120);
            return Agg{0, 0};
        }
        uint32_t Q = 0;
        unsigned long long Qdeg = 0;
        uint32_t maxkey = 0;
        constexpr uint32_t TILE = B * MAXEPT;
        for (uint32_t base0 = 0; base0 < D; base0 += TILE) {
            uint32_t nv = 0;
            uint32_t dg[MAXEPT];
            bool ok[MAXEPT];
#pragma unroll
            for (int r = 0; r < MAXEPT; ++r) {
                const uint32_t e = base0 + t * MAXEPT + r;
                ok[r] = false;
                if (e < D && PB_CHECK(M.res, rs + e < M.nnz, 121)) {
                    const uint32_t c = ld_ro(M.ci + rs + e);
                    if (PB_CHECK(M.res, c < M.n, 122)) {
                        const uint4 nd = ld_node(M.node + c);
                        if (claim_of(M, nd) == base - 1u - (eb + e)) {
                            dg[r] = nd.z;
                            ok[r] = true;
                            ++nv;
                        }
                    }
                }
            }
            uint32_t tot;
            uint32_t q = block_scan1<B>(nv, tot, s.scanbuf[3]);
            uint32_t lsum = 0, lmax = 0;
#pragma unroll
            for (int r = 0; r < MAXEPT; ++r) {
                if (ok[r]) {
                    const uint32_t w = r0 + Q + q;
                    if (PB_CHECK(M.res, w < M.nnz, 123)) {
                        hk0()[w] = dg[r];
                        hv0()[w] = base0 + t * MAXEPT + r;
                    }
                    lsum += dg[r];
                    lmax = max(lmax, dg[r]);
                    ++q;
                }
            }
            Qdeg += block_reduce_sum<B, unsigned long long>(lsum, s.tmp64);
            maxkey = max(maxkey, block_reduce_max<B, uint32_t>(lmax, s.tmp32));
            Q += tot;
        }
        if (sorted && Q > 1) {
            // stable LSD radix sort, 8-bit digits, an even number of passes
            // so that the result lands back in key0/val0
            uint32_t passes = 0;
            while (passes < 4 && (maxkey >> (8 * passes)) != 0)
                ++passes;
            if (passes == 0)
                passes = 1;
            passes += passes & 1;
            for (uint32_t ps = 0; ps < passes; ++ps) {
                uint32_t* sk = (ps & 1) ? hk1() : hk0();
                uint32_t* sv = (ps & 1) ? hv1() : hv0();
                uint32_t* dk = (ps & 1) ? hk0() : hk1();
                uint32_t* dv = (ps & 1) ? hv0() : hv1();
                radix_pass(sk + r0, sv + r0, dk + r0, dv + r0, Q, 8 * ps);
            }
        }
        if (t == 0) {
            __stcg(hk1() + r0, Q);
            __stcg(hk1() + r0 + 1, (uint32_t)Qdeg);
        }
        gsync<B>();
        return Agg{Q, (uint32_t)Qdeg};
    }

    // One stable counting pass on digit (key >> shift) & 255.
    __device__ void radix_pass(const uint32_t* sk, const uint32_t* sv, uint32_t* dk, uint32_t* dv, uint32_t Q,
                               uint32_t shift)
    {
        const uint32_t t = gtid<B>(), lane = t & 31, w = t >> 5;
        for (uint32_t d = t; d < 256; d += B)
            s.hist[d] = 0;
        gsync<B>();
        for (uint32_t i = t; i < Q; i += B)
            atomicAdd(&s.hist[(__ldcg(sk + i) >> shift) & 255u], 1u);
        gsync<B>();
        if (t == 0) {
            uint32_t run = 0;
            for (int d = 0; d < 256; ++d) {
                const uint32_t h = s.hist[d];
                s.hist[d] = run;
                run += h;
            }
        }
        gsync<B>();
        for (uint32_t base0 = 0; base0 < Q; base0 += B) {
            for (uint32_t i = t; i < (uint32_t)(Smem<B, EMAX>::W * 256); i += B)
                s.hcnt[i] = 0;
            gsync<B>();
            const uint32_t i = base0 + t;
            const bool act = i < Q;
            uint32_t key = 0, val = 0, dgt = 0;
            if (act) {
                key = __ldcg(sk + i);
                val = __ldcg(sv + i);
                dgt = (key >> shift) & 255u;
            }
            const uint32_t peers = __match_any_sync(kFull, act ? dgt : 256u + lane);
            const uint32_t below = peers & ((1u << lane) - 1u);
            const uint32_t rank_w = __popc(below);
            const bool leader = act && below == 0;
            if (leader)
                s.hcnt[w * 256 + dgt] = __popc(peers);
            gsync<B>();
            if (act) {
                uint32_t before = 0;
                for (uint32_t ww = 0; ww < w; ++ww)
                    before += s.hcnt[ww * 256 + dgt];
                const uint32_t dst = s.hist[dgt] + before + rank_w;
                dk[dst] = key;
                dv[dst] = val;
            }
            gsync<B>();
            for (uint32_t d = t; d < 256; d += B) {
                uint32_t add = 0;
                for (int ww = 0; ww < Smem<B, EMAX>::W; ++ww)
                    add += s.hcnt[ww * 256 + d];
                s.hist[d] += add;
            }
            gsync<B>();
        }
    }

    // Places the sorted hub children (count Q) at P0.. / K0.. in tiles of
    // EMAX, reusing the chunk arrays, and claims their edges.
    __device__ void hub_place_and_claim(uint32_t r0, uint32_t Q, uint32_t P0, uint32_t K0, bool write_perm,
                                        bool reverse)
    {
        const uint32_t t = gtid<B>();
        const uint32_t rs = s.prs[0];
        uint32_t done = 0, kdone = 0;
        while (done < Q) {
            const uint32_t cnt = min((uint32_t)EMAX, Q - done);
            uint32_t loc = 0;
            const uint32_t per = (cnt + B - 1) / B;
            const uint32_t i0 = min(t * per, cnt), i1 = min(i0 + per, cnt);
            for (uint32_t i = i0; i < i1; ++i) {
                const uint32_t slot = __ldcg(hv0() + r0 + done + i);
                const uint32_t node = ld_ro(M.ci + rs + slot);
                const uint4 nd = ld_node(M.node + node);
                s.ch_node[i] = node;
                s.ch_rs[i] = nd.y;
                s.ch_deg[i] = nd.z;
                s.so_idx[i] = i;
                loc += nd.z;
            }
            uint32_t tot;
            uint32_t off = block_scan1<B>(loc, tot, s.scanbuf[4]);
            for (uint32_t i = i0; i < i1; ++i) {
                s.so_eoff[i] = off;
                off += s.ch_deg[i];
            }
            if (t == 0) {
                s.so_eoff[cnt] = tot;
                s.Q = cnt;
                s.Qdeg = tot;
                s.npre = 0;
            }
            gsync<B>();
            place_and_claim(P0 + done, K0 + kdone, write_perm, reverse);
            gsync<B>();
            done += cnt;
            kdone += tot;
        }
    }
};

// ---------------------------------------------------------------------------
// Level state of one pass.
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// One ordered BFS pass from `start` with pass key `base`.  Fills
// rec[0..placed) and, when write_perm, the output.  Returns false if the team
// must stop.  nlevels: number of levels; last_start: first position of the
// last level.
// ---------------------------------------------------------------------------
template <int B, int EMAX, class TeamT>
__device__ bool bfs_pass(Smem<B, EMAX>& s, const MatrixView& M, TeamT& team, unsigned long long* agg,
                         uint32_t& step, const Options& opt, uint32_t start, uint32_t base, bool sorted,
                         bool write_perm, bool reverse, uint32_t& placed, uint32_t& nlevels, uint32_t& last_start,
                         uint32_t& wide_f, uint32_t& wide_e)
{
    Chunk<B, EMAX> ch{s, M, base};
    const uint32_t t = gtid<B>();
    const uint32_t G = team.size, R = team.rank;
    const uint32_t n = M.n;

    LevelState st;
    const uint4 sn = ld_node(M.node + start);
    const uint32_t rs0 = sn.y, deg0 = sn.z;
    st.a = 0;
    st.b = 1;
    st.Ka = 0;
    st.Kb = deg0;
    st.L = 0;
    st.last_start = 0;
    // CTA 0 places the start and claims its edges
    if (R == 0) {
        if (t == 0) {
            atomicMax(claim_ptr(M, start), base);
            __stcg(reinterpret_cast<uint4*>(M.rec), make_uint4(start, rs0, deg0, 0u));
            if (write_perm)
                M.perm[reverse ? n - 1 : 0] = start;
        }
        for (uint32_t k = t; k < deg0; k += B) {
            const uint32_t d = ld_ro(M.ci + rs0 + k);
            if (PB_CHECK(M.res, d < n, 110))
                atomicMax(claim_ptr(M, d), base - 1u - k);
        }
    }
    auto is_solo = [&](const LevelState& x) {
        return G == 1 || ((x.b - x.a) <= opt.solo_parents && (x.Kb - x.Ka) <= opt.solo_edges);
    };
    bool solo = is_solo(st);
    if (!solo) {
        if (!team.sync(2))
            return false;
    }
    while (true) {
        if (solo) {
            // ---- CTA 0 alone: chunk by chunk with running offsets ----------
            if (R == 0) {
                // carry: the frontier and its adjacency are still in shared
                // memory from the previous level (it fitted one chunk)
                bool carry = false;
                bool solo_fail = false;  // stop after handing the gate over
                while (true) {
                    uint32_t P = st.b, K = st.Kb;
                    bool next_carry = false;
                    if (carry) {
                        ch.form_from_children(st.Ka);
                        const Agg g = ch.collect(sorted, true);
                        ch.prefetch();
                        ch.place_and_claim(P, K, write_perm, reverse);
                        P += g.cnt;
                        K += g.esum;
                        next_carry = g.cnt > 0 && g.cnt <= (uint32_t)B && g.esum <= (uint32_t)EMAX &&
                                     s.npre == g.esum;
                        gsync<B>();
                    } else {
                        uint32_t p = st.a;
                        while (p < st.b) {
                            const uint32_t used = ch.form(p, st.b);
                            const bool single = p == st.a && used == st.b - st.a;
                            if (s.hub) {
                                const uint32_t r0 = s.peb[0] - st.Ka;
                                const Agg g = ch.hub_collect(r0, sorted);
                                ch.hub_place_and_claim(r0, g.cnt, P, K, write_perm, reverse);
                                P += g.cnt;
                                K += g.esum;
                            } else {
                                const Agg g = ch.collect(sorted);
                                if (single)
                                    ch.prefetch();
                                ch.place_and_claim(P, K, write_perm, reverse);
                                P += g.cnt;
                                K += g.esum;
                                next_carry = single && g.cnt > 0 && g.cnt <= (uint32_t)B &&
                                             g.esum <= (uint32_t)EMAX && s.npre == g.esum;
                            }
                            gsync<B>();
                            p += used;
                        }
                    }
                    carry = next_carry;
                    if (!team.block_ok()) {
                        solo_fail = true;
                        break;
                    }
                    const uint32_t tot = P - st.b;
                    if (tot == 0) {
                        st.a = st.b;  // an empty frontier marks the end of the pass
                        break;
                    }
                    st.last_start = st.b;
                    st.a = st.b;
                    st.b = P;
                    st.Ka = st.Kb;
                    st.Kb = K;
                    st.L += 1;
                    if (st.b > n) {
                        set_status(M.res, kErrCheck, 111);
                        solo_fail = true;
                        break;
                    }
                    if (G > 1)
                        team.beat();
                    if (!is_solo(st))
                        break;
                }
                if (G > 1) {
                    if (!team.gate_open(st, !solo_fail))
                        return false;
                } else if (solo_fail) {
                    return false;
                }
            } else {
                if (!team.gate_wait(st))
                    return false;
            }
            if (st.a == st.b) {
                // the pass ended during the solo run: every CTA leaves it
                // together, so that none can still be reading this gate's
                // state when CTA 0 opens the next one
                if (G > 1 && !team.sync(8))
                    return false;
                break;
            }
            solo = false;
            continue;
        }
        // ---- whole team ---------------------------------------------------
        const uint32_t F = st.b - st.a;
        wide_f = max(wide_f, F);
        wide_e = max(wide_e, st.Kb - st.Ka);
        const uint32_t p_beg = st.a + (uint32_t)(((uint64_t)F * R) / G);
        const uint32_t p_end = st.a + (uint32_t)(((uint64_t)F * (R + 1)) / G);
        // A1: collect and count.  A CTA whose parents take several chunks
        // stages each chunk's ranked children (M.stage, at the level-relative
        // edge offset of its first parent: the CTAs' regions are disjoint and
        // hold their children, which are at most their parents' edges), so
        // that placing them needs no second collect.
        uint32_t my_cnt = 0, my_esum = 0, nunits = 0;
        bool last_hub = false;
        bool staged = M.stage != nullptr;  // every unit staged (no hub among them)
        uint32_t stage_base = 0;
        uint32_t p = p_beg;
        while (p < p_end) {
            const uint32_t used = ch.form(p, p_end);
            if (nunits == 0)
                stage_base = s.peb[0] - st.Ka;
            Agg g;
            last_hub = s.hub != 0;
            if (last_hub) {
                g = ch.hub_collect(s.peb[0] - st.Ka, sorted);
                staged = false;
            } else {
                g = ch.collect(sorted);
                if (staged && !(nunits == 0 && used == p_end - p))
                    ch.stage_children(stage_base + my_cnt, my_esum);
            }
            my_cnt += g.cnt;
            my_esum += g.esum;
            ++nunits;
            p += used;
            gsync<B>();
        }
        // publish (level-tagged), then prefetch while the others finish
        ++step;
        team.ag_publish(my_cnt, my_esum, step, agg);
        const bool keep = nunits == 1 && !last_hub;
        if (keep)
            ch.prefetch();
        // all-gather of the per-CTA totals
        unsigned long long pre = 0, all = 0;
        if (!team.template ag_collect<B>(step, agg, pre, all, s.gat64))
            return false;
        const uint32_t tot_cnt = (uint32_t)(all & 0xFFFFFFFFull);
        const uint32_t tot_esum = (uint32_t)(all >> 32);
        if (opt.wide_at != 0 && tot_cnt >= opt.wide_at && base == 2u * M.nnz + 3u && M.cf == 0 &&
            G == gridDim.x) {
            // a level this wide in the first pass of the whole team (key base
            // of pass 1 in the main claim word; never a half team, whose
            // other half would wait for it): the level-synchronous engine
            // takes the matrix (every CTA has the same totals and leaves)
            if (R == 0 && t == 0)
                set_status(M.res, kNeedWide, 0);
            return false;
        }
        uint32_t P = st.b + (uint32_t)(pre & 0xFFFFFFFFull);
        uint32_t K = st.Kb + (uint32_t)(pre >> 32);
        // A2: place (the only unit is still in shared memory, or all are staged)
        if (keep) {
            ch.place_and_claim(P, K, write_perm, reverse);
        } else if (nunits > 0 && staged) {
            ch.place_staged(stage_base, my_cnt, P, K, write_perm, reverse);
        } else if (nunits > 0) {
            p = p_beg;
            while (p < p_end) {
                const uint32_t used = ch.form(p, p_end);
                if (s.hub) {
                    const uint32_t r0 = s.peb[0] - st.Ka;
                    const uint32_t q = __ldcg(ch.hk1() + r0);
                    const uint32_t qd = __ldcg(ch.hk1() + r0 + 1);
                    ch.hub_place_and_claim(r0, q, P, K, write_perm, reverse);
                    P += q;
                    K += qd;
                } else {
                    const Agg g = ch.collect(sorted);
                    ch.place_and_claim(P, K, write_perm, reverse);
                    P += g.cnt;
                    K += g.esum;
                }
                gsync<B>();
                p += used;
            }
        }
        if (!team.sync(5))
            return false;
        if (tot_cnt == 0)
            break;
        st.last_start = st.b;
        st.a = st.b;
        st.b += tot_cnt;
        st.Ka = st.Kb;
        st.Kb += tot_esum;
        st.L += 1;
        if (st.b > n) {
            set_status(M.res, kErrCheck, 112);
            return false;
        }
        solo = is_solo(st);
    }
    placed = st.b;
    nlevels = st.L + 1;
    last_start = st.last_start;
    return true;
}

// Next start of the pseudo-peripheral search (simple_peripheral.cpp:110-127)
// from the ordered BFS just run: among the last min(outnodes, n-1) positions,
// those on the last level; the last of minimal valence.  Thread 0 computes.
__device__ __forceinline__ uint32_t next_peripheral_start(const MatrixView& M, uint32_t outnodes, uint32_t last_start)
{
    const uint32_t n = M.n;
    uint32_t lo = n - min(outnodes, n - 1);
    lo = max(lo, max(last_start, 1u));
    uint32_t best = 0, bestdeg = kUnvisited;
    for (uint32_t pos = lo; pos < n; ++pos) {
        const uint4 r = __ldcg(reinterpret_cast<const uint4*>(M.rec) + pos);
        if (r.z <= bestdeg) {
            bestdeg = r.z;
            best = r.x;
        }
    }
    return best;
}

// Fills the node table (claim 0, row start, valence) of the matrix.
template <int B>
__device__ void init_nodes(const MatrixView& M, uint32_t R, uint32_t G)
{
    for (uint64_t v = (uint64_t)R * B + gtid<B>(); v < M.n; v += (uint64_t)G * B) {
        const uint32_t a = ld_ro(M.rp + v), e = ld_ro(M.rp + v + 1);
        __stcg(reinterpret_cast<uint4*>(M.node) + v, make_uint4(0u, a, e - a, 0u));
    }
}

// ---------------------------------------------------------------------------
// Full reorder of one matrix by one team: start search, final ordered pass,
// bandwidth.  Every CTA of the team runs this; CTA 0 thread 0 writes *res.
// ---------------------------------------------------------------------------
template <int B, int EMAX, class TeamT>
__device__ void reorder_matrix(Smem<B, EMAX>& s, const MatrixView& M, TeamT& team, unsigned long long* agg,
                               const Options& opt)
{
    const uint32_t t = gtid<B>();
    const uint32_t n = M.n;
    const uint32_t G = team.size, R = team.rank;
    uint32_t start = opt.start;
    uint32_t passes = 0, ecc = 0, placed = 0, nlevels = 0, last_start = 0;
    uint32_t step = 0;

    if (start != kUnvisited && start >= n) {
        if (R == 0 && t == 0)
            set_status(M.res, kErrArg, 2);
        return;
    }
    if (R == 0 && t == 0)
        M.res->t_begin = globaltimer();
    init_nodes<B>(M, R, G);
    if (!team.sync(1))
        return;
    // pass keys: pass p owns [p*kspan, p*kspan + nnz + 1], separately in
    // each claim word (claim: start-search and final passes; inv: the
    // speculative ordered passes)
    const uint32_t kspan = M.nnz + 2u;
    const uint32_t pmax = (uint32_t)(0xFFFFFFFFull / kspan) - 1u;
    uint32_t pass_id = 0, pass_id2 = 0;

    // Speculation.  Once the first start-search pass has run, every later
    // pass may be the last one (its eccentricity equals the previous one);
    // the final ordered pass then starts from the same node.  So the team
    // splits in two halves: one runs the start-search pass from the
    // candidate, the other runs the ordered pass from it at the same time
    // (claim word inv, queue records rec2, writing the output).  If the
    // candidate is confirmed, the ordered pass is already done; if not, its
    // output is overwritten later.  Pays off when most levels are small
    // enough for one CTA (each half runs them on its first CTA); a level that
    // needs the whole team takes a half team about 1.5x as long.  Not with
    // hubs (both halves would share the hub scratch); grid teams only.
    const bool spec = TeamT::kGrid && M.rec2 != nullptr && G >= 2 && start == kUnvisited && n > 1 &&
                      opt.mode == kModeFull && __ldcg(&M.res->maxdeg) <= (uint32_t)EMAX;
    const uint32_t half = G / 2;
    const bool low = R < half;
    TeamT sub = team;  // this CTA's half
    unsigned long long* sub_agg = agg;
    uint32_t sub_step = 0;
    if constexpr (TeamT::kGrid) {
        if (spec) {
            const size_t pw = team_part_bytes((int)G) / sizeof(unsigned long long);
            sub_agg = agg + (low ? pw : 2 * pw);
            sub.size = low ? half : G - half;
            sub.rank = low ? R : R - half;
            sub.gs = sub.size > 1 ? team.gs + (low ? 1 : 2) : nullptr;
            sub.flags = reinterpret_cast<unsigned int*>(sub_agg + 2 * sub.size);
            sub.expected = sub.size;
            sub.target = 0;
            sub.epoch = 0;
        }
    }
    MatrixView M2 = M;  // the speculative ordered pass's view
    M2.rec = M.rec2;
    M2.cf = 3;
    M2.stage = M.stage != nullptr ? M.stage + M.nnz : nullptr;  // its own half of the staging array
    bool spec_on = false;    // the next search pass runs beside the speculative ordered pass
    bool solo_dom = false;   // most levels of the first pass ran on one CTA
    bool narrow = false;     // every team level of the first pass is narrow enough for a half team
    bool spec_done = false;  // the speculative ordered pass wrote the output

    // pseudo-peripheral search (simple_peripheral.cpp:92-141), then the
    // degree-sorted pass that writes the permutation.  Every pass goes
    // through the one call of bfs_pass below (it is large: a single inlined
    // copy keeps the kernel's registers down).
    bool searching = start == kUnvisited && n > 1;
    if (n == 1) {
        // one node: the start search runs one pass and records nothing
        passes = start == kUnvisited ? 1 : 0;
        start = 0;
    } else if (searching) {
        start = n / 2;
    }
    uint32_t lastdist = 0;
    while (true) {
        if (!searching && opt.mode == kModeStartOnly)
            break;
        const bool split = searching && spec_on;  // spec_on implies a first pass has run
        const bool spec_half = split && !low;     // this CTA runs the speculative ordered pass
        const bool ordered = !searching || spec_half;
        TeamT& tm = split ? sub : team;
        unsigned long long* ag = split ? sub_agg : agg;
        uint32_t& stp = split ? sub_step : step;
        uint32_t& pid = spec_half ? pass_id2 : pass_id;
        if (searching)
            ++passes;
        if (pid + 1 > pmax) {
            // reset this pass's claim word (the other half never touches it)
            const uint32_t cf = spec_half ? 3u : 0u;
            for (uint64_t v = (uint64_t)tm.rank * B + t; v < n; v += (uint64_t)tm.size * B)
                reinterpret_cast<uint32_t*>(M.node + v)[cf] = 0u;
            pid = 0;
            if (!tm.sync(7))
                return;
        }
        ++pid;
        const uint32_t base = pid * kspan + M.nnz + 1u;
        const uint32_t step0 = step;
        uint32_t pl = 0, nl = 0, ls = 0, wf = 0, we = 0;
        if (!bfs_pass<B, EMAX>(s, spec_half ? M2 : M, tm, ag, stp, opt, start, base, ordered, ordered,
                               ordered && opt.reverse != 0, pl, nl, ls, wf, we))
            return;
        if (!searching) {
            placed = pl;
            nlevels = nl;
            last_start = ls;
            break;
        }
        uint32_t dist = 0, next = 0;
        if (!split) {
            if (pl != n) {
                if (R == 0 && t == 0)
                    set_status(M.res, kErrDisconnected, 0);
                return;
            }
            // speculate from the next pass on if at most a quarter of the
            // levels needed the whole team (step counts them); otherwise from
            // pass opt.spec_from on, where the search usually ends, if the
            // widest level takes a CTA of a half team at most four chunks
            // (measured: the 128^3 grid, 1.6 chunks, gains 14 %; a 1M-node
            // RGG, 20 chunks, would lose 30 %)
            if (passes == 1) {
                solo_dom = 4ull * (step - step0) <= nl;
                narrow = (uint64_t)wf <= 4ull * half * B && (uint64_t)we <= 4ull * half * EMAX;
            }
            spec_on = spec && (solo_dom || (narrow && opt.spec_from != 0 && passes + 1 >= opt.spec_from));
            dist = nl - 1;
            if (dist == lastdist) {
                ecc = dist;
                searching = false;  // the ordered pass from the same start comes next
                continue;
            }
            if (t == 0)
                s.bcast[0] = next_peripheral_start(M, opt.outnodes, ls);
            gsync<B>();
            next = s.bcast[0];
            gsync<B>();
        } else {
            if constexpr (TeamT::kGrid) {
                // the halves meet in the team's GridSync words st[8..12]
                if (sub.rank == 0 && t == 0) {
                    if (low) {
                        team.gs->st[8] = pl;
                        team.gs->st[9] = nl;
                        team.gs->st[10] = pl == n ? next_peripheral_start(M, opt.outnodes, ls) : 0u;
                    } else {
                        team.gs->st[11] = pl;
                        team.gs->st[12] = nl;
                    }
                }
                if (!team.sync(10))
                    return;
                const uint32_t pl_u = __ldcg(&team.gs->st[8]), nl_u = __ldcg(&team.gs->st[9]);
                next = __ldcg(&team.gs->st[10]);
                const uint32_t pl_s = __ldcg(&team.gs->st[11]), nl_s = __ldcg(&team.gs->st[12]);
                if (!team.sync(11))  // everyone has read st[8..12] before the next round writes them
                    return;
                if (pl_u != n) {
                    if (R == 0 && t == 0)
                        set_status(M.res, kErrDisconnected, 0);
                    return;
                }
                if (pl_s != n || nl_s != nl_u) {  // same start, same levels: cannot differ
                    if (R == 0 && t == 0)
                        set_status(M.res, kErrCheck, 4);
                    return;
                }
                dist = nl_u - 1;
                if (dist == lastdist) {
                    ecc = dist;
                    placed = pl_s;
                    nlevels = nl_s;
                    spec_done = true;
                    break;
                }
            }
        }
        if (passes > n) {  // eccentricities only grow; cannot happen on a valid run
            if (R == 0 && t == 0)
                set_status(M.res, kErrCheck, 3);
            return;
        }
        start = next;
        lastdist = dist;
    }
    if (opt.mode == kModeStartOnly) {
        if (R == 0 && t == 0) {
            M.res->start = start;
            M.res->passes = passes;
            M.res->ecc = ecc;
            M.res->placed = n;
        }
        return;
    }
    if (placed != n) {
        if (R == 0 && t == 0) {
            set_status(M.res, kErrDisconnected, 1);
            M.res->placed = placed;
        }
        return;
    }
    const PosRec* final_rec = spec_done ? M.rec2 : M.rec;

    if (opt.want_bw) {
        // inverse permutation (CM positions) into node[].inv
        for (uint64_t pos = (uint64_t)R * B + t; pos < n; pos += (uint64_t)G * B) {
            const uint4 r = __ldcg(reinterpret_cast<const uint4*>(final_rec) + pos);
            M.node[r.x].inv = (uint32_t)pos;
        }
        if (!team.sync(6))
            return;
        unsigned long long bw = 0, bw0 = 0, plo = 0, phi = 0;
        for (uint64_t i = (uint64_t)R * B + t; i < n; i += (uint64_t)G * B) {
            const uint32_t a = ld_ro(M.rp + i), e = ld_ro(M.rp + i + 1);
            if (a == e)
                continue;
            const uint32_t me = __ldcg(&M.node[i].inv);
            uint32_t mnr = kUnvisited, mxr = 0;
            for (uint32_t k = a; k < e; ++k) {
                const uint32_t p = __ldcg(&M.node[ld_ro(M.ci + k)].inv);
                mnr = min(mnr, p);
                mxr = max(mxr, p);
            }
            // computeBandwidth (main.cpp:143-184): max(row - min, max - row), >= 0
            const unsigned long long b1 = me >= mnr ? (unsigned long long)(me - mnr) : 0ull;
            const unsigned long long b2 = mxr >= me ? (unsigned long long)(mxr - me) : 0ull;
            bw = max(bw, max(b1, b2));
            // profile of the CM order (row - min col) and of its reverse (max col - row)
            plo += b1;
            phi += b2;
            // initial bandwidth: first / last stored column (main.cpp:114-129)
            const uint32_t c0 = ld_ro(M.ci + a), c1 = ld_ro(M.ci + e - 1);
            const unsigned long long i0 = i >= c0 ? i - c0 : 0, i1 = c1 >= i ? c1 - i : 0;
            bw0 = max(bw0, max(i0, i1));
        }
        bw = block_reduce_max<B, unsigned long long>(bw, s.tmp64);
        bw0 = block_reduce_max<B, unsigned long long>(bw0, s.tmp64);
        block_reduce_sum2<B>(plo, phi, s.tmp64);
        if (t == 0) {
            atomicMax(&M.res->bandwidth, bw);
            atomicMax(&M.res->initial_bw, bw0);
            atomicAdd(&M.res->profile_lo, plo);
            atomicAdd(&M.res->profile_hi, phi);
        }
    }
    if (R == 0 && t == 0) {
        M.res->start = start;
        M.res->passes = passes;
        M.res->ecc = ecc;
        M.res->levels = nlevels;
        M.res->placed = placed;
        M.res->t_end = globaltimer();
    }
}

// ---------------------------------------------------------------------------
// CSR check of one matrix by one thread group (the batch kernels; the
// single-matrix path runs k_validate over the whole GPU instead): rows
// ordered and inside [0, nnz], every column below n, and the largest valence
// (decides whether hub scratch is needed) into res->maxdeg.  Coalesced.
template <int B>
__device__ void validate_group(const MatrixView& M, uint32_t* red)
{
    const uint32_t t = gtid<B>();
    uint32_t mx = 0;
    bool bad = false;
    for (uint32_t i = t; i < M.n; i += B) {
        const uint32_t a = ld_ro(M.rp + i), b = ld_ro(M.rp + i + 1);
        if (b < a || b > M.nnz)
            bad = true;
        else
            mx = max(mx, b - a);
    }
    if (t == 0 && (ld_ro(M.rp) != 0 || ld_ro(M.rp + M.n) != M.nnz))
        bad = true;
#pragma unroll 4
    for (uint32_t k = t; k < M.nnz; k += B)
        if (ld_ro(M.ci + k) >= M.n)
            bad = true;
    if (bad)
        set_status(M.res, kErrArg, 200);
    mx = block_reduce_max<B, uint32_t>(mx, red);
    if (t == 0)
        atomicMax(&M.res->maxdeg, mx);
    gsync<B>();
}

// validate_group without the column pass: row pointers and the largest
// valence (the solo batch kernel tests the columns while it builds the edge
// records, solo_build_edges).
template <int B>
__device__ void validate_rows(const MatrixView& M, uint32_t* red)
{
    const uint32_t t = gtid<B>();
    uint32_t mx = 0;
    bool bad = false;
    for (uint32_t i = t; i < M.n; i += B) {
        const uint32_t a = ld_ro(M.rp + i), b = ld_ro(M.rp + i + 1);
        if (b < a || b > M.nnz)
            bad = true;
        else
            mx = max(mx, b - a);
    }
    if (t == 0 && (ld_ro(M.rp) != 0 || ld_ro(M.rp + M.n) != M.nnz))
        bad = true;
    if (bad)
        set_status(M.res, kErrArg, 200);
    mx = block_reduce_max<B, uint32_t>(mx, red);
    if (t == 0)
        atomicMax(&M.res->maxdeg, mx);
    gsync<B>();
}

// Bounded wait of a thread group for a matrix's CSR to arrive (the word
// `ready` is written by a host-to-device copy after the CSR's copies).  A
// wait that runs out posts PBRCM_ERR_TIMEOUT for the matrix.  The word is
// read with acquire semantics; the CSR's lines are read only afterwards, and
// no other matrix shares them (every CSR starts on a 128-byte boundary).
template <int B>
__device__ void wait_ready(const uint32_t* ready, unsigned long long wait_ns, DevResult* res, int* flag)
{
    if (gtid<B>() == 0) {
        int ok = 1;
        unsigned long long t0 = 0;
        uint32_t spins = 0;
        while (ld_acquire(ready) == 0u) {
            if ((++spins & 63u) == 0) {
                const unsigned long long now = globaltimer();
                if (t0 == 0) {
                    t0 = now;
                } else if (now - t0 > wait_ns) {
                    set_status(res, kErrTimeout, 210);
                    ok = 0;
                    break;
                }
            }
            __nanosleep(spins > 4096 ? 1024 : 128);
        }
        *flag = ok;
    }
    gsync<B>();
}

// ---------------------------------------------------------------------------
// Early exits shared by the reorder kernels.  Returns true if the matrix must
// not be processed.  Every CTA reads the same values, so all agree.
template <int EMAX>
__device__ __forceinline__ bool skip_matrix(const MatrixView& M, bool first_thread)
{
    if (read_status(M.res) != 0)
        return true;
    if (__ldcg(&M.res->maxdeg) > (uint32_t)EMAX && M.hub == nullptr) {
        if (first_thread)
            set_status(M.res, kNeedHub, 0);
        return true;
    }
    return false;
}

}  // namespace pbrcm
