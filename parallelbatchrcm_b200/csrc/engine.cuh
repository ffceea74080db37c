// engine.cuh -- device core of the B200 Cuthill-McKee engine (sm_100a).
//
// What it computes
//   The serial stable Cuthill-McKee order of the reference
//   (src/rcm_cpu.cpp:57-104): FIFO over positions; parent at position i
//   appends its still-unvisited neighbours, stable-sorted by valence (row
//   length).  The reference's GPU_BATCH reaches it with a chain of speculative
//   batches (include/device/batchWorker.cuh); this engine reaches it level by
//   level with every CTA of a team working on one BFS level at a time.
//
// The claim key
//   Edges of the frontier are numbered in queue order: edge (position i, slot
//   k) has the global id ebase(i) + k, where ebase(i) = sum of the valences of
//   the nodes at positions < i.  Every frontier edge does
//   atomicMin(claim[child], id + 1).  Once a level's claims are done, a node's
//   claim is the id + 1 of the FIRST edge that reaches it in queue order --
//   exactly the (parent, slot) that discovers it in the serial algorithm,
//   duplicates in a row included.  An edge is a "child edge" iff
//   claim[col] == id + 1, a purely local test.  The key is an order-preserving
//   lexicographic (parent position, slot) code; the reference's batch code
//   (batchId << 11 | offset, batchWorker.cuh:574-586) plays the same role for
//   its batches.
//
// One level (frontier = positions [a, b), its edges have ids [Ka, Kb))
//   collect: each CTA takes a contiguous range of parents, splits it into
//            chunks (<= B parents, <= EMAX edges), finds the child edges,
//            compacts them in (parent, slot) order and sorts each parent's
//            children by (valence, slot) with a counting rank.
//   place:   children get positions b + (children of earlier parents) + rank
//            and edge bases Kb + (valences of earlier children); their
//            records go to rec[], the output to perm[].
//   claim:   the placed children immediately claim their own edges for the
//            next level.  Keys of the next level are > Kb, so they never
//            disturb nodes already placed (their claims are <= Kb).
//   A team of one CTA places chunk by chunk with a running offset; a grid
//   team publishes per-CTA totals, meets at a barrier, then places.
//   Parents with more than EMAX edges ("hubs") are collected and
//   radix-sorted in global scratch by one CTA.
//
// Every wait is bounded by %globaltimer and reports PBRCM_ERR_TIMEOUT.
// With PBRCM_CHECKS defined, every global index is range-checked and a
// failure records PBRCM_ERR_CHECK and skips the access.
#pragma once

#include <cstdint>
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

__device__ __forceinline__ void st_release(unsigned int* p, unsigned int v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ uint32_t ld_cg(const uint32_t* p) { return __ldcg(p); }

__device__ __forceinline__ uint32_t ld_ro(const uint32_t* p) { return __ldg(p); }

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

// Block-wide exclusive scan of one value per thread (T = uint32_t or
// unsigned long long).  `tmp` holds B/32 + 1 entries.  Ends with a barrier,
// so `tmp` can be reused right away.
template <int B, typename T>
__device__ __forceinline__ T block_exclusive_scan(T v, T& total, T* tmp)
{
    constexpr int W = B / 32;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(kFull, x, o);
        if (lane >= o)
            x += y;
    }
    if (lane == 31)
        tmp[w] = x;
    __syncthreads();
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
    __syncthreads();
    T r = (w ? tmp[w - 1] : T(0)) + x - v;
    total = tmp[W - 1];
    __syncthreads();
    return r;
}

template <int B, typename T>
__device__ __forceinline__ T block_reduce_max(T v, T* tmp)
{
    constexpr int W = B / 32;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        T y = __shfl_xor_sync(kFull, v, o);
        v = v > y ? v : y;
    }
    if (lane == 0)
        tmp[w] = v;
    __syncthreads();
    T r = tmp[0];
    for (int i = 1; i < W; ++i)
        r = r > tmp[i] ? r : tmp[i];
    __syncthreads();
    return r;
}

template <int B, typename T>
__device__ __forceinline__ T block_reduce_sum(T v, T* tmp)
{
    constexpr int W = B / 32;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(kFull, v, o);
    if (lane == 0)
        tmp[w] = v;
    __syncthreads();
    T r = 0;
    for (int i = 0; i < W; ++i)
        r += tmp[i];
    __syncthreads();
    return r;
}

// ---------------------------------------------------------------------------
// Team: one CTA, or all CTAs of a cooperative launch (grid barrier).
// ---------------------------------------------------------------------------
struct Team {
    GridSync* gs;        // nullptr for a one-CTA team
    uint32_t size;       // CTAs in the team
    uint32_t rank;       // this CTA
    uint32_t expected;   // arrivals a barrier waits for (size + phantom)
    unsigned int gen;    // local barrier generation
    unsigned long long wait_ns;
    DevResult* res;

    // Returns false if the team must stop (error anywhere or timeout).
    __device__ bool sync(uint32_t where)
    {
        __shared__ int s_ok;
        if (gs == nullptr) {
            // one CTA: thread 0 reads the status once so that every thread
            // takes the same branch afterwards
            __syncthreads();
            if (threadIdx.x == 0)
                s_ok = read_status(res) == 0;
            __syncthreads();
            return s_ok != 0;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int ok = 1;
            __threadfence();
            unsigned int prev = atomicAdd(&gs->arrive, 1u);
            if (prev == expected - 1) {
                atomicExch(&gs->arrive, 0u);
                __threadfence();
                st_release(&gs->gen, gen + 1);
            } else {
                unsigned long long t0 = globaltimer();
                unsigned int spins = 0;
                while (ld_acquire(&gs->gen) == gen) {
                    if (read_status(res) != 0) {
                        ok = 0;
                        break;
                    }
                    if ((++spins & 63u) == 0 && globaltimer() - t0 > wait_ns) {
                        set_status(res, kErrTimeout, where);
                        ok = 0;
                        break;
                    }
                    if (spins > 256)
                        __nanosleep(64);
                }
            }
            gen += 1;
            __threadfence();
            s_ok = ok && read_status(res) == 0;
        }
        __syncthreads();
        return s_ok != 0;
    }
};

// ---------------------------------------------------------------------------
// Shared memory of one CTA.
// ---------------------------------------------------------------------------
template <int B, int EMAX>
struct Smem {
    static constexpr int W = B / 32;
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
    uint32_t so_idx[EMAX];       // sorted position -> compacted index
    uint32_t so_eoff[EMAX + 1];  // edge offset of the child at sorted position
    uint32_t tmp32[W + 1];
    unsigned long long tmp64[W + 1];
    uint32_t hist[256];
    // chunk scalars
    uint32_t m, Ec, Q, Qdeg, hub;
    uint32_t bcast[8];
};

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

    // Loads up to B parents starting at position p (< pend) and forms the
    // next chunk: the longest run with <= EMAX edges.  Sets s.m (0 = the
    // first parent is a hub; s.hub = 1 then) and s.Ec.  Returns the number of
    // parents consumed (the hub counts as 1).
    __device__ uint32_t form(uint32_t p, uint32_t pend)
    {
        const uint32_t t = threadIdx.x;
        uint32_t deg = 0;
        const bool have = p + t < pend;
        if (have) {
            uint32_t pos = p + t;
            if (PB_CHECK(M.res, pos < M.n, 101)) {
                uint4 r = __ldcg(reinterpret_cast<const uint4*>(M.rec) + pos);
                s.pn[t] = r.x;
                s.prs[t] = r.y;
                s.pdeg[t] = r.z;
                s.peb[t] = r.w;
                deg = r.z;
            }
        }
        uint32_t total;
        uint32_t excl = block_exclusive_scan<B, uint32_t>(deg, total, s.tmp32);
        // parents whose inclusive edge count stays within EMAX
        uint32_t incl = excl + deg;
        int fits = have && incl <= (uint32_t)EMAX && excl <= (uint32_t)EMAX;
        int m = __syncthreads_count(fits);
        // incl is monotone in t, so the fitting parents are a prefix
        if (fits)
            s.soff[t] = excl;
        if (t == 0) {
            s.m = (uint32_t)m;
            s.hub = (m == 0 && p < pend) ? 1u : 0u;
        }
        __syncthreads();
        if (t == (uint32_t)(m > 0 ? m - 1 : 0) && m > 0)
            s.soff[m] = incl;
        if (t == 0 && m == 0)
            s.soff[0] = 0;
        __syncthreads();
        if (t == 0)
            s.Ec = m > 0 ? s.soff[m] : 0;
        __syncthreads();
        return m > 0 ? (uint32_t)m : (p < pend ? 1u : 0u);
    }

    // Finds the child edges of the chunk, compacts them, sorts every parent's
    // children (sorted = by valence, stable; else slot order) and computes the
    // edge offsets of the sorted children.  Returns (children, valence sum).
    __device__ Agg collect(bool sorted)
    {
        const uint32_t t = threadIdx.x;
        const uint32_t m = s.m, Ec = s.Ec;
        if (t < m)
            s.cc[t] = 0;
        const uint32_t ept = (Ec + B - 1) / B;
        const uint32_t e0 = t * ept;
        const uint32_t e1 = min(e0 + ept, Ec);
        // parent of e0: largest j with soff[j] <= e0
        uint32_t j = 0;
        if (e0 < e1) {
            uint32_t lo = 0, hi = m;  // soff[lo] <= e0 < soff[hi]
            while (hi - lo > 1) {
                uint32_t mid = (lo + hi) >> 1;
                if (s.soff[mid] <= e0)
                    lo = mid;
                else
                    hi = mid;
            }
            j = lo;
        }
        __syncthreads();  // cc zeroed
        uint32_t c[MAXEPT], jj[MAXEPT], key[MAXEPT], kk[MAXEPT];
#pragma unroll
        for (int r = 0; r < MAXEPT; ++r) {
            const uint32_t e = e0 + r;
            c[r] = kUnvisited;
            if (e < e1) {
                while (s.soff[j + 1] <= e)
                    ++j;
                uint32_t k = e - s.soff[j];
                uint32_t idx = s.prs[j] + k;
                jj[r] = j;
                kk[r] = k;
                key[r] = s.peb[j] + k + 1;
                if (PB_CHECK(M.res, idx < M.nnz, 102))
                    c[r] = ld_ro(M.ci + idx);
            }
        }
        uint32_t cl[MAXEPT];
#pragma unroll
        for (int r = 0; r < MAXEPT; ++r) {
            cl[r] = 0;
            if (c[r] != kUnvisited && PB_CHECK(M.res, c[r] < M.n, 103))
                cl[r] = ld_cg(M.claim + c[r]);
        }
        uint32_t r0[MAXEPT], r1[MAXEPT];
        uint32_t nvalid = 0;
#pragma unroll
        for (int r = 0; r < MAXEPT; ++r) {
            const bool valid = c[r] != kUnvisited && c[r] < M.n && cl[r] == key[r];
            if (valid) {
                r0[r] = ld_ro(M.rp + c[r]);
                r1[r] = ld_ro(M.rp + c[r] + 1);
                ++nvalid;
            } else {
                c[r] = kUnvisited;
            }
        }
        uint32_t Q;
        uint32_t q = block_exclusive_scan<B, uint32_t>(nvalid, Q, s.tmp32);
#pragma unroll
        for (int r = 0; r < MAXEPT; ++r) {
            const uint32_t e = e0 + r;
            if (e < e1) {
                if (kk[r] == 0)
                    s.cs[jj[r]] = q;
                if (c[r] != kUnvisited) {
                    if (PB_CHECK(M.res, q < (uint32_t)EMAX, 104)) {
                        s.ch_node[q] = c[r];
                        s.ch_rs[q] = r0[r];
                        s.ch_deg[q] = r1[r] - r0[r];
                        s.ch_par[q] = jj[r];
                        atomicAdd(&s.cc[jj[r]], 1u);
                    }
                    ++q;
                }
            }
        }
        __syncthreads();
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
        __syncthreads();
        // edge offsets in sorted order (blocked exclusive scan)
        const uint32_t per = (Q + B - 1) / B;
        const uint32_t i0 = min(t * per, Q), i1 = min(i0 + per, Q);
        uint32_t loc = 0;
        for (uint32_t i = i0; i < i1; ++i)
            loc += s.ch_deg[s.so_idx[i]];
        uint32_t Qdeg;
        uint32_t off = block_exclusive_scan<B, uint32_t>(loc, Qdeg, s.tmp32);
        for (uint32_t i = i0; i < i1; ++i) {
            s.so_eoff[i] = off;
            off += s.ch_deg[s.so_idx[i]];
        }
        if (t == 0) {
            s.so_eoff[Q] = Qdeg;
            s.Q = Q;
            s.Qdeg = Qdeg;
        }
        __syncthreads();
        return Agg{Q, Qdeg};
    }

    // Writes the sorted children of the chunk at positions P0.. and edge
    // bases K0.., then claims their edges for the next level.
    __device__ void place_and_claim(uint32_t P0, uint32_t K0, bool write_perm, bool reverse)
    {
        const uint32_t t = threadIdx.x;
        const uint32_t Q = s.Q, Qdeg = s.Qdeg;
        for (uint32_t i = t; i < Q; i += B) {
            const uint32_t x = s.so_idx[i];
            const uint32_t pos = P0 + i;
            if (PB_CHECK(M.res, pos < M.n, 105)) {
                uint4 r = make_uint4(s.ch_node[x], s.ch_rs[x], s.ch_deg[x], K0 + s.so_eoff[i]);
                __stcg(reinterpret_cast<uint4*>(M.rec) + pos, r);
                if (write_perm)
                    M.perm[reverse ? M.n - 1 - pos : pos] = r.x;
            }
        }
        // claims: edge-parallel over the children's rows
        for (uint32_t f = t; f < Qdeg; f += B) {
            uint32_t lo = 0, hi = Q;  // so_eoff[lo] <= f < so_eoff[hi]
            while (hi - lo > 1) {
                uint32_t mid = (lo + hi) >> 1;
                if (s.so_eoff[mid] <= f)
                    lo = mid;
                else
                    hi = mid;
            }
            const uint32_t x = s.so_idx[lo];
            const uint32_t idx = s.ch_rs[x] + (f - s.so_eoff[lo]);
            if (PB_CHECK(M.res, idx < M.nnz, 106)) {
                const uint32_t d = ld_ro(M.ci + idx);
                if (PB_CHECK(M.res, d < M.n, 107))
                    atomicMin(M.claim + d, K0 + f + 1);
            }
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
        const uint32_t t = threadIdx.x;
        const uint32_t rs = s.prs[0], D = s.pdeg[0], eb = s.peb[0];
        if (M.hub == nullptr) {
            set_status(M.res, kErrCheck, 120);
            return Agg{0, 0};
        }
        uint32_t Q = 0;
        unsigned long long Qdeg = 0;
        uint32_t maxkey = 0;
        constexpr uint32_t TILE = B * MAXEPT;
        for (uint32_t base = 0; base < D; base += TILE) {
            uint32_t nv = 0;
            uint32_t dg[MAXEPT];
            bool ok[MAXEPT];
#pragma unroll
            for (int r = 0; r < MAXEPT; ++r) {
                const uint32_t e = base + t * MAXEPT + r;
                ok[r] = false;
                if (e < D && PB_CHECK(M.res, rs + e < M.nnz, 121)) {
                    const uint32_t c = ld_ro(M.ci + rs + e);
                    if (PB_CHECK(M.res, c < M.n, 122) && ld_cg(M.claim + c) == eb + e + 1) {
                        dg[r] = ld_ro(M.rp + c + 1) - ld_ro(M.rp + c);
                        ok[r] = true;
                        ++nv;
                    }
                }
            }
            uint32_t tot;
            uint32_t q = block_exclusive_scan<B, uint32_t>(nv, tot, s.tmp32);
            uint32_t lsum = 0, lmax = 0;
#pragma unroll
            for (int r = 0; r < MAXEPT; ++r) {
                if (ok[r]) {
                    const uint32_t w = r0 + Q + q;
                    if (PB_CHECK(M.res, w < M.nnz, 123)) {
                        hk0()[w] = dg[r];
                        hv0()[w] = base + t * MAXEPT + r;
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
        __syncthreads();
        return Agg{Q, (uint32_t)Qdeg};
    }

    // One stable counting pass on digit (key >> shift) & 255.
    __device__ void radix_pass(const uint32_t* sk, const uint32_t* sv, uint32_t* dk, uint32_t* dv, uint32_t Q,
                               uint32_t shift)
    {
        const uint32_t t = threadIdx.x, lane = t & 31, w = t >> 5;
        for (uint32_t d = t; d < 256; d += B)
            s.hist[d] = 0;
        __syncthreads();
        for (uint32_t i = t; i < Q; i += B)
            atomicAdd(&s.hist[(__ldcg(sk + i) >> shift) & 255u], 1u);
        __syncthreads();
        if (t == 0) {
            uint32_t run = 0;
            for (int d = 0; d < 256; ++d) {
                uint32_t h = s.hist[d];
                s.hist[d] = run;
                run += h;
            }
        }
        __syncthreads();
        for (uint32_t base = 0; base < Q; base += B) {
            for (uint32_t i = t; i < (uint32_t)(Smem<B, EMAX>::W * 256); i += B)
                s.hcnt[i] = 0;
            __syncthreads();
            const uint32_t i = base + t;
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
            __syncthreads();
            if (act) {
                uint32_t before = 0;
                for (uint32_t ww = 0; ww < w; ++ww)
                    before += s.hcnt[ww * 256 + dgt];
                const uint32_t dst = s.hist[dgt] + before + rank_w;
                dk[dst] = key;
                dv[dst] = val;
            }
            __syncthreads();
            for (uint32_t d = t; d < 256; d += B) {
                uint32_t add = 0;
                for (int ww = 0; ww < Smem<B, EMAX>::W; ++ww)
                    add += s.hcnt[ww * 256 + d];
                s.hist[d] += add;
            }
            __syncthreads();
        }
    }

    // Places the sorted hub children (count Q) at P0.. / K0.. in tiles of
    // EMAX, reusing the chunk arrays, and claims their edges.
    __device__ void hub_place_and_claim(uint32_t r0, uint32_t Q, uint32_t P0, uint32_t K0, bool write_perm,
                                        bool reverse)
    {
        const uint32_t t = threadIdx.x;
        const uint32_t rs = s.prs[0];
        uint32_t done = 0, kdone = 0;
        while (done < Q) {
            const uint32_t cnt = min((uint32_t)EMAX, Q - done);
            uint32_t loc = 0;
            // blocked layout for the scan
            const uint32_t per = (cnt + B - 1) / B;
            const uint32_t i0 = min(t * per, cnt), i1 = min(i0 + per, cnt);
            for (uint32_t i = i0; i < i1; ++i) {
                const uint32_t slot = __ldcg(hv0() + r0 + done + i);
                const uint32_t node = ld_ro(M.ci + rs + slot);
                const uint32_t a = ld_ro(M.rp + node), b = ld_ro(M.rp + node + 1);
                s.ch_node[i] = node;
                s.ch_rs[i] = a;
                s.ch_deg[i] = b - a;
                s.so_idx[i] = i;
                loc += b - a;
            }
            uint32_t tot;
            uint32_t off = block_exclusive_scan<B, uint32_t>(loc, tot, s.tmp32);
            for (uint32_t i = i0; i < i1; ++i) {
                s.so_eoff[i] = off;
                off += s.ch_deg[i];
            }
            if (t == 0) {
                s.so_eoff[cnt] = tot;
                s.Q = cnt;
                s.Qdeg = tot;
            }
            __syncthreads();
            place_and_claim(P0 + done, K0 + kdone, write_perm, reverse);
            __syncthreads();
            done += cnt;
            kdone += tot;
        }
    }
};

// ---------------------------------------------------------------------------
// One ordered BFS pass from `start`.  Fills rec[0..placed) and, when
// write_perm, the output.  Returns false if the team must stop.
// level_out: number of levels; last_start: first position of the last level.
// ---------------------------------------------------------------------------
template <int B, int EMAX>
__device__ bool bfs_pass(Smem<B, EMAX>& s, const MatrixView& M, Team& team, unsigned long long* agg, uint32_t start,
                         bool sorted, bool write_perm, bool reverse, uint32_t& placed, uint32_t& nlevels,
                         uint32_t& last_start)
{
    Chunk<B, EMAX> ch{s, M};
    const uint32_t t = threadIdx.x;
    const uint32_t G = team.size, R = team.rank;
    const uint32_t n = M.n;

    // reset claims
    for (uint64_t i = (uint64_t)R * B + t; i < n; i += (uint64_t)G * B)
        M.claim[i] = kUnvisited;
    if (!team.sync(1))
        return false;

    // seed the start (CTA 0 places it and claims its edges)
    const uint32_t rs0 = ld_ro(M.rp + start), deg0 = ld_ro(M.rp + start + 1) - rs0;
    if (R == 0) {
        if (t == 0) {
            atomicMin(M.claim + start, 0u);
            __stcg(reinterpret_cast<uint4*>(M.rec), make_uint4(start, rs0, deg0, 0u));
            if (write_perm)
                M.perm[reverse ? n - 1 : 0] = start;
        }
        for (uint32_t k = t; k < deg0; k += B) {
            const uint32_t d = ld_ro(M.ci + rs0 + k);
            if (PB_CHECK(M.res, d < n, 110))
                atomicMin(M.claim + d, k + 1);
        }
    }
    if (!team.sync(2))
        return false;

    uint32_t a = 0, b = 1, Kb = deg0, Ka = 0;
    uint32_t L = 0;
    last_start = 0;
    while (true) {
        const uint32_t F = b - a;
        // this CTA's parents
        const uint32_t p_beg = a + (uint32_t)(((uint64_t)F * R) / G);
        const uint32_t p_end = a + (uint32_t)(((uint64_t)F * (R + 1)) / G);
        uint32_t tot_cnt = 0, tot_esum = 0;
        if (G == 1) {
            // collect and place chunk by chunk
            uint32_t P = b, K = Kb;
            uint32_t p = p_beg;
            while (p < p_end) {
                const uint32_t used = ch.form(p, p_end);
                if (s.hub) {
                    const uint32_t r0 = s.peb[0] - Ka;
                    Agg g = ch.hub_collect(r0, sorted);
                    ch.hub_place_and_claim(r0, g.cnt, P, K, write_perm, reverse);
                    P += g.cnt;
                    K += g.esum;
                } else {
                    Agg g = ch.collect(sorted);
                    ch.place_and_claim(P, K, write_perm, reverse);
                    P += g.cnt;
                    K += g.esum;
                }
                __syncthreads();
                p += used;
            }
            tot_cnt = P - b;
            tot_esum = K - Kb;
            if (!team.sync(3))
                return false;
        } else {
            // A1: count
            uint32_t my_cnt = 0, my_esum = 0, nunits = 0;
            uint32_t p = p_beg;
            while (p < p_end) {
                const uint32_t used = ch.form(p, p_end);
                Agg g;
                if (s.hub)
                    g = ch.hub_collect(s.peb[0] - Ka, sorted);
                else
                    g = ch.collect(sorted);
                my_cnt += g.cnt;
                my_esum += g.esum;
                ++nunits;
                p += used;
                __syncthreads();
            }
            if (t == 0)
                __stcg(agg + R, ((unsigned long long)my_esum << 32) | my_cnt);
            if (!team.sync(4))
                return false;
            // prefix of the CTAs before this one, and the level total
            unsigned long long pre = 0, all = 0;
            for (uint32_t i = t; i < G; i += B) {
                unsigned long long v = __ldcg(agg + i);
                all += v;
                if (i < R)
                    pre += v;
            }
            pre = block_reduce_sum<B, unsigned long long>(pre, s.tmp64);
            all = block_reduce_sum<B, unsigned long long>(all, s.tmp64);
            tot_cnt = (uint32_t)(all & 0xFFFFFFFFull);
            tot_esum = (uint32_t)(all >> 32);
            uint32_t P = b + (uint32_t)(pre & 0xFFFFFFFFull);
            uint32_t K = Kb + (uint32_t)(pre >> 32);
            // A2: place (the last unit is still in shared memory if it was the only one)
            if (nunits == 1 && !s.hub) {
                ch.place_and_claim(P, K, write_perm, reverse);
            } else {
                p = p_beg;
                while (p < p_end) {
                    const uint32_t used = ch.form(p, p_end);
                    if (s.hub) {
                        const uint32_t r0 = s.peb[0] - Ka;
                        const uint32_t q = __ldcg(ch.hk1() + r0);
                        const uint32_t qd = __ldcg(ch.hk1() + r0 + 1);
                        ch.hub_place_and_claim(r0, q, P, K, write_perm, reverse);
                        P += q;
                        K += qd;
                    } else {
                        Agg g = ch.collect(sorted);
                        ch.place_and_claim(P, K, write_perm, reverse);
                        P += g.cnt;
                        K += g.esum;
                    }
                    __syncthreads();
                    p += used;
                }
            }
            if (!team.sync(5))
                return false;
        }
        if (tot_cnt == 0)
            break;
        last_start = b;
        a = b;
        b += tot_cnt;
        Ka = Kb;
        Kb += tot_esum;
        ++L;
        if (b > n) {
            set_status(M.res, kErrCheck, 111);
            return false;
        }
    }
    placed = b;
    nlevels = L + 1;
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
        uint4 r = __ldcg(reinterpret_cast<const uint4*>(M.rec) + pos);
        if (r.z <= bestdeg) {
            bestdeg = r.z;
            best = r.x;
        }
    }
    return best;
}

// ---------------------------------------------------------------------------
// Full reorder of one matrix by one team: start search, final ordered pass,
// bandwidth.  Every CTA of the team runs this; CTA 0 thread 0 writes *res.
// ---------------------------------------------------------------------------
template <int B, int EMAX>
__device__ void reorder_matrix(Smem<B, EMAX>& s, const MatrixView& M, Team& team, unsigned long long* agg,
                               const Options& opt)
{
    const uint32_t t = threadIdx.x;
    const uint32_t n = M.n;
    uint32_t start = opt.start;
    uint32_t passes = 0, ecc = 0, placed = 0, nlevels = 0, last_start = 0;

    if (start != kUnvisited && start >= n) {
        if (team.rank == 0 && t == 0)
            set_status(M.res, kErrArg, 2);
        return;
    }
    if (n == 1) {
        // one node: the start search runs one pass and records nothing
        passes = start == kUnvisited ? 1 : 0;
        start = 0;
    } else if (start == kUnvisited) {
        // pseudo-peripheral search (simple_peripheral.cpp:92-141)
        start = n / 2;
        uint32_t lastdist = 0;
        while (true) {
            ++passes;
            if (!bfs_pass<B, EMAX>(s, M, team, agg, start, false, false, false, placed, nlevels, last_start))
                return;
            if (placed != n) {
                if (team.rank == 0 && t == 0)
                    set_status(M.res, kErrDisconnected, 0);
                return;
            }
            const uint32_t dist = nlevels - 1;
            if (dist == lastdist) {
                ecc = dist;
                break;
            }
            if (passes > n) {  // eccentricities only grow; cannot happen on a valid run
                if (team.rank == 0 && t == 0)
                    set_status(M.res, kErrCheck, 3);
                return;
            }
            if (t == 0)
                s.bcast[0] = next_peripheral_start(M, opt.outnodes, last_start);
            __syncthreads();
            start = s.bcast[0];
            lastdist = dist;
            __syncthreads();
        }
    }
    if (opt.mode == kModeStartOnly) {
        if (team.rank == 0 && t == 0) {
            M.res->start = start;
            M.res->passes = passes;
            M.res->ecc = ecc;
            M.res->placed = n;
        }
        return;
    }
    // the final, degree-sorted pass writes the permutation
    if (!bfs_pass<B, EMAX>(s, M, team, agg, start, true, true, opt.reverse != 0, placed, nlevels, last_start))
        return;
    if (placed != n) {
        if (team.rank == 0 && t == 0) {
            set_status(M.res, kErrDisconnected, 1);
            M.res->placed = placed;
        }
        return;
    }

    if (opt.want_bw) {
        const uint32_t G = team.size, R = team.rank;
        // inverse permutation (CM positions) into claim[]
        for (uint64_t pos = (uint64_t)R * B + t; pos < n; pos += (uint64_t)G * B) {
            uint4 r = __ldcg(reinterpret_cast<const uint4*>(M.rec) + pos);
            M.claim[r.x] = (uint32_t)pos;
        }
        if (!team.sync(6))
            return;
        unsigned long long bw = 0, bw0 = 0, plo = 0, phi = 0;
        for (uint64_t i = (uint64_t)R * B + t; i < n; i += (uint64_t)G * B) {
            const uint32_t a = ld_ro(M.rp + i), e = ld_ro(M.rp + i + 1);
            if (a == e)
                continue;
            const uint32_t me = __ldcg(M.claim + i);
            uint32_t mn = me, mx = me, mnr = kUnvisited, mxr = 0;
            for (uint32_t k = a; k < e; ++k) {
                const uint32_t p = __ldcg(M.claim + ld_ro(M.ci + k));
                mnr = min(mnr, p);
                mxr = max(mxr, p);
            }
            mn = min(mn, mnr);
            mx = max(mx, mxr);
            // computeBandwidth (main.cpp:143-184): max(row - min, max - row), >= 0
            const unsigned long long b1 = me >= mnr ? (unsigned long long)(me - mnr) : 0ull;
            const unsigned long long b2 = mxr >= me ? (unsigned long long)(mxr - me) : 0ull;
            bw = max(bw, max(b1, b2));
            // profile of the CM order and of its reverse
            plo += (unsigned long long)(me - mn);
            phi += (unsigned long long)(mx - me);
            // initial bandwidth: first / last stored column (main.cpp:114-129)
            const uint32_t c0 = ld_ro(M.ci + a), c1 = ld_ro(M.ci + e - 1);
            unsigned long long i0 = i >= c0 ? i - c0 : 0, i1 = c1 >= i ? c1 - i : 0;
            bw0 = max(bw0, max(i0, i1));
        }
        bw = block_reduce_max<B, unsigned long long>(bw, s.tmp64);
        bw0 = block_reduce_max<B, unsigned long long>(bw0, s.tmp64);
        plo = block_reduce_sum<B, unsigned long long>(plo, s.tmp64);
        phi = block_reduce_sum<B, unsigned long long>(phi, s.tmp64);
        if (t == 0) {
            atomicMax(&M.res->bandwidth, bw);
            atomicMax(&M.res->initial_bw, bw0);
            atomicAdd(&M.res->profile_lo, plo);
            atomicAdd(&M.res->profile_hi, phi);
        }
    }
    if (team.rank == 0 && t == 0) {
        M.res->start = start;
        M.res->passes = passes;
        M.res->ecc = ecc;
        M.res->levels = nlevels;
        M.res->placed = placed;
    }
}

}  // namespace pbrcm
