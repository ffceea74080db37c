// solo.cuh -- the one-group engine of the batch kernels: the whole reorder of
// one matrix (start search, Cuthill-McKee pass, reverse, bandwidth) by one
// thread group, with the visited set in shared memory.
//
// What it computes is what engine.cuh computes (the serial stable order of
// src/rcm_cpu.cpp:57-104 from the start node of
// src/simple_peripheral.cpp:92-141, and the bandwidth of src/main.cpp:143-184);
// how differs, because a group that owns its matrix alone needs no claim
// protocol:
//
//   * the queue is walked in chunks of consecutive positions (at most B
//     parents and EMAX edges, never across a level boundary); a chunk's
//     children are the still-unvisited neighbours, each taken by the first
//     (parent, slot) that reaches it -- exactly the serial loop, since every
//     node an earlier chunk placed is already marked;
//   * visited is a bitmap in shared memory (n <= kSoloMaxN), so checking a
//     neighbour costs no global load and marking one no atomic in global
//     memory; a larger matrix keeps the bitmap in global memory (n / 8
//     bytes, L2-resident: one L2 round trip more per chunk); inside a chunk a
//     shared-memory hash keeps the first edge to a node (atomicMin of the
//     edge index);
//   * every entry's neighbour record -- its column and that column's row
//     start and valence -- is one 8-byte record of an edge table built once
//     per matrix (solo_build_edges, during the CSR check), so a chunk needs
//     one dependent global load per edge (coalesced along each row) instead
//     of a column load followed by a node-table load; the queue holds the
//     same 8-byte records (node and valence in one word, row start in the
//     other: n <= kSoloMaxNodes, valences < 4,096);
//   * the children of a chunk that is a whole level, if they fit one chunk,
//     stay in shared memory as the next chunk's parents.
//
// Per chunk: each edge's parent by a binary search of the parents' edge
// offsets, the edge records, the visited test and the dedup-table insert, a
// warp-ballot compaction in edge order, the rank of each parent's children
// by (valence, slot), the writes of the queue records and the permutation,
// and the visited marks -- four group barriers in the chunk and three where
// its parents are formed.
#pragma once

#include "engine.cuh"

namespace pbrcm {

constexpr uint32_t kSoloEmpty = 0xFFFFFFFFu;

// Shared memory of one solo group (B threads, EMAX edges per chunk).
template <int B, int EMAX>
struct SoloSmem {
    static constexpr int W = B / 32;
    static constexpr int H = 2 * EMAX;  // dedup table slots (power of two, > 2x a chunk's candidates)
    uint32_t vis[kSoloMaxN / 32];
    // parents of the chunk
    uint32_t pn[B], prs[B], pdeg[B];
    uint32_t soff[B + 1];
    uint32_t cs[B], cc[B];  // first compacted child / child count per parent (clear between chunks)
    // the dedup table: (node << kEdgeBits | chunk edge) of the first edge to
    // each unvisited node of the chunk; kSoloEmpty where free (clear between
    // chunks)
    uint32_t tab[H];
    uint32_t so_idx[EMAX];  // the children's ranked order: rank -> compacted index
    // the chunk's children in edge order: node, row start, and valence with
    // the parent's chunk index in the high bits (valence < 2^kParShift)
    uint32_t ch_c[EMAX], ch_rs[EMAX], ch_dp[EMAX];
    uint32_t wcnt[W], wdeg[W];
    uint32_t scanbuf[2][W];
    uint32_t tmp32[W + 1];
    unsigned long long tmp64[2 * W + 2];
    uint32_t m, Ec;
    uint32_t bcast[4];
};

// Chunk edge indices take kEdgeBits bits below the node in a dedup word
// (nodes < 2^20, chunks of at most 2,048 edges: 31 bits).
constexpr uint32_t kEdgeBits = 11;
constexpr uint32_t kParShift = 20;  // ch_dp: valence in the low 20 bits, parent index above
constexpr uint32_t kDegMask = (1u << kParShift) - 1u;

// Edge and queue records of the solo engine: (node | valence << 20, row
// start).  A record word never equals kSoloEmpty (valences stay below 4,096).
constexpr uint32_t kRecNodeBits = 20;
constexpr uint32_t kRecNodeMask = (1u << kRecNodeBits) - 1u;
__device__ __forceinline__ uint2 solo_rec(uint32_t node, uint32_t deg, uint32_t rs)
{
    return make_uint2(node | (deg << kRecNodeBits), rs);
}
__device__ __forceinline__ uint32_t rec_node(uint2 r) { return r.x & kRecNodeMask; }
__device__ __forceinline__ uint32_t rec_deg(uint2 r) { return r.x >> kRecNodeBits; }

// Requests the lines of e2[rs .. rs + deg) into L2 (at most four 128-byte
// lines: the rows the engine chunks are short), without waiting.
__device__ __forceinline__ void prefetch_row(const uint2* e2, uint32_t rs, uint32_t deg)
{
    if (deg == 0)
        return;
    const uintptr_t a = reinterpret_cast<uintptr_t>(e2 + rs) & ~(uintptr_t)127;
    const uintptr_t z = reinterpret_cast<uintptr_t>(e2 + rs + deg - 1) & ~(uintptr_t)127;
    for (uintptr_t l = a; l <= z && l < a + 4 * 128; l += 128)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(l));
}

template <int B, int EMAX>
struct Solo {
    static constexpr int MAXEPT = EMAX / B;
    static_assert(EMAX % B == 0 && (EMAX & (EMAX - 1)) == 0, "EMAX: a power of two, a multiple of B");
    static_assert(EMAX <= (1 << kEdgeBits), "a chunk edge index fits the dedup word");
    SoloSmem<B, EMAX>& s;
    const MatrixView& M;
    const uint2* e2;
    uint2* q;  // the queue: rec[] of the matrix as 8-byte records
    uint32_t* gvis;  // visited bitmap in global memory (matrices over kSoloMaxN nodes), or nullptr
    // queue record of position pf_base + (group thread), loaded by the last
    // form() for the chunk after it (its latency hides behind that chunk);
    // pf_base == kUnvisited: none
    uint32_t pf_base = kUnvisited;
    uint2 pf = make_uint2(0u, 0u);
    bool pf_ok = false;  // this thread holds a record in pf

    __device__ __forceinline__ bool visited(uint32_t c) const
    {
        const uint32_t w = gvis ? __ldcg(gvis + (c >> 5)) : s.vis[c >> 5];
        return (w >> (c & 31)) & 1u;
    }
    __device__ __forceinline__ void mark(uint32_t c)
    {
        atomicOr(gvis ? gvis + (c >> 5) : &s.vis[c >> 5], 1u << (c & 31));
    }

    // Loads the next chunk's parents from the queue records rec[p .. pend):
    // the longest prefix of at most B parents with at most EMAX edges (every
    // row fits one chunk: the engine is only used when the largest valence
    // is at most EMAX).  Returns the number of parents.
    __device__ uint32_t form(uint32_t p, uint32_t pend)
    {
        const uint32_t t = gtid<B>();
        uint32_t deg = 0;
        const bool have = p + t < pend;
        if (have) {
            const uint2 r = p == pf_base ? pf : __ldcg(q + p + t);
            deg = rec_deg(r);
            s.pn[t] = rec_node(r);
            s.prs[t] = r.y;
            s.pdeg[t] = deg;
        }
        uint32_t total;
        const uint32_t excl = block_scan1<B>(deg, total, s.scanbuf[0]);
        const uint32_t incl = excl + deg;
        const int fits = have && incl <= (uint32_t)EMAX;
        const int m = gsync_count<B>(fits);
        if (fits)
            s.soff[t] = excl;
        if (m > 0 && t == (uint32_t)(m - 1)) {
            s.soff[m] = incl;
            s.m = (uint32_t)m;
            s.Ec = incl;
        }
        // the next chunk of this level starts where this one ends: load its
        // records now
        const uint32_t nb = p + (uint32_t)m;
        pf_base = kUnvisited;
        pf_ok = false;
        if (nb < pend) {
            pf_base = nb;
            if (nb + t < pend) {
                pf = __ldcg(q + nb + t);
                pf_ok = true;
            }
        }
        gsync<B>();
        return (uint32_t)m;
    }

    // next_peripheral_start (engine.cuh) over this queue's 8-byte records:
    // among the last min(outnodes, n-1) positions, those on the last level;
    // the last of minimal valence.  One thread.
    __device__ uint32_t next_start(uint32_t outnodes, uint32_t last_start) const
    {
        const uint32_t n = M.n;
        uint32_t lo = n - min(outnodes, n - 1);
        lo = max(lo, max(last_start, 1u));
        uint32_t best = 0, bestdeg = kUnvisited;
        for (uint32_t pos = lo; pos < n; ++pos) {
            const uint2 r = __ldcg(q + pos);
            if (rec_deg(r) <= bestdeg) {
                bestdeg = rec_deg(r);
                best = rec_node(r);
            }
        }
        return best;
    }

    // The Q ranked children of the last chunk become the parents of the next.
    __device__ void form_from_children(uint32_t Q)
    {
        const uint32_t t = gtid<B>();
        uint32_t deg = 0;
        if (t < Q) {
            const uint32_t x = s.so_idx[t];
            deg = s.ch_dp[x] & kDegMask;
            s.pn[t] = s.ch_c[x];
            s.prs[t] = s.ch_rs[x];
            s.pdeg[t] = deg;
        }
        uint32_t total;
        const uint32_t excl = block_scan1<B>(deg, total, s.scanbuf[1]);
        if (t < Q)
            s.soff[t] = excl;
        if (t == 0) {
            s.soff[Q] = total;
            s.m = Q;
            s.Ec = total;
        }
        gsync<B>();
    }

    // One chunk: finds the children of parents [0, m), ranks them (sorted:
    // by valence, stable; else slot order), writes their queue records at
    // positions P.. and, with write_perm, the permutation, and marks them
    // visited.  Returns the number of children; qdeg = their valences' sum.
    // Four group barriers.  Ends without one: the next form() has barriers
    // before anyone touches this chunk's shared buffers again (the caller
    // adds one where the next chunk reads the queue records this one
    // wrote).  Leaves the dedup table and the parent counters clear.
    __device__ uint32_t step(uint32_t P, bool sorted, bool write_perm, bool reverse, uint32_t& qdeg)
    {
        const uint32_t t = gtid<B>(), lane = t & 31u, w = t >> 5;
        const uint32_t m = s.m, Ec = s.Ec;
        // warp w owns edges [w * 32 * MAXEPT, ...); lane l takes e = base +
        // l + 32 r, so that a warp reads consecutive records of a row
        const uint32_t base = w * 32u * MAXEPT;
        uint2 v[MAXEPT];
        uint32_t par[MAXEPT], slot[MAXEPT];
        bool cand[MAXEPT];
        // each edge's parent (the last j < m with soff[j] <= e: a binary
        // search of fixed depth, the edges' searches side by side; a parent
        // of valence 0 owns no edge), then the edge's record
#pragma unroll
        for (int r = 0; r < MAXEPT; ++r) {
            const uint32_t e = base + lane + 32u * r;
            uint32_t lo = 0;
#pragma unroll
            for (uint32_t d = (uint32_t)B / 2u; d > 0; d >>= 1) {
                const uint32_t mid = lo + d;
                if (mid < m && s.soff[mid] <= e)
                    lo = mid;
            }
            par[r] = lo;
            v[r] = make_uint2(kSoloEmpty, 0u);
            if (e < Ec) {
                const uint64_t idx = (uint64_t)s.prs[lo] + (e - s.soff[lo]);
                if (PB_CHECK(M.res, idx < M.nnz, 601))
                    v[r] = __ldcg(e2 + idx);
            }
        }
        // the next chunk's rows into L2 while these records are in flight
        // (its queue records came with the last form())
        if (pf_ok)
            prefetch_row(e2, pf.y, rec_deg(pf));
        // the visited test after all the records are in flight
#pragma unroll
        for (int r = 0; r < MAXEPT; ++r)
            cand[r] = v[r].x != kSoloEmpty && PB_CHECK(M.res, rec_node(v[r]) < M.n, 602) && !visited(rec_node(v[r]));
        // first edge to each unvisited node: (node, edge) in one word, so
        // that the word's minimum under a fixed node is the first edge; the
        // node's slot by linear probing (at most EMAX distinct nodes in 2
        // EMAX slots: a free slot is always found)
        constexpr uint32_t mask = (uint32_t)SoloSmem<B, EMAX>::H - 1u;
#pragma unroll
        for (int r = 0; r < MAXEPT; ++r) {
            slot[r] = 0;
            if (cand[r]) {
                const uint32_t c = rec_node(v[r]);
                const uint32_t key = (c << kEdgeBits) | (base + lane + 32u * r);
                uint32_t h = (c * 2654435761u) & mask;
                while (true) {
                    const uint32_t old = atomicCAS(&s.tab[h], kSoloEmpty, key);
                    if (old == kSoloEmpty)
                        break;
                    if ((old >> kEdgeBits) == c) {
                        atomicMin(&s.tab[h], key);
                        break;
                    }
                    h = (h + 1u) & mask;
                }
                slot[r] = h;
            }
        }
        gsync<B>();
        // the winners, compacted in edge order: per warp by ballot, then the
        // warps' counts
        uint32_t cnt = 0, posr[MAXEPT], dsum = 0;
        bool win[MAXEPT];
#pragma unroll
        for (int r = 0; r < MAXEPT; ++r) {
            win[r] = cand[r] && s.tab[slot[r]] == ((rec_node(v[r]) << kEdgeBits) | (base + lane + 32u * r));
            const uint32_t bal = __ballot_sync(kFull, win[r]);
            posr[r] = cnt + __popc(bal & ((1u << lane) - 1u));
            cnt += __popc(bal);
            dsum += win[r] ? rec_deg(v[r]) : 0u;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            dsum += __shfl_xor_sync(kFull, dsum, o);
        if (lane == 0) {
            s.wcnt[w] = cnt;
            s.wdeg[w] = dsum;
        }
        gsync<B>();
        uint32_t wbase = 0, Q = 0;
        qdeg = 0;
#pragma unroll
        for (int i = 0; i < SoloSmem<B, EMAX>::W; ++i) {
            const uint32_t c = s.wcnt[i];
            wbase += (uint32_t)i < w ? c : 0u;
            Q += c;
            qdeg += s.wdeg[i];
        }
#pragma unroll
        for (int r = 0; r < MAXEPT; ++r) {
            if (win[r]) {
                const uint32_t x = wbase + posr[r];
                const uint32_t j = par[r];
                s.ch_c[x] = rec_node(v[r]);
                s.ch_rs[x] = v[r].y;
                s.ch_dp[x] = rec_deg(v[r]) | (j << kParShift);
                atomicAdd(&s.cc[j], 1u);
                atomicMin(&s.cs[j], x);
            }
        }
        gsync<B>();
        // rank inside each parent's run: (valence, position) when sorted
        for (uint32_t x = t; x < Q; x += B) {
            const uint32_t j = s.ch_dp[x] >> kParShift;
            const uint32_t st = s.cs[j], len = s.cc[j];
            uint32_t rank = x - st;
            if (sorted && len > 1) {
                const uint32_t dx = s.ch_dp[x] & kDegMask;
                rank = 0;
                for (uint32_t y = st; y < st + len; ++y) {
                    const uint32_t dy = s.ch_dp[y] & kDegMask;
                    rank += (dy < dx) || (dy == dx && y < x);
                }
            }
            s.so_idx[st + rank] = x;
        }
        gsync<B>();
        // place: queue records, the permutation, the visited marks
        for (uint32_t i = t; i < Q; i += B) {
            const uint32_t x = s.so_idx[i];
            const uint32_t pos = P + i;
            if (PB_CHECK(M.res, pos < M.n, 603)) {
                __stcg(q + pos, solo_rec(s.ch_c[x], s.ch_dp[x] & kDegMask, s.ch_rs[x]));
                if (write_perm)
                    M.perm[reverse ? M.n - 1 - pos : pos] = s.ch_c[x];
            }
            mark(s.ch_c[x]);
        }
        // the table slots and parent counters this chunk used, clear again
        // (their last readers are behind the barriers above)
#pragma unroll
        for (int r = 0; r < MAXEPT; ++r)
            if (cand[r])
                s.tab[slot[r]] = kSoloEmpty;
        for (uint32_t j = t; j < m; j += B) {
            s.cs[j] = kSoloEmpty;
            s.cc[j] = 0;
        }
        return Q;
    }
};

// The per-edge neighbour records of a matrix (e2[k] = solo_rec(c, rp[c+1] -
// rp[c], rp[c]) for c = ci[k]) by one group, coalesced.  A column out of
// range gets an empty record (the CSR check reports it); a valence of 4,096
// or more does not fit a record, but such a matrix never reaches the solo
// engine (its rows exceed every chunk).
template <int B>
__device__ void solo_build_edges(const MatrixView& M, uint2* e2)
{
    bool bad = false;
#pragma unroll 8
    for (uint32_t k = gtid<B>(); k < M.nnz; k += B) {
        const uint32_t c = ld_ro(M.ci + k);
        uint2 r = make_uint2(kSoloEmpty, 0u);
        if (c < M.n) {
            const uint32_t a = ld_ro(M.rp + c), b = ld_ro(M.rp + c + 1);
            r = solo_rec(c, b - a, a);
        } else {
            bad = true;
        }
        __stcg(e2 + k, r);
    }
    // the CSR check's column test (validate_rows leaves it to this pass)
    if (bad)
        set_status(M.res, kErrArg, 200);
}

// One ordered BFS pass from `start` by one solo group.  Fills rec[0 ..
// placed); returns the level count and the first position of the last level.
template <int B, int EMAX>
__device__ void solo_pass(Solo<B, EMAX>& so, uint32_t start, bool sorted, bool write_perm, bool reverse,
                          uint32_t& placed, uint32_t& nlevels, uint32_t& last_start)
{
    SoloSmem<B, EMAX>& s = so.s;
    const MatrixView& M = so.M;
    const uint32_t t = gtid<B>();
    const uint32_t words = (M.n + 31u) / 32u;
    uint32_t* vis = so.gvis ? so.gvis : s.vis;
    for (uint32_t i = t; i < words; i += B)
        vis[i] = 0u;
    // the dedup table and the parent counters start clear (each chunk
    // leaves them so)
    for (uint32_t i = t; i < (uint32_t)SoloSmem<B, EMAX>::H; i += B)
        s.tab[i] = kSoloEmpty;
    s.cs[t] = kSoloEmpty;
    s.cc[t] = 0;
    gsync<B>();
    if (t == 0) {
        const uint32_t a = ld_ro(M.rp + start), b = ld_ro(M.rp + start + 1);
        __stcg(so.q, solo_rec(start, b - a, a));
        if (write_perm)
            M.perm[reverse ? M.n - 1 : 0] = start;
        so.mark(start);
    }
    gsync<B>();
    uint32_t head = 0, tail = 1, lvl_end = 1, L = 0, lstart = 0;
    bool carry = false;  // the chunk's parents are the last chunk's children, still in shared memory
    uint32_t q = 0;
    while (head < tail) {
        if (head == lvl_end) {
            L += 1;
            lstart = head;
            lvl_end = tail;
        }
        uint32_t m;
        if (carry) {
            so.form_from_children(q);
            m = q;
        } else {
            m = so.form(head, lvl_end);
        }
        // a whole level in one chunk whose children fit one chunk: they are
        // the next chunk's parents
        const bool whole_level = head + m == lvl_end && head + m == tail;
        uint32_t qdeg = 0;
        q = so.step(tail, sorted, write_perm, reverse, qdeg);
        head += m;
        tail += q;
        carry = whole_level && q > 0 && q <= (uint32_t)B && qdeg <= (uint32_t)EMAX;
        // a chunk that ends its level hands its children over through the
        // queue records it has just written (unless they stay in shared
        // memory): every thread's records must be in before the next chunk
        // reads them.  Otherwise the next chunk's parents were written by
        // earlier chunks, behind barriers already passed.
        if (head == lvl_end && !carry)
            gsync<B>();
        if (tail > M.n) {  // cannot happen on a valid run
            if (t == 0)
                set_status(M.res, kErrCheck, 604);
            break;
        }
    }
    placed = tail;
    nlevels = L + 1;
    last_start = lstart;
}

// Full reorder of one matrix by one solo group: start search
// (simple_peripheral.cpp:92-141), the sorted pass, reverse, bandwidth.
// e2: the matrix's edge records; inv: n words for the inverse permutation;
// gvis: ceil(n / 32) words for the visited bitmap when n > kSoloMaxN (else
// nullptr: the bitmap is in shared memory).
template <int B, int EMAX>
__device__ void solo_reorder(SoloSmem<B, EMAX>& s, const MatrixView& M, const uint2* e2, uint32_t* inv,
                             uint32_t* gvis, const Options& opt)
{
    const uint32_t t = gtid<B>();
    const uint32_t n = M.n;
    if (t == 0)
        M.res->t_begin = globaltimer();
    Solo<B, EMAX> so{s, M, e2, reinterpret_cast<uint2*>(M.rec), gvis};
    uint32_t start = opt.start;
    if (start != kUnvisited && start >= n) {
        if (t == 0)
            set_status(M.res, kErrArg, 2);
        return;
    }
    uint32_t passes = 0, ecc = 0, placed = 0, nlevels = 0, last_start = 0;
    bool searching = start == kUnvisited && n > 1;
    if (n == 1) {
        passes = start == kUnvisited ? 1 : 0;
        start = 0;
    } else if (searching) {
        start = n / 2;
    }
    uint32_t lastdist = 0;
    while (true) {
        if (!searching && opt.mode == kModeStartOnly)
            break;
        if (searching)
            ++passes;
        solo_pass<B, EMAX>(so, start, !searching, !searching, opt.reverse != 0, placed, nlevels, last_start);
        if (read_status(M.res) != 0)
            return;
        if (!searching)
            break;
        if (placed != n) {
            if (t == 0)
                set_status(M.res, kErrDisconnected, 0);
            return;
        }
        const uint32_t dist = nlevels - 1;
        if (dist == lastdist) {
            ecc = dist;
            searching = false;  // the sorted pass from the same start comes next
            continue;
        }
        if (t == 0)
            s.bcast[0] = so.next_start(opt.outnodes, last_start);
        gsync<B>();
        start = s.bcast[0];
        gsync<B>();
        lastdist = dist;
        if (passes > n) {
            if (t == 0)
                set_status(M.res, kErrCheck, 3);
            return;
        }
    }
    if (opt.mode == kModeStartOnly) {
        if (t == 0) {
            M.res->start = start;
            M.res->passes = passes;
            M.res->ecc = ecc;
            M.res->placed = n;
        }
        return;
    }
    if (placed != n) {
        if (t == 0) {
            set_status(M.res, kErrDisconnected, 1);
            M.res->placed = placed;
        }
        return;
    }
    if (opt.want_bw) {
        // the inverse permutation (four records in flight per thread)
        for (uint32_t pos = t; pos < n; pos += 4 * B) {
            uint2 r[4];
#pragma unroll
            for (int u = 0; u < 4; ++u)
                r[u] = pos + u * B < n ? __ldcg(so.q + pos + u * B) : make_uint2(0u, 0u);
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (pos + u * B < n)
                    inv[rec_node(r[u])] = pos + u * B;
        }
        gsync<B>();
        unsigned long long bw = 0, bw0 = 0, plo = 0, phi = 0;
        for (uint32_t i = t; i < n; i += B) {
            const uint32_t a = ld_ro(M.rp + i), e = ld_ro(M.rp + i + 1);
            if (a == e)
                continue;
            const uint32_t me = __ldcg(inv + i);
            uint32_t mnr = kUnvisited, mxr = 0, c0 = 0, c1 = 0;
            // the row's columns four at a time, then their positions (the
            // loads of a group side by side)
            for (uint32_t k = a; k < e; k += 4) {
                uint32_t c[4];
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    c[u] = k + u < e ? ld_ro(M.ci + k + u) : kUnvisited;
                if (k == a)
                    c0 = c[0];
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (c[u] != kUnvisited) {
                        const uint32_t p = __ldcg(inv + c[u]);
                        mnr = min(mnr, p);
                        mxr = max(mxr, p);
                        c1 = c[u];
                    }
            }
            // computeBandwidth (main.cpp:143-184): max(row - min, max - row)
            const unsigned long long b1 = me >= mnr ? (unsigned long long)(me - mnr) : 0ull;
            const unsigned long long b2 = mxr >= me ? (unsigned long long)(mxr - me) : 0ull;
            bw = max(bw, max(b1, b2));
            plo += b1;
            phi += b2;
            // initial bandwidth: first / last stored column (main.cpp:114-129)
            const unsigned long long i0 = i >= c0 ? i - c0 : 0, i1 = c1 >= i ? c1 - i : 0;
            bw0 = max(bw0, max(i0, i1));
        }
        bw = block_reduce_max<B, unsigned long long>(bw, s.tmp64);
        bw0 = block_reduce_max<B, unsigned long long>(bw0, s.tmp64);
        block_reduce_sum2<B>(plo, phi, s.tmp64);
        if (t == 0) {
            M.res->bandwidth = bw;
            M.res->initial_bw = bw0;
            M.res->profile_lo = plo;
            M.res->profile_hi = phi;
        }
    }
    if (t == 0) {
        M.res->start = start;
        M.res->passes = passes;
        M.res->ecc = ecc;
        M.res->levels = nlevels;
        M.res->placed = placed;
        M.res->t_end = globaltimer();
    }
}

}  // namespace pbrcm
