// resident.cu -- the shared-memory engine: the whole reorder of one small
// matrix (start search, Cuthill-McKee pass, reverse, bandwidth) by one CTA
// that holds the matrix itself in shared memory.
//
// What it computes is what engine.cuh and solo.cuh compute: the serial stable
// order of src/rcm_cpu.cpp:57-104 from the start node of
// src/simple_peripheral.cpp:92-141, and the bandwidth of src/main.cpp:143-184.
// The other engines walk a small matrix's BFS levels at the latency of L2 or
// HBM (a dependent global load or two per level step, ~2.3 us a level on one
// CTA); here row_ptr and col_idx are copied into shared memory once
// (cp.async, all copies in flight at once) and every level step after that
// touches shared memory only.
//
// Layout (dynamic shared memory): two groups' chunk scratch, row_ptr (n + 1
// words), col_idx (nnz), per group a claim word and a queue slot per node
// (2 x 4n bytes; the second group's only when the speculative pass is on),
// and a valence byte per node.
//
// One BFS pass (res_pass) walks the FIFO queue in chunks of at most G parents
// and EW = G x R edges (never across a level boundary).  Per chunk: each
// parent's edges get its index (epar) and row start; edge e claims its column
// with atomicMin(w[c], kClaim | e) -- a node already placed holds 0 and stays
// there -- so after a group barrier a node's word is the claim of the FIRST
// edge in (parent, slot) order that reaches it, which is the (parent, slot)
// that discovers it in the serial loop; the child edges are compacted in
// edge order by warp ballots, marked placed (w = 0), and written to the queue
// in edge order (start-search pass: the FIFO BFS of simple_peripheral.cpp) or
// ranked by (valence, slot) inside each parent's run (the Cuthill-McKee
// pass).  Five group barriers per chunk, six when sorting; three when every
// row has at most 16 entries (res_pass_short: one parent per thread).
//
// Two groups of G threads: with room for two workspaces, from the second
// start-search pass on group 1 runs the sorted pass from the same start while
// group 0 runs the search pass; when the search confirms the eccentricity, the
// sorted pass beside it is the answer (one pass less on the critical path).
// No wait in this kernel spins: the groups meet at CTA barriers only.
#include "engine.cuh"
#include "kernels.h"

namespace pbrcm {

constexpr uint32_t kResClaim = 0x80000000u;  // claim words: kResClaim | chunk edge; 0 = placed

// One group's chunk scratch.
template <int G, int R>
struct alignas(16) ResScratch {
    static constexpr int W = G / 32;
    static constexpr int EW = G * R;
    uint32_t soff[G + 1];  // edge offset of parent j inside the chunk (soff[m] = edges)
    uint32_t prs[G];       // row start of parent j
    uint32_t cs[G], cc[G]; // first child / child count of parent j (cc clear between chunks)
    uint32_t epar[EW];     // parent of each chunk edge
    uint32_t ch_node[EW], ch_deg[EW], ch_par[EW];  // children in edge order (sorted pass)
    uint32_t wq[R][W];     // child edges per (round, warp)
    uint32_t scanbuf[W];
};

template <int G, int R>
struct ResGroup {
    ResScratch<G, R>& s;
    const uint32_t* rp;  // shared memory, n + 1
    const uint32_t* ci;  // shared memory, nnz
    uint32_t* w;         // shared memory, n: claim word per node
    uint32_t* q;         // shared memory, n: the queue
    uint32_t n, nnz;
    DevResult* res;
    const uint8_t* dg;   // shared memory, n: valence per node (rows of at most 255 entries)
};

// One BFS pass from `start` by one group; the queue ends up in g.q[0 ..
// placed).  nlevels: levels of the pass; last_start: first position of its
// last level.
template <int G, int R>
__device__ void res_pass(ResGroup<G, R>& g, uint32_t start, bool sorted, uint32_t& placed, uint32_t& nlevels,
                         uint32_t& last_start)
{
    constexpr uint32_t EW = (uint32_t)(G * R), W = (uint32_t)(G / 32);
    ResScratch<G, R>& s = g.s;
    const uint32_t n = g.n;
    const uint32_t t = gtid<G>(), lane = t & 31u, wi = t >> 5;
    for (uint32_t i = t; i < n; i += G)
        g.w[i] = kUnvisited;
    s.cc[t] = 0;
    gsync<G>();
    if (t == 0) {
        g.q[0] = start;
        g.w[start] = 0;
    }
    gsync<G>();
    uint32_t head = 0, tail = 1, lvl_end = 1, L = 0, lstart = 0;
    while (head < tail) {
        if (head == lvl_end) {
            L += 1;
            lstart = head;
            lvl_end = tail;
        }
        // form: the next parents of this level, at most G of them and EW edges
        uint32_t a = 0, deg = 0;
        const bool have = head + t < lvl_end;
        if (have) {
            const uint32_t p = g.q[head + t];
            a = g.rp[p];
            deg = g.rp[p + 1] - a;
        }
        uint32_t total;
        const uint32_t excl = block_scan1<G>(deg, total, s.scanbuf);
        const uint32_t incl = excl + deg;
        // incl grows with t, so the parents that fit are a prefix
        const bool fits = have && incl <= EW;
        if (fits) {
            s.soff[t] = excl;
            s.soff[t + 1] = incl;  // the next thread writes the same value, or t is the last parent
            s.prs[t] = a;
            for (uint32_t k = 0; k < deg; ++k)
                s.epar[excl + k] = t;
        }
        const uint32_t m = (uint32_t)gsync_count<G>(fits);
        if (m == 0) {  // a row longer than a chunk: the host admits none
            if (t == 0)
                set_status(g.res, kErrCheck, 620);
            break;
        }
        const uint32_t Ec = s.soff[m];
        // claim: every chunk edge e bids kResClaim | e for its column
        uint32_t c[R], dg[R], jj[R], pos[R];
        bool first[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const uint32_t e = t + (uint32_t)G * r;
            c[r] = kUnvisited;
            dg[r] = 0;
            jj[r] = 0;
            first[r] = false;
            if (e < Ec) {
                const uint32_t j = s.epar[e];
                const uint32_t k = e - s.soff[j];
                const uint32_t idx = s.prs[j] + k;
                jj[r] = j;
                first[r] = k == 0;
                if (PB_CHECK(g.res, idx < g.nnz, 621))
                    c[r] = g.ci[idx];
            }
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (c[r] != kUnvisited && PB_CHECK(g.res, c[r] < n, 622)) {
                const uint32_t e = t + (uint32_t)G * r;
                if (atomicMin(&g.w[c[r]], kResClaim | e) == 0u)
                    c[r] = kUnvisited;  // placed before this chunk
                else if (sorted)
                    dg[r] = g.rp[c[r] + 1] - g.rp[c[r]];
            } else {
                c[r] = kUnvisited;
            }
        }
        gsync<G>();
        // the child edges: those whose bid stands (the first edge to each
        // new node), compacted in edge order: a ballot per (round, warp)
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const uint32_t e = t + (uint32_t)G * r;
            const bool win = c[r] != kUnvisited && g.w[c[r]] == (kResClaim | e);
            if (!win)
                c[r] = kUnvisited;
            const uint32_t bal = __ballot_sync(kFull, win);
            pos[r] = __popc(bal & ((1u << lane) - 1u));
            if (lane == 0)
                s.wq[r][wi] = __popc(bal);
        }
        gsync<G>();
        uint32_t Q = 0;
#pragma unroll
        for (int r = 0; r < R; ++r) {
#pragma unroll
            for (uint32_t i = 0; i < W; ++i) {
                const uint32_t n_ = s.wq[r][i];
                pos[r] += i < wi ? n_ : 0u;
                Q += n_;
            }
            if (r + 1 < R)
                pos[r + 1] += Q;  // the child edges of the rounds before
        }
        if (!sorted) {
            // row order: the queue takes the children as they are
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (c[r] != kUnvisited && PB_CHECK(g.res, tail + pos[r] < n, 623)) {
                    g.q[tail + pos[r]] = c[r];
                    g.w[c[r]] = 0;
                }
        } else {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const uint32_t e = t + (uint32_t)G * r;
                if (e < Ec) {
                    if (first[r])
                        s.cs[jj[r]] = pos[r];
                    if (c[r] != kUnvisited) {
                        s.ch_node[pos[r]] = c[r];
                        s.ch_deg[pos[r]] = dg[r];
                        s.ch_par[pos[r]] = jj[r];
                        atomicAdd(&s.cc[jj[r]], 1u);
                        g.w[c[r]] = 0;
                    }
                }
            }
            gsync<G>();
            // each child's rank inside its parent's run: by valence, then slot
            for (uint32_t x = t; x < Q; x += G) {
                const uint32_t jp = s.ch_par[x];
                const uint32_t st = s.cs[jp], len = s.cc[jp];
                uint32_t rank = x - st;
                if (len > 1) {
                    const uint32_t dx = s.ch_deg[x];
                    rank = 0;
                    for (uint32_t y = st; y < st + len; ++y) {
                        const uint32_t dy = s.ch_deg[y];
                        rank += (dy < dx) || (dy == dx && y < x);
                    }
                }
                if (PB_CHECK(g.res, tail + st + rank < n, 624))
                    g.q[tail + st + rank] = s.ch_node[x];
            }
        }
        // the queue entries are in before the next chunk reads them (and
        // every rank has read the child counts before they are cleared)
        gsync<G>();
        if (sorted && t < m)
            s.cc[t] = 0;
        head += m;
        tail += Q;
        if (tail > n) {  // cannot happen on a valid run
            if (t == 0)
                set_status(g.res, kErrCheck, 625);
            break;
        }
    }
    placed = tail;
    nlevels = L + 1;
    last_start = lstart;
}

// Matrices whose rows all have at most ROW entries (6, 8 or 16): the same pass
// with one parent per thread and the row in registers.  Thread j loads its
// parent's whole row at once (the loop over slots is unrolled, so every load
// of the row is in flight together) and slot k bids kResClaim | j << 5 | k
// (the (parent, slot) order of the chunk), so no edge needs its parent looked
// up; the children's valences (a byte table built with the CSR check) are
// loaded beside the bids.  After the barrier
// the thread tests its own bids into a bit mask, one scan gives each parent
// its first queue position, and the thread writes its children in slot order
// or ranked by (valence, slot) among themselves -- register arithmetic.
// Three group barriers per chunk.
// Shared-memory accesses in the shared state space (the engine's arrays are
// carved out of one dynamic shared allocation; a generic access would pay
// the generic-to-shared path on every load and atomic).
__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ uint32_t lds(uint32_t a)
{
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(a) : "memory");
    return v;
}
__device__ __forceinline__ uint32_t ldsb(uint32_t a)
{
    uint32_t v;
    asm volatile("ld.shared.u8 %0, [%1];" : "=r"(v) : "r"(a) : "memory");
    return v;
}
__device__ __forceinline__ void sts(uint32_t a, uint32_t v)
{
    asm volatile("st.shared.u32 [%0], %1;" ::"r"(a), "r"(v) : "memory");
}
__device__ __forceinline__ void reds_min(uint32_t a, uint32_t v)
{
    asm volatile("red.shared.min.u32 [%0], %1;" ::"r"(a), "r"(v) : "memory");
}

// Exclusive scan over a group of values below 2^BITS: the warp part from
// BITS independent ballots (bit-sliced counts) instead of five dependent
// shuffles; same buffer rule as block_scan1 (read after its barrier, written
// again only after another group barrier).
template <int B, int BITS>
__device__ __forceinline__ uint32_t block_scan_bits(uint32_t v, uint32_t& total, uint32_t* buf)
{
    constexpr uint32_t W = (uint32_t)(B / 32);
    const uint32_t lane = threadIdx.x & 31u, w = gtid<B>() >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    uint32_t excl = 0, wsum = 0;
#pragma unroll
    for (int b = 0; b < BITS; ++b) {
        const uint32_t bal = __ballot_sync(kFull, (v >> b) & 1u);
        excl += (uint32_t)__popc(bal & lt) << b;
        wsum += (uint32_t)__popc(bal) << b;
    }
    if (lane == 0)
        buf[w] = wsum;
    gsync<B>();
    uint32_t before = 0, all = 0;
#pragma unroll
    for (uint32_t i = 0; i < W; ++i) {
        const uint32_t x = buf[i];
        before += i < w ? x : 0u;
        all += x;
    }
    total = all;
    return before + excl;
}

// bits that hold 0..x
__host__ __device__ constexpr int res_bits(int x) { return x < 8 ? 3 : x < 16 ? 4 : x < 32 ? 5 : 6; }

template <int G, int R, int ROW>
__device__ __noinline__ void res_pass_short(ResGroup<G, R>& g, uint32_t start, bool sorted, uint32_t& placed, uint32_t& nlevels,
                               uint32_t& last_start)
{
    static_assert(ROW <= 32 && G <= 1024, "slot bits and parent bits of a bid");
    ResScratch<G, R>& s = g.s;
    const uint32_t n = g.n;
    const uint32_t t = gtid<G>();
    for (uint32_t i = t; i < n; i += G)
        g.w[i] = kUnvisited;
    gsync<G>();
    if (t == 0) {
        g.q[0] = start;
        g.w[start] = 0;
    }
    gsync<G>();
    uint32_t head = 0, tail = 1, lvl_end = 1, L = 0, lstart = 0;
    const uint32_t key0 = kResClaim | (t << 5);
    const uint32_t qa = saddr(g.q), wa = saddr(g.w), rpa = saddr(g.rp), cia = saddr(g.ci), dga = saddr(g.dg);
    while (head < tail) {
        if (head == lvl_end) {
            L += 1;
            lstart = head;
            lvl_end = tail;
        }
        const uint32_t m = min((uint32_t)G, lvl_end - head);
        uint32_t a = 0, deg = 0;
        if (t < m) {
            const uint32_t p = lds(qa + 4 * (head + t));
            a = lds(rpa + 4 * p);
            deg = lds(rpa + 4 * (p + 1)) - a;
            if (!PB_CHECK(g.res, deg <= (uint32_t)ROW, 626))
                deg = 0;
        }
        // a warp without parents skips the row work (its threads still meet
        // every barrier)
        const bool wbusy = (t & ~31u) < m;
        uint32_t c[ROW], d[ROW];
        if (wbusy) {
#pragma unroll
            for (int k = 0; k < ROW; ++k)
                c[k] = (uint32_t)k < deg ? lds(cia + 4 * (a + k)) : kUnvisited;
#pragma unroll
            for (int k = 0; k < ROW; ++k) {
                d[k] = 0;
                if (c[k] != kUnvisited && PB_CHECK(g.res, c[k] < n, 627)) {
                    reds_min(wa + 4 * c[k], key0 | (uint32_t)k);
                    if (sorted)
                        d[k] = ldsb(dga + c[k]);
                } else {
                    c[k] = kUnvisited;
                }
            }
        }
        gsync<G>();
        // this parent's child slots: the bids that stand
        uint32_t win = 0;
        if (wbusy) {
#pragma unroll
            for (int k = 0; k < ROW; ++k)
                if (c[k] != kUnvisited && lds(wa + 4 * c[k]) == (key0 | (uint32_t)k))
                    win |= 1u << k;
        }
        uint32_t Q;
        const uint32_t base = tail + block_scan_bits<G, res_bits(ROW)>((uint32_t)__popc(win), Q, s.scanbuf);
        // (every bid was tested before the scan's barrier: marking is safe)
        if (win != 0) {
            // children of one valence keep slot order: no ranking
            bool mixed = false;
            if (sorted) {
                uint32_t dmin = kUnvisited, dmax = 0;
#pragma unroll
                for (int k = 0; k < ROW; ++k)
                    if ((win >> k) & 1u) {
                        dmin = min(dmin, d[k]);
                        dmax = max(dmax, d[k]);
                    }
                mixed = dmin != dmax;
            }
#pragma unroll
            for (int k = 0; k < ROW; ++k) {
                if (!((win >> k) & 1u))
                    continue;
                uint32_t r = (uint32_t)__popc(win & ((1u << k) - 1u));
                if (mixed) {
                    r = 0;
#pragma unroll
                    for (int k2 = 0; k2 < ROW; ++k2)
                        r += ((win >> k2) & 1u) && (d[k2] < d[k] || (d[k2] == d[k] && k2 < k));
                }
                if (PB_CHECK(g.res, base + r < n, 628))
                    sts(qa + 4 * (base + r), c[k]);
                sts(wa + 4 * c[k], 0u);
            }
        }
        // the queue entries are in before the next chunk reads them
        gsync<G>();
        head += m;
        tail += Q;
        if (tail > n) {  // cannot happen on a valid run
            if (t == 0)
                set_status(g.res, kErrCheck, 629);
            break;
        }
    }
    placed = tail;
    nlevels = L + 1;
    last_start = lstart;
}

// CTA-wide reductions (both groups; barrier 0).
__device__ __forceinline__ unsigned long long cta_max(unsigned long long v, unsigned long long* tmp)
{
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long y = __shfl_xor_sync(kFull, v, o);
        v = v > y ? v : y;
    }
    if (lane == 0)
        tmp[w] = v;
    __syncthreads();
    unsigned long long r = 0;
    for (uint32_t i = 0; i < nw; ++i)
        r = r > tmp[i] ? r : tmp[i];
    __syncthreads();
    return r;
}

__device__ __forceinline__ unsigned long long cta_sum(unsigned long long v, unsigned long long* tmp)
{
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(kFull, v, o);
    if (lane == 0)
        tmp[w] = v;
    __syncthreads();
    unsigned long long r = 0;
    for (uint32_t i = 0; i < nw; ++i)
        r += tmp[i];
    __syncthreads();
    return r;
}

__device__ __forceinline__ void cp_async4(uint32_t* dst, const uint32_t* src)
{
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    const size_t g = __cvta_generic_to_global(src);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(g) : "memory");
}

// Bytes of dynamic shared memory for n nodes and nnz entries, one or two
// workspaces.
template <int G, int R>
PBRCM_HD inline size_t res_smem(uint32_t n, uint32_t nnz, bool spec)
{
    return 2 * sizeof(ResScratch<G, R>) + 4 * ((size_t)n + 1 + (size_t)nnz) + (spec ? 16 : 8) * (size_t)n +
           (((size_t)n + 3) & ~(size_t)3);
}

// One matrix, one CTA of two groups.  spec: room for the second workspace.
template <int G, int R>
__global__ void __launch_bounds__(2 * G, 1)
    k_reorder_resident(const uint32_t* __restrict__ g_rp, const uint32_t* __restrict__ g_ci, uint32_t n, uint32_t nnz,
                       uint32_t* perm, DevResult* res, Options opt, uint32_t spec)
{
    constexpr uint32_t EW = (uint32_t)(G * R);
    static_assert(EW == kResidentMaxRow, "every shape chunks kResidentMaxRow edges");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ unsigned long long red[2 * G / 32];
    __shared__ uint32_t ctl[8];
    using S = ResScratch<G, R>;
    S* scr = reinterpret_cast<S*>(smem_raw);
    uint32_t* rp = reinterpret_cast<uint32_t*>(smem_raw + 2 * sizeof(S));
    uint32_t* ci = rp + (n + 1);
    uint32_t* w0 = ci + nnz;
    uint32_t* q0 = w0 + n;
    uint32_t* w1 = spec ? q0 + n : w0;
    uint32_t* q1 = spec ? w1 + n : q0;
    uint8_t* dg8 = reinterpret_cast<uint8_t*>((spec ? q1 : q0) + n);
    const uint32_t tid = threadIdx.x, nthr = blockDim.x;
    const uint32_t grp = tid / G;
    if (tid == 0)
        res->t_begin = globaltimer();
    // the matrix into shared memory: every copy in flight at once
    for (uint32_t i = tid; i <= n; i += nthr)
        cp_async4(rp + i, g_rp + i);
    for (uint32_t k = tid; k < nnz; k += nthr)
        cp_async4(ci + k, g_ci + k);
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    // the checks of k_validate, and the largest valence
    bool bad = false;
    uint32_t mx = 0;
    for (uint32_t i = tid; i < n; i += nthr) {
        const uint32_t a = rp[i], b = rp[i + 1];
        if (b < a || b > nnz) {
            bad = true;
        } else {
            mx = max(mx, b - a);
            dg8[i] = (uint8_t)min(b - a, 255u);
        }
    }
    if (tid == 0 && (rp[0] != 0 || rp[n] != nnz))
        bad = true;
    for (uint32_t k = tid; k < nnz; k += nthr)
        if (ci[k] >= n)
            bad = true;
    const int any_bad = __syncthreads_or(bad);
    const unsigned long long maxdeg = cta_max(mx, red);
    if (any_bad) {
        if (tid == 0)
            set_status(res, kErrArg, 200);
        return;
    }
    if (tid == 0)
        res->maxdeg = (uint32_t)maxdeg;
    if (maxdeg > EW) {
        // a row longer than a chunk: the host reruns the matrix on the team
        if (tid == 0)
            set_status(res, kNeedTeam, 0);
        return;
    }
    uint32_t start = opt.start;
    if (start != kUnvisited && start >= n) {
        if (tid == 0)
            set_status(res, kErrArg, 2);
        return;
    }
    uint32_t passes = 0, ecc = 0;
    bool searching = start == kUnvisited && n > 1;
    if (n == 1) {
        passes = start == kUnvisited ? 1 : 0;
        start = 0;
    } else if (searching) {
        start = n / 2;
    }
    ResGroup<G, R> gr{scr[grp], rp, ci, grp ? w1 : w0, grp ? q1 : q0, n, nnz, res, dg8};
    const uint32_t sorter = spec ? 1u : 0u;  // the group that runs sorted passes
    // rows of at most 6, 8 or 16 entries: the one-parent-a-thread pass
    const uint32_t row_class = maxdeg <= 6 ? 6u : maxdeg <= 8 ? 8u : maxdeg <= 16 ? 16u : 0u;
    uint32_t lastdist = 0, sorted_from = kUnvisited, s_placed = 0, s_levels = 0;
    // rounds: group 0 runs a start-search pass while (with spec) group 1
    // runs the sorted pass from the same start, from the second search on
    while (true) {
        if (!searching && (opt.mode == kModeStartOnly || sorted_from == start))
            break;
        const bool run_search = searching;
        // (without the second workspace a sorted pass only comes after the search)
        const bool run_sort = opt.mode != kModeStartOnly && (!searching || (spec && passes >= 1));
        if (run_search && grp == 0) {
            uint32_t pl, nl, ls;
            if (row_class == 6)
                res_pass_short<G, R, 6>(gr, start, false, pl, nl, ls);
            else if (row_class == 8)
                res_pass_short<G, R, 8>(gr, start, false, pl, nl, ls);
            else if (row_class == 16)
                res_pass_short<G, R, 16>(gr, start, false, pl, nl, ls);
            else
                res_pass<G, R>(gr, start, false, pl, nl, ls);
            if (tid == 0) {
                ctl[0] = pl;
                ctl[1] = nl;
                ctl[2] = ls;
            }
        }
        if (run_sort && grp == sorter) {
            uint32_t pl, nl, ls;
            if (row_class == 6)
                res_pass_short<G, R, 6>(gr, start, true, pl, nl, ls);
            else if (row_class == 8)
                res_pass_short<G, R, 8>(gr, start, true, pl, nl, ls);
            else if (row_class == 16)
                res_pass_short<G, R, 16>(gr, start, true, pl, nl, ls);
            else
                res_pass<G, R>(gr, start, true, pl, nl, ls);
            if (gtid<G>() == 0) {
                ctl[3] = pl;
                ctl[4] = nl;
            }
        }
        __syncthreads();
        if (read_status(res) != 0)
            return;
        if (run_sort) {
            sorted_from = start;
            s_placed = ctl[3];
            s_levels = ctl[4];
        }
        if (run_search) {
            ++passes;
            if (ctl[0] != n) {
                if (tid == 0)
                    set_status(res, kErrDisconnected, 0);
                return;
            }
            const uint32_t dist = ctl[1] - 1;
            if (dist == lastdist) {
                ecc = dist;
                searching = false;  // the sorted pass from this start is the answer
            } else {
                // next_peripheral_start: among the last min(outnodes, n-1)
                // positions, those on the last level; the last of minimal
                // valence (simple_peripheral.cpp:118-127)
                if (tid == 0) {
                    uint32_t lo = n - min(opt.outnodes, n - 1);
                    lo = max(lo, max(ctl[2], 1u));
                    uint32_t best = 0, bestdeg = kUnvisited;
                    for (uint32_t p = lo; p < n; ++p) {
                        const uint32_t v = q0[p];
                        const uint32_t d = rp[v + 1] - rp[v];
                        if (d <= bestdeg) {
                            bestdeg = d;
                            best = v;
                        }
                    }
                    ctl[5] = best;
                }
                __syncthreads();
                start = ctl[5];
                lastdist = dist;
                if (passes > n) {
                    if (tid == 0)
                        set_status(res, kErrCheck, 3);
                    return;
                }
            }
        }
        __syncthreads();  // ctl is read by all before the next round writes it
    }
    if (opt.mode == kModeStartOnly) {
        if (tid == 0) {
            res->start = start;
            res->passes = passes;
            res->ecc = ecc;
            res->placed = n;
            res->t_end = globaltimer();
        }
        return;
    }
    if (s_placed != n) {
        if (tid == 0) {
            set_status(res, kErrDisconnected, 1);
            res->placed = s_placed;
        }
        return;
    }
    const uint32_t* qs = sorter ? q1 : q0;
    const bool reverse = opt.reverse != 0;
    for (uint32_t p = tid; p < n; p += nthr)
        perm[reverse ? n - 1 - p : p] = qs[p];
    if (opt.want_bw) {
        // inverse permutation in group 0's claim words (free now)
        uint32_t* inv = w0;
        for (uint32_t p = tid; p < n; p += nthr)
            inv[qs[p]] = p;
        __syncthreads();
        unsigned long long bw = 0, bw0 = 0, plo = 0, phi = 0;
        for (uint32_t i = tid; i < n; i += nthr) {
            const uint32_t a = rp[i], e = rp[i + 1];
            if (a == e)
                continue;
            const uint32_t me = inv[i];
            uint32_t mnr = kUnvisited, mxr = 0;
            for (uint32_t k = a; k < e; ++k) {
                const uint32_t p = inv[ci[k]];
                mnr = min(mnr, p);
                mxr = max(mxr, p);
            }
            // computeBandwidth (main.cpp:143-184): max(row - min, max - row)
            const unsigned long long b1 = me >= mnr ? (unsigned long long)(me - mnr) : 0ull;
            const unsigned long long b2 = mxr >= me ? (unsigned long long)(mxr - me) : 0ull;
            bw = max(bw, max(b1, b2));
            plo += b1;
            phi += b2;
            // initial bandwidth: first / last stored column (main.cpp:114-129)
            const uint32_t c0 = ci[a], c1 = ci[e - 1];
            const unsigned long long i0 = i >= c0 ? i - c0 : 0, i1 = c1 >= i ? c1 - i : 0;
            bw0 = max(bw0, max(i0, i1));
        }
        bw = cta_max(bw, red);
        bw0 = cta_max(bw0, red);
        plo = cta_sum(plo, red);
        phi = cta_sum(phi, red);
        if (tid == 0) {
            res->bandwidth = bw;
            res->initial_bw = bw0;
            res->profile_lo = plo;
            res->profile_hi = phi;
        }
    }
    if (tid == 0) {
        res->start = start;
        res->passes = passes;
        res->ecc = ecc;
        res->levels = s_levels;
        res->placed = s_placed;
        res->t_end = globaltimer();
    }
}

namespace {
template <int G, int R>
struct ResVariant {
    static size_t smem(uint32_t n, uint32_t nnz, bool spec) { return res_smem<G, R>(n, nnz, spec); }
    static cudaError_t launch(const uint32_t* rp, const uint32_t* ci, uint32_t n, uint32_t nnz, uint32_t* perm,
                              DevResult* res, const Options& opt, int max_smem, cudaStream_t st)
    {
        static cudaError_t once = cudaFuncSetAttribute(k_reorder_resident<G, R>,
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem);
        if (once != cudaSuccess)
            return once;
        const bool spec = smem(n, nnz, true) <= (size_t)max_smem;
        const size_t bytes = smem(n, nnz, spec);
        if (bytes > (size_t)max_smem)
            return cudaErrorInvalidValue;
        k_reorder_resident<G, R><<<1, 2 * G, bytes, st>>>(rp, ci, n, nnz, perm, res, opt, spec ? 1u : 0u);
        return cudaGetLastError();
    }
};
}  // namespace

// Group sizes of the shared-memory engine: 32, 64, 128 or 256 threads (two
// groups per CTA), chunks of 512 edges in every shape.
#define PBRCM_RES_DISPATCH(g, CALL)            \
    switch (g) {                               \
    case 32: return ResVariant<32, 16>::CALL;  \
    case 64: return ResVariant<64, 8>::CALL;   \
    case 128: return ResVariant<128, 4>::CALL; \
    case 256: return ResVariant<256, 2>::CALL; \
    default: break;                            \
    }

bool resident_group_ok(int g) { return g == 32 || g == 64 || g == 128 || g == 256; }

size_t resident_smem(int g, uint32_t n, uint32_t nnz, bool spec)
{
    PBRCM_RES_DISPATCH(g, smem(n, nnz, spec));
    return ~(size_t)0;
}

cudaError_t launch_resident(int g, const uint32_t* rp, const uint32_t* ci, uint32_t n, uint32_t nnz, uint32_t* perm,
                            DevResult* res, const Options& opt, int max_smem, cudaStream_t st)
{
    PBRCM_RES_DISPATCH(g, launch(rp, ci, n, nnz, perm, res, opt, max_smem, st));
    return cudaErrorInvalidValue;
}

}  // namespace pbrcm
