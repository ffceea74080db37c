// connect.cu -- the connectivity repair of the reference loader, on the device.
//
// prepareRCM (include/Graph.h:160-263) walks the matrix breadth-first from
// its first non-empty row `minn`; while nodes are left over it links the
// smallest unvisited node i to the largest visited node below i (or, with
// none below, to the smallest visited node above i), then walks on from i,
// and finally rebuilds the CSR sorted by (row, col) with both directions of
// every link added.  Every node below the smallest unvisited one has been
// visited by then, so the links depend on the components alone:
//   - a component whose smallest node m > 0 is not minn's gets (m - 1, m);
//   - the component {0} (row 0 empty, so minn > 0) gets (0, minn).
// An empty row is a component of its own.  (The reference never finishes on
// an empty row, which it queues without marking; the host loader of this
// library and this pass link it like any other component.)
//
// Passes (all HBM-bound, one thread per 8 consecutive entries or per row):
//   1. k_cc_init: parent[v] = min(v, first column of row v) (rows are sorted,
//      so that is the smallest neighbour) and minn;
//   2. k_cc_hook: union-find over the entries (u, v), u < v, hooking the
//      larger root under the smaller with atomicCAS and halving paths on the
//      way up -- the minimum-label form of the ECL-CC algorithm (Jaiganesh and
//      Burtscher, HPDC 2018), so that each component's root is its smallest
//      node and "m is a component minimum" is parent[m] == m afterwards.  The
//      same pass checks each entry: column in range, row sorted, and the
//      transposed entry present (the repair is defined on symmetric patterns);
//   3. k_connect_rowlen: row length plus the links of the row (at most two),
//      scanned into row_ptr_out (the three scan kernels of permute.cu);
//   4. k_connect_copy: each entry shifted to its place in the output row, then
//      each link inserted at its sorted position.
#include <algorithm>
#include <cstdint>

#include <cuda_runtime.h>

#include "kernels.h"
#include "types.h"

namespace pbrcm {

namespace {

constexpr int kEntriesPerThread = 8;
constexpr int kThreads = 256;

// counters[0] minn, [1] links, [2] check flags
constexpr uint32_t kFlagRange = 1, kFlagUnsorted = 2, kFlagAsym = 4, kFlagDepth = 8;

// Row v's entry range, clamped into [0, nnz] (the CSR check runs beside these
// kernels on the same stream; a bad row_ptr must not send them out of bounds).
__device__ __forceinline__ void row_range(const uint32_t* __restrict__ rp, uint32_t v, uint32_t nnz, uint32_t& b,
                                          uint32_t& e)
{
    b = min(rp[v], nnz);
    e = min(max(rp[v + 1], b), nnz);
}

// The row containing entry k: the largest v < n with rp[v] <= k.
__device__ __forceinline__ uint32_t row_of(const uint32_t* __restrict__ rp, uint32_t n, uint32_t k)
{
    uint32_t lo = 0, hi = n - 1;
    while (lo < hi) {
        const uint32_t mid = lo + (hi - lo + 1) / 2;
        if (rp[mid] <= k)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// First index in ci[b, e) whose column is >= x (a sorted row).
__device__ __forceinline__ uint32_t lower_bound(const uint32_t* __restrict__ ci, uint32_t b, uint32_t e, uint32_t x)
{
    while (b < e) {
        const uint32_t mid = b + (e - b) / 2;
        if (ci[mid] < x)
            b = mid + 1;
        else
            e = mid;
    }
    return b;
}

// Root of v.  Parents only ever point to smaller nodes of the same component,
// so x strictly decreases and the climb ends within v steps; each visited
// node is re-pointed to its grandparent (path halving).  Parent words are
// read through L2 (other threads hook roots concurrently); a halving store
// only ever replaces a non-root's parent by one of its ancestors, and roots
// change only by the atomicCAS in cc_unite, so no hook is lost.
__device__ __forceinline__ uint32_t cc_root(uint32_t* parent, uint32_t v)
{
    uint32_t x = v;
    uint32_t p = __ldcg(parent + x);
    while (p != x) {
        const uint32_t g = __ldcg(parent + p);
        if (g != p)
            parent[x] = g;
        x = g;
        p = __ldcg(parent + x);
    }
    return x;
}

// Joins the components of a and b: the larger root is hooked under the
// smaller.  A failed atomicCAS means that root was hooked meanwhile; the
// union climbs on from its new parent.  Every retry follows a successful hook
// by another thread, and there are at most n - 1 hooks, so the loop is
// bounded by the size of the graph; the explicit limit only guards that.
__device__ __forceinline__ bool cc_unite(uint32_t* parent, uint32_t a, uint32_t b, uint32_t limit)
{
    uint32_t ra = cc_root(parent, a), rb = cc_root(parent, b);
    for (uint32_t it = 0; ra != rb; ++it) {
        if (it > limit)
            return false;
        if (ra < rb) {
            const uint32_t t = ra;
            ra = rb;
            rb = t;
        }
        const uint32_t old = atomicCAS(parent + ra, ra, rb);
        if (old == ra)
            return true;
        ra = cc_root(parent, old);
        rb = cc_root(parent, rb);
    }
    return true;
}

__device__ __forceinline__ bool is_link_min(const uint32_t* __restrict__ parent, uint32_t n, uint32_t minn, uint32_t x)
{
    return x < n && minn < n && x != minn && __ldg(parent + x) == x;
}

// The links of row v in ascending column order; returns their count (0-2).
__device__ __forceinline__ int row_links(const uint32_t* __restrict__ parent, uint32_t n, uint32_t minn, uint32_t v,
                                         uint32_t e[2])
{
    uint32_t c[3];
    int k = 0;
    if (v == minn && minn > 0 && is_link_min(parent, n, minn, 0))
        c[k++] = 0;  // row minn takes (0, minn)
    if (is_link_min(parent, n, minn, v))
        c[k++] = v > 0 ? v - 1 : minn;  // v is a component's smallest node
    if (v + 1 < n && is_link_min(parent, n, minn, v + 1))
        c[k++] = v + 1;  // v + 1 is one, linked to v
    // at most two of the three hold (v == minn excludes the second); sort
    if (k == 2 && c[0] > c[1]) {
        const uint32_t t = c[0];
        c[0] = c[1];
        c[1] = t;
    }
    e[0] = k > 0 ? c[0] : 0;
    e[1] = k > 1 ? c[1] : 0;
    return k > 2 ? 2 : k;
}

__global__ void __launch_bounds__(kThreads) k_cc_init(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                                                      uint32_t n, uint32_t nnz, uint32_t* __restrict__ parent,
                                                      uint32_t* counters)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint32_t first = kFull;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t v = (uint32_t)i;
        uint32_t b, e;
        row_range(rp, v, nnz, b, e);
        uint32_t p = v;
        if (e > b) {
            first = min(first, v);
            const uint32_t c = ci[b];
            if (c < p)
                p = c;
        }
        parent[v] = p;
    }
    first = __reduce_min_sync(0xFFFFFFFFu, first);
    if ((threadIdx.x & 31) == 0 && first != kFull)
        atomicMin(counters, first);
}

__global__ void __launch_bounds__(kThreads) k_cc_hook(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                                                      uint32_t n, uint32_t nnz, uint32_t* parent, uint32_t* counters)
{
    const uint64_t chunks = ((uint64_t)nnz + kEntriesPerThread - 1) / kEntriesPerThread;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint32_t flags = 0;
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < chunks; t += stride) {
        const uint32_t k0 = (uint32_t)(t * kEntriesPerThread);
        const uint32_t k1 = (uint32_t)min((uint64_t)k0 + kEntriesPerThread, (uint64_t)nnz);
        uint32_t v = row_of(rp, n, k0);
        uint32_t b, e;
        row_range(rp, v, nnz, b, e);
        uint32_t prev = k0 > b && k0 - 1 < e ? ci[k0 - 1] : 0u;
        for (uint32_t k = k0; k < k1; ++k) {
            while (k >= e && v + 1 < n) {  // next non-empty row
                ++v;
                row_range(rp, v, nnz, b, e);
            }
            if (k < b || k >= e) {  // only a bad row_ptr leaves k outside every row
                flags |= kFlagRange;
                break;
            }
            const uint32_t u = ci[k];
            if (u >= n) {
                flags |= kFlagRange;
                continue;
            }
            if (k > b && prev > u)
                flags |= kFlagUnsorted;
            prev = u;
            if (u == v)
                continue;
            uint32_t ub, ue;
            row_range(rp, u, nnz, ub, ue);
            const uint32_t at = lower_bound(ci, ub, ue, v);
            if (at >= ue || ci[at] != v)
                flags |= kFlagAsym;
            if (u < v && !cc_unite(parent, u, v, n))
                flags |= kFlagDepth;
        }
    }
    flags = __reduce_or_sync(0xFFFFFFFFu, flags);
    if ((threadIdx.x & 31) == 0 && flags)
        atomicOr(counters + 2, flags);
}

// out_rp[v + 1] = length of row v + its links; counters[1] = number of links.
__global__ void __launch_bounds__(kThreads) k_connect_rowlen(const uint32_t* __restrict__ rp, uint32_t n, uint32_t nnz,
                                                             const uint32_t* __restrict__ parent,
                                                             uint32_t* counters, uint32_t* __restrict__ out_rp)
{
    const uint32_t minn = __ldcg(counters);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint32_t links = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t v = (uint32_t)i;
        uint32_t b, e, lk[2];
        row_range(rp, v, nnz, b, e);
        out_rp[v + 1] = (e - b) + (uint32_t)row_links(parent, n, minn, v, lk);
        links += is_link_min(parent, n, minn, v) ? 1u : 0u;
        if (v == 0)
            out_rp[0] = 0;
    }
    links = __reduce_add_sync(0xFFFFFFFFu, links);
    if ((threadIdx.x & 31) == 0 && links)
        atomicAdd(counters + 1, links);
}

// Entry k of row v goes to out_rp[v] + (k - rp[v]) + (links of v below its
// column); a link e_j goes to out_rp[v] + (entries of v below e_j) + j.
// Links never coincide with an entry (they join different components).
// Writes past `cap` are dropped (the host reports the size needed).
__global__ void __launch_bounds__(kThreads) k_connect_copy(const uint32_t* __restrict__ rp,
                                                           const uint32_t* __restrict__ ci, uint32_t n, uint32_t nnz,
                                                           const uint32_t* __restrict__ parent,
                                                           const uint32_t* counters, const uint32_t* __restrict__ out_rp,
                                                           uint32_t* __restrict__ out_ci, uint64_t cap)
{
    const uint32_t minn = __ldcg(counters);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t chunks = ((uint64_t)nnz + kEntriesPerThread - 1) / kEntriesPerThread;
    for (uint64_t t = tid; t < chunks; t += stride) {
        const uint32_t k0 = (uint32_t)(t * kEntriesPerThread);
        const uint32_t k1 = (uint32_t)min((uint64_t)k0 + kEntriesPerThread, (uint64_t)nnz);
        uint32_t v = row_of(rp, n, k0);
        uint32_t b, e, lk[2];
        row_range(rp, v, nnz, b, e);
        int nl = out_rp[v + 1] - out_rp[v] != e - b ? row_links(parent, n, minn, v, lk) : 0;
        uint64_t base = (uint64_t)out_rp[v] - b;
        for (uint32_t k = k0; k < k1; ++k) {
            while (k >= e && v + 1 < n) {
                ++v;
                row_range(rp, v, nnz, b, e);
                nl = out_rp[v + 1] - out_rp[v] != e - b ? row_links(parent, n, minn, v, lk) : 0;
                base = (uint64_t)out_rp[v] - b;
            }
            if (k < b || k >= e)
                break;
            const uint32_t c = ci[k];
            const uint64_t at = base + k + (nl > 0 && lk[0] < c ? 1 : 0) + (nl > 1 && lk[1] < c ? 1 : 0);
            if (at < cap)
                out_ci[at] = c;
        }
    }
    for (uint64_t i = tid; i < n; i += stride) {
        const uint32_t v = (uint32_t)i;
        uint32_t lk[2];
        const int nl = row_links(parent, n, minn, v, lk);
        if (nl == 0)
            continue;
        uint32_t b, e;
        row_range(rp, v, nnz, b, e);
        for (int j = 0; j < nl; ++j) {
            const uint64_t at = (uint64_t)out_rp[v] + (lower_bound(ci, b, e, lk[j]) - b) + j;
            if (at < cap)
                out_ci[at] = lk[j];
        }
    }
}

}  // namespace

cudaError_t launch_connect(const uint32_t* rp, const uint32_t* ci, uint32_t n, uint32_t nnz, uint32_t* out_rp,
                           uint32_t* out_ci, uint64_t cap, uint32_t* parent, uint32_t* partials, uint32_t* counters,
                           int sms, cudaStream_t st)
{
    const int rows_blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)n + kThreads - 1) / kThreads,
                                                                          (uint64_t)sms * 8));
    const uint64_t chunks = ((uint64_t)nnz + kEntriesPerThread - 1) / kEntriesPerThread;
    const int entry_blocks =
        (int)std::max<uint64_t>(1, std::min<uint64_t>((chunks + kThreads - 1) / kThreads, (uint64_t)sms * 16));
    cudaError_t e = cudaMemsetAsync(counters, 0xFF, sizeof(uint32_t), st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(counters + 1, 0, 3 * sizeof(uint32_t), st);
    if (e != cudaSuccess)
        return e;
    k_cc_init<<<rows_blocks, kThreads, 0, st>>>(rp, ci, n, nnz, parent, counters);
    if (nnz > 0)
        k_cc_hook<<<entry_blocks, kThreads, 0, st>>>(rp, ci, n, nnz, parent, counters);
    k_connect_rowlen<<<rows_blocks, kThreads, 0, st>>>(rp, n, nnz, parent, counters, out_rp);
    e = launch_scan(out_rp + 1, n, partials, st);
    if (e != cudaSuccess)
        return e;
    k_connect_copy<<<std::max(entry_blocks, rows_blocks), kThreads, 0, st>>>(rp, ci, n, nnz, parent, counters,
                                                                             out_rp, out_ci, cap);
    return cudaGetLastError();
}

}  // namespace pbrcm
