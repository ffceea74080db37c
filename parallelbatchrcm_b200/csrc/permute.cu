// permute.cu -- the reordered matrix B = P A P^T on the device.
//
// Row i of B is row perm[i] of A with every column c renamed inv[c] (inv is
// the inverse permutation) and its entries sorted by the new column, equal
// new columns (duplicate entries of A) in their original order; values move
// with their entries and map[k] names the entry of A that entry k of B came
// from.  This is what the reference's `-o` path computes with
// cusolverSpXcsrpermHost(p = q = perm) plus its value shuffle
// (include/device/rcm_cusolver.cuh:154-185); here it is an HBM-bound gather /
// scatter:
//   1. inv[perm[k]] = k with a bijection check (k_bw_inverse, kernels.cu);
//   2. new row lengths, scanned into row_ptr_out (three small kernels);
//   3. eight lanes per row of at most kGroupRow entries (rows of sparse
//      matrices are short: 5-7 for grids), four rows per warp: the row's
//      entries load coalesced and are ranked with shuffles;
//   4. one warp per listed row of at most kWarpRow entries: the same rank
//      count over the warp's shared memory;
//   5. one CTA per longer row: a stable 8-bit LSD radix sort of (new column,
//      slot) in global scratch (4 words per entry).
#include <algorithm>
#include <cstdint>

#include <cuda_runtime.h>

#include "kernels.h"
#include "types.h"

namespace pbrcm {

namespace {

constexpr uint32_t kGroupRow = 8;               // longest row the lane-group path takes
constexpr int kWarpRow = (int)kPermuteWarpRow;  // longest row the warp path takes
constexpr int kRowWarps = 8;       // warps per CTA of the warp path
constexpr int kScanItems = 8;      // elements per thread of the scan
constexpr int kScanThreads = 1024;
constexpr int kLongThreads = 512;  // threads of the long-row CTA

__device__ __forceinline__ void fail(DevResult* r, uint32_t where)
{
    if (atomicCAS(&r->status, 0u, (uint32_t)kErrArg) == 0u)
        r->where = where;
}

// row_ptr_out[i + 1] = length of row perm[i]; row_ptr_out[0] = 0.
__global__ void __launch_bounds__(256) k_perm_rowlen(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ perm,
                                                     uint32_t n, uint32_t* __restrict__ out_rp, DevResult* res)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t src = perm[i];
        uint32_t len = 0;
        if (src < n)
            len = rp[src + 1] - rp[src];
        else
            fail(res, 310);
        out_rp[i + 1] = len;
        if (i == 0)
            out_rp[0] = 0;
    }
}

// In-place inclusive scan of data[0..m), pass 1: each block scans its
// kScanThreads * kScanItems elements and writes its total to partials[b].
__device__ __forceinline__ uint32_t block_incl_scan(uint32_t v, uint32_t* warp_sums)
{
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= (uint32_t)o)
            x += y;
    }
    if (lane == 31)
        warp_sums[w] = x;
    __syncthreads();
    if (w == 0) {
        uint32_t s = lane < (blockDim.x >> 5) ? warp_sums[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, s, o);
            if (lane >= (uint32_t)o)
                s += y;
        }
        warp_sums[lane] = s;
    }
    __syncthreads();
    const uint32_t r = x + (w > 0 ? warp_sums[w - 1] : 0u);
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_local(uint32_t* data, uint64_t m, uint32_t* partials)
{
    __shared__ uint32_t ws[32];
    const uint64_t base = (uint64_t)blockIdx.x * kScanThreads * kScanItems + (uint64_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t local = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < m ? data[base + k] : 0u;
        local += v[k];
    }
    const uint32_t incl = block_incl_scan(local, ws);
    uint32_t run = incl - local;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        run += v[k];
        if (base + k < m)
            data[base + k] = run;
    }
    if (threadIdx.x == kScanThreads - 1)
        partials[blockIdx.x] = incl;
}

// Pass 2: exclusive scan of the block totals (one block, any count).
__global__ void __launch_bounds__(kScanThreads) k_scan_partials(uint32_t* partials, uint32_t nb)
{
    __shared__ uint32_t ws[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0)
        carry = 0;
    __syncthreads();
    for (uint32_t b0 = 0; b0 < nb; b0 += kScanThreads) {
        const uint32_t i = b0 + threadIdx.x;
        const uint32_t v = i < nb ? partials[i] : 0u;
        const uint32_t incl = block_incl_scan(v, ws);
        const uint32_t c = carry;
        if (i < nb)
            partials[i] = c + incl - v;
        __syncthreads();
        if (threadIdx.x == kScanThreads - 1)
            carry = c + incl;
        __syncthreads();
    }
}

// Pass 3: add each block's exclusive prefix.
__global__ void __launch_bounds__(kScanThreads) k_scan_add(uint32_t* data, uint64_t m, const uint32_t* partials)
{
    const uint32_t add = partials[blockIdx.x];
    const uint64_t base = (uint64_t)blockIdx.x * kScanThreads * kScanItems;
    for (uint32_t k = threadIdx.x; k < (uint32_t)(kScanThreads * kScanItems); k += kScanThreads)
        if (base + k < m)
            data[base + k] += add;
}

struct PermView {
    const uint32_t* rp;
    const uint32_t* ci;
    const void* vals;
    const uint32_t* perm;
    const uint32_t* inv;
    const uint32_t* out_rp;
    uint32_t* out_ci;
    void* out_vals;
    uint32_t* out_map;
    uint32_t n;
    uint32_t nnz;
    DevResult* res;
};

// Rows of B of at most kGroupRow entries, kGroupRow lanes each (four rows
// per warp): a row's entries load with adjacent lanes (coalesced), the
// renamed columns are ranked across the group with shuffles.  Longer rows are
// listed for k_permute_rows (mid[0..counters[0])).
template <typename V>
__global__ void __launch_bounds__(256) k_permute_short(PermView a, uint32_t* mid, uint32_t* counters)
{
    constexpr uint32_t G = kGroupRow;
    const V* vals = static_cast<const V*>(a.vals);
    V* out_vals = static_cast<V*>(a.out_vals);
    const uint32_t lane = threadIdx.x & 31, q = lane & (G - 1), grp = lane / G;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    constexpr uint32_t RPW = 32 / G;  // rows per warp
    // base is the same in the whole warp, so every lane reaches every shuffle
    for (uint64_t base = warp * RPW; base < a.n; base += nwarps * RPW) {
        const uint64_t i = base + grp;
        bool act = i < a.n;
        uint32_t beg = 0, len = 0, dst = 0;
        if (act) {
            const uint32_t src = a.perm[i];
            if (src >= a.n) {
                act = false;  // reported by k_perm_rowlen
            } else {
                beg = a.rp[src];
                len = a.rp[src + 1] - beg;
                dst = a.out_rp[i];
                if (dst > a.nnz || len > a.nnz - dst || beg > a.nnz || len > a.nnz - beg) {
                    if (q == 0)
                        fail(a.res, 311);  // not a permutation: the rows do not tile the output
                    act = false;
                } else if (len > G) {
                    if (q == 0)
                        mid[atomicAdd(counters, 1u)] = (uint32_t)i;  // at most n rows: the list holds n
                    act = false;
                }
            }
        }
        const bool mine = act && q < len;
        uint32_t key = 0xFFFFFFFFu;
        if (mine) {
            const uint32_t c = a.ci[beg + q];
            key = c < a.n ? a.inv[c] : 0xFFFFFFFFu;
        }
        uint32_t r = 0;
#pragma unroll
        for (uint32_t t = 0; t < G; ++t) {
            const uint32_t kt = __shfl_sync(0xFFFFFFFFu, key, (lane & ~(G - 1)) + t);
            r += (t < len) && ((kt < key) || (kt == key && t < q));
        }
        if (mine) {
            a.out_ci[dst + r] = key;
            if (out_vals)
                out_vals[dst + r] = vals[beg + q];
            if (a.out_map)
                a.out_map[dst + r] = beg + q;
        }
    }
}

// Listed rows of B by one warp each (rows of at most kWarpRow entries);
// longer rows are listed for k_permute_long.
template <typename V>
__global__ void __launch_bounds__(kRowWarps * 32) k_permute_rows(PermView a, const uint32_t* mid,
                                                                 const uint32_t* counters, uint32_t* long_rows,
                                                                 uint32_t cap_long, uint32_t* nlong)
{
    __shared__ uint32_t keys[kRowWarps][kWarpRow];
    const uint32_t w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t* kw = keys[w];
    const V* vals = static_cast<const V*>(a.vals);
    V* out_vals = static_cast<V*>(a.out_vals);
    const uint32_t nmid = min(counters[0], a.n);
    for (uint32_t r0 = blockIdx.x * kRowWarps + w; r0 < nmid; r0 += gridDim.x * kRowWarps) {
        const uint32_t i = mid[r0];
        const uint32_t src = a.perm[i];
        const uint32_t beg = a.rp[src], len = a.rp[src + 1] - beg, dst = a.out_rp[i];
        if (len > (uint32_t)kWarpRow) {
            if (lane == 0) {
                const uint32_t k = atomicAdd(nlong, 1u);
                if (k < cap_long)
                    long_rows[k] = (uint32_t)i;
                else
                    fail(a.res, 312);
            }
            continue;
        }
        for (uint32_t j = lane; j < len; j += 32) {
            const uint32_t c = a.ci[beg + j];
            kw[j] = c < a.n ? a.inv[c] : 0xFFFFFFFFu;
        }
        __syncwarp();
        for (uint32_t j = lane; j < len; j += 32) {
            const uint32_t kj = kw[j];
            uint32_t r = 0;
            for (uint32_t t = 0; t < len; ++t) {
                const uint32_t kt = kw[t];
                r += (kt < kj) || (kt == kj && t < j);
            }
            a.out_ci[dst + r] = kj;
            if (out_vals)
                out_vals[dst + r] = vals[beg + j];
            if (a.out_map)
                a.out_map[dst + r] = beg + j;
        }
        __syncwarp();
    }
}

// One stable counting pass on digit (key >> shift) & 255 over len entries,
// by the whole CTA: per-digit histogram, then tiles in which every warp
// ranks equal digits with a match mask and the warps add up in order.
__device__ void radix_pass(const uint32_t* sk, const uint32_t* sv, uint32_t* dk, uint32_t* dv, uint32_t len,
                           uint32_t shift, uint32_t* hist, uint32_t* wcnt)
{
    constexpr int W = kLongThreads / 32;
    const uint32_t t = threadIdx.x, lane = t & 31, w = t >> 5;
    for (uint32_t d = t; d < 256; d += kLongThreads)
        hist[d] = 0;
    __syncthreads();
    for (uint32_t i = t; i < len; i += kLongThreads)
        atomicAdd(&hist[(sk[i] >> shift) & 255u], 1u);
    __syncthreads();
    if (t == 0) {
        uint32_t run = 0;
        for (int d = 0; d < 256; ++d) {
            const uint32_t h = hist[d];
            hist[d] = run;
            run += h;
        }
    }
    __syncthreads();
    for (uint32_t base = 0; base < len; base += kLongThreads) {
        for (uint32_t i = t; i < (uint32_t)(W * 256); i += kLongThreads)
            wcnt[i] = 0;
        __syncthreads();
        const uint32_t i = base + t;
        const bool act = i < len;
        uint32_t key = 0, val = 0, dg = 0;
        if (act) {
            key = sk[i];
            val = sv[i];
            dg = (key >> shift) & 255u;
        }
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, act ? dg : 256u + lane);
        const uint32_t below = peers & ((1u << lane) - 1u);
        if (act && below == 0)
            wcnt[w * 256 + dg] = __popc(peers);
        __syncthreads();
        if (act) {
            uint32_t before = 0;
            for (uint32_t ww = 0; ww < w; ++ww)
                before += wcnt[ww * 256 + dg];
            const uint32_t pos = hist[dg] + before + __popc(below);
            dk[pos] = key;
            dv[pos] = val;
        }
        __syncthreads();
        for (uint32_t d = t; d < 256; d += kLongThreads) {
            uint32_t add = 0;
            for (int ww = 0; ww < W; ++ww)
                add += wcnt[ww * 256 + d];
            hist[d] += add;
        }
        __syncthreads();
    }
}

// Rows longer than kWarpRow, one CTA each.  scratch: 4 * nnz words; the row
// with output offset dst uses [dst, dst + len) of each quarter.
template <typename V>
__global__ void __launch_bounds__(kLongThreads) k_permute_long(PermView a, const uint32_t* long_rows,
                                                               const uint32_t* nlong, uint32_t cap_long,
                                                               uint32_t* scratch, uint32_t key_passes)
{
    __shared__ uint32_t hist[256];
    __shared__ uint32_t wcnt[(kLongThreads / 32) * 256];
    const V* vals = static_cast<const V*>(a.vals);
    V* out_vals = static_cast<V*>(a.out_vals);
    const uint32_t count = min(*nlong, cap_long);
    for (uint32_t r = blockIdx.x; r < count; r += gridDim.x) {
        const uint32_t i = long_rows[r];
        const uint32_t src = a.perm[i];
        const uint32_t beg = a.rp[src], len = a.rp[src + 1] - beg, dst = a.out_rp[i];
        uint32_t* k0 = scratch + dst;
        uint32_t* v0 = scratch + (size_t)a.nnz + dst;
        uint32_t* k1 = scratch + 2 * (size_t)a.nnz + dst;
        uint32_t* v1 = scratch + 3 * (size_t)a.nnz + dst;
        for (uint32_t j = threadIdx.x; j < len; j += kLongThreads) {
            const uint32_t c = a.ci[beg + j];
            k0[j] = c < a.n ? a.inv[c] : 0xFFFFFFFFu;
            v0[j] = j;
        }
        __syncthreads();
        for (uint32_t p = 0; p < key_passes; ++p) {
            if (p & 1)
                radix_pass(k1, v1, k0, v0, len, 8 * p, hist, wcnt);
            else
                radix_pass(k0, v0, k1, v1, len, 8 * p, hist, wcnt);
        }
        const uint32_t* kf = (key_passes & 1) ? k1 : k0;
        const uint32_t* vf = (key_passes & 1) ? v1 : v0;
        for (uint32_t j = threadIdx.x; j < len; j += kLongThreads) {
            const uint32_t slot = vf[j];
            a.out_ci[dst + j] = kf[j];
            if (out_vals)
                out_vals[dst + j] = vals[beg + slot];
            if (a.out_map)
                a.out_map[dst + j] = beg + slot;
        }
        __syncthreads();
    }
}

template <typename V>
cudaError_t launch_rows(const PermView& a, uint32_t* mid, uint32_t* counters, uint32_t* long_rows, uint32_t cap_long,
                        uint32_t* scratch, int sms, cudaStream_t st)
{
    uint32_t* nlong = counters + 1;
    const int sb = (int)std::min<uint64_t>(((uint64_t)a.n + 31) / 32, (uint64_t)sms * 16);
    k_permute_short<V><<<sb < 1 ? 1 : sb, 256, 0, st>>>(a, mid, counters);
    k_permute_rows<V><<<sms * 4, kRowWarps * 32, 0, st>>>(a, mid, counters, long_rows, cap_long, nlong);
    if (scratch != nullptr && cap_long > 0) {
        uint32_t bits = 1;
        while (bits < 32 && (a.n - 1u) >> bits)
            ++bits;
        const uint32_t passes = (bits + 7) / 8;
        k_permute_long<V><<<sms, kLongThreads, 0, st>>>(a, long_rows, nlong, cap_long, scratch, passes);
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_scan(uint32_t* data, uint64_t m, uint32_t* partials, cudaStream_t st)
{
    const uint64_t per = (uint64_t)kScanThreads * kScanItems;
    const uint32_t nb = (uint32_t)((m + per - 1) / per);
    if (nb == 0)
        return cudaSuccess;
    k_scan_local<<<nb, kScanThreads, 0, st>>>(data, m, partials);
    k_scan_partials<<<1, kScanThreads, 0, st>>>(partials, nb);
    k_scan_add<<<nb, kScanThreads, 0, st>>>(data, m, partials);
    return cudaGetLastError();
}

cudaError_t launch_permute(const uint32_t* rp, const uint32_t* ci, const void* vals, uint32_t val_bytes, uint32_t n,
                           uint32_t nnz, const uint32_t* perm, uint32_t* inv, uint32_t* out_rp, uint32_t* out_ci,
                           void* out_vals, uint32_t* out_map, uint32_t* partials, uint32_t* mid_rows,
                           uint32_t* long_rows, uint32_t cap_long, uint32_t* counters, uint32_t* scratch,
                           DevResult* res, int sms, cudaStream_t st)
{
    int blocks = (int)std::min<uint64_t>(((uint64_t)n + 255) / 256, (uint64_t)sms * 8);
    if (blocks < 1)
        blocks = 1;
    cudaError_t e = cudaMemsetAsync(inv, 0xFF, sizeof(uint32_t) * (size_t)n, st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(counters, 0, 2 * sizeof(uint32_t), st);
    if (e != cudaSuccess)
        return e;
    launch_perm_inverse(perm, n, inv, res, blocks, st);
    k_perm_rowlen<<<blocks, 256, 0, st>>>(rp, perm, n, out_rp, res);
    e = launch_scan(out_rp + 1, n, partials, st);
    if (e != cudaSuccess)
        return e;
    PermView a{rp, ci, val_bytes ? vals : nullptr, perm, inv, out_rp, out_ci, val_bytes ? out_vals : nullptr,
               out_map, n, nnz, res};
    if (val_bytes == 8)
        return launch_rows<unsigned long long>(a, mid_rows, counters, long_rows, cap_long, scratch, sms, st);
    return launch_rows<uint32_t>(a, mid_rows, counters, long_rows, cap_long, scratch, sms, st);
}

cudaError_t launch_permute_long(const uint32_t* rp, const uint32_t* ci, const void* vals, uint32_t val_bytes,
                                uint32_t n, uint32_t nnz, const uint32_t* perm, const uint32_t* inv,
                                const uint32_t* out_rp, uint32_t* out_ci, void* out_vals, uint32_t* out_map,
                                const uint32_t* long_rows, uint32_t cap_long, const uint32_t* counters,
                                uint32_t* scratch, DevResult* res, int sms, cudaStream_t st)
{
    PermView a{rp, ci, val_bytes ? vals : nullptr, perm, inv, out_rp, out_ci, val_bytes ? out_vals : nullptr,
               out_map, n, nnz, res};
    uint32_t bits = 1;
    while (bits < 32 && (n - 1u) >> bits)
        ++bits;
    const uint32_t passes = (bits + 7) / 8;
    if (val_bytes == 8)
        k_permute_long<unsigned long long><<<sms, kLongThreads, 0, st>>>(a, long_rows, counters + 1, cap_long,
                                                                         scratch, passes);
    else
        k_permute_long<uint32_t><<<sms, kLongThreads, 0, st>>>(a, long_rows, counters + 1, cap_long, scratch,
                                                               passes);
    return cudaGetLastError();
}

uint32_t scan_partials_count(uint32_t n)
{
    const uint64_t per = (uint64_t)kScanThreads * kScanItems;
    return (uint32_t)(((uint64_t)n + per - 1) / per);
}

uint32_t permute_long_cap(uint32_t n, uint64_t nnz)
{
    // a row longer than kWarpRow takes more than kWarpRow of the nnz entries
    return (uint32_t)std::min<uint64_t>(n, nnz / (kWarpRow + 1) + 1);
}

}  // namespace pbrcm
