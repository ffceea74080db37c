// wide.cu -- the level-synchronous engine for wide, shallow graphs.
//
// The team engine (k_reorder_team) runs every level inside one cooperative
// launch of one CTA per SM: right for deep graphs (meshes: hundreds of
// levels of a few thousand nodes), but a level of a million nodes then keeps
// each CTA busy with hundreds of chunks one after the other, each a chain of
// dependent loads.  Graphs whose BFS levels hold a large share of the nodes
// (random and expander-like graphs: 10-20 levels) are run here instead, as
// the reference's GPU_SIMPLE does (src/device/rcm_gpu.cu:310-389: a loop of
// kernels per BFS level), but with the team engine's exact chunk machinery
// and many CTAs per SM:
//   k_wide_collect  every CTA takes a contiguous run of the frontier, forms
//                   chunks (<= B parents, <= EMAX edges), finds and ranks the
//                   children (engine.cuh Chunk::collect) and stages them at
//                   its run's level-relative edge offset; per-CTA totals;
//   k_wide_place    the same runs: prefix of the totals, then the staged
//                   children placed (records, permutation) and their edges
//                   claimed for the next level, 16 lanes per child; the
//                   last CTA to finish advances the state: the next level,
//                   or at the end of a pass the start search's next step
//                   (simple_peripheral.cpp:92-141, as reorder_matrix runs
//                   it) and the next pass's start.
// The host enqueues level steps in batches sized by the previous pass's
// level count and reads the state only between batches; steps after the end
// return at once.  Every result (start, passes, levels, permutation,
// bandwidth) is the team engine's.
#include <algorithm>
#include <cstdint>

#include "engine.cuh"
#include "kernels.h"

namespace pbrcm {

namespace {

__device__ __forceinline__ WideState load_state(const WideState* ws)
{
    WideState st;
    const uint4* p = reinterpret_cast<const uint4*>(ws);
    const uint4 q0 = __ldcg(p), q1 = __ldcg(p + 1), q2 = __ldcg(p + 2);
    st.a = q0.x;
    st.b = q0.y;
    st.Ka = q0.z;
    st.Kb = q0.w;
    st.L = q1.x;
    st.last_start = q1.y;
    st.phase = q1.z;
    st.base = q1.w;
    st.start = q2.x;
    st.passes = q2.y;
    st.ecc = q2.z;
    st.lastdist = q2.w;
    st.pid = __ldcg(&ws->pid);
    st.steps = __ldcg(&ws->steps);
    return st;
}

// The contiguous run of frontier positions of CTA R of G.
__device__ __forceinline__ void cta_run(const WideState& st, uint32_t R, uint32_t G, uint32_t& p0, uint32_t& p1)
{
    const uint32_t F = st.b - st.a;
    p0 = st.a + (uint32_t)(((uint64_t)F * R) / G);
    p1 = st.a + (uint32_t)(((uint64_t)F * (R + 1)) / G);
}

}  // namespace

template <int B, int EMAX>
__global__ void __launch_bounds__(B) k_wide_collect(MatrixView M, const WideState* ws, unsigned long long* tot)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    auto& s = *reinterpret_cast<Smem<B, EMAX>*>(smem_raw);
    const WideState st = load_state(ws);
    if (st.phase == kWideDone || read_status(M.res) != 0)
        return;
    Chunk<B, EMAX> ch{s, M, st.base};
    uint32_t p0, p1;
    cta_run(st, blockIdx.x, gridDim.x, p0, p1);
    uint32_t cnt = 0, esum = 0, stage_base = 0;
    for (uint32_t p = p0; p < p1;) {
        const uint32_t used = ch.form(p, p1);
        if (p == p0)
            stage_base = s.peb[0] - st.Ka;
        if (s.hub) {  // the host hands no matrix with rows over EMAX to this engine
            if (threadIdx.x == 0)
                set_status(M.res, kErrCheck, 140);
            break;
        }
        const Agg g = ch.collect(st.phase == kWideFinal);
        ch.stage_children(stage_base + cnt, esum);
        cnt += g.cnt;
        esum += g.esum;
        p += used;
        __syncthreads();
    }
    if (threadIdx.x == 0)
        tot[blockIdx.x] = (unsigned long long)cnt | ((unsigned long long)esum << 32);
}

// Starts a pass from st.start: key base, level 0 = the start node, its edges
// claimed.  Block-wide; st is this CTA's shared copy, written back by the
// caller.
template <int B>
__device__ bool wide_begin_pass(const MatrixView& M, WideState& st, bool reverse)
{
    const uint32_t kspan = M.nnz + 2u;
    const uint32_t pmax = (uint32_t)(0xFFFFFFFFull / kspan) - 1u;
    if (st.pid + 1 > pmax)
        return false;  // the key space is spent: the team engine (it resets claims) takes over
    const uint32_t pid = st.pid + 1;
    const uint32_t base = pid * kspan + M.nnz + 1u;
    const uint4 sn = ld_node(M.node + st.start);
    const uint32_t rs0 = sn.y, deg0 = sn.z;
    if (threadIdx.x == 0) {
        atomicMax(claim_ptr(M, st.start), base);
        __stcg(reinterpret_cast<uint4*>(M.rec), make_uint4(st.start, rs0, deg0, 0u));
        if (st.phase == kWideFinal)
            M.perm[reverse ? M.n - 1 : 0] = st.start;
    }
    for (uint32_t k = threadIdx.x; k < deg0; k += B) {
        const uint32_t d = ld_ro(M.ci + rs0 + k);
        if (PB_CHECK(M.res, d < M.n, 141))
            atomicMax(claim_ptr(M, d), base - 1u - k);
    }
    st.pid = pid;
    st.base = base;
    st.a = 0;
    st.b = 1;
    st.Ka = 0;
    st.Kb = deg0;
    st.L = 0;
    st.last_start = 0;
    return true;
}

__device__ __forceinline__ void store_state(WideState* ws, const WideState& st)
{
    uint4* p = reinterpret_cast<uint4*>(ws);
    __stcg(p, make_uint4(st.a, st.b, st.Ka, st.Kb));
    __stcg(p + 1, make_uint4(st.L, st.last_start, st.phase, st.base));
    __stcg(p + 2, make_uint4(st.start, st.passes, st.ecc, st.lastdist));
    __stcg(&ws->pid, st.pid);
    __stcg(&ws->steps, st.steps);
}

__device__ __forceinline__ void wide_finish(const MatrixView& M, WideState& st, uint32_t status, uint32_t where)
{
    if (threadIdx.x == 0 && status != kOk)
        set_status(M.res, status, where);
    st.phase = kWideDone;
}

// First pass: node table, then the start (the caller's, or n/2 and the
// search).  One CTA of B threads after k_wide_init.
template <int B>
__global__ void __launch_bounds__(B) k_wide_begin(MatrixView M, WideState* ws, Options opt)
{
    WideState st{};
    if (opt.start != kUnvisited && opt.start >= M.n) {
        wide_finish(M, st, kErrArg, 2);
        if (threadIdx.x == 0)
            store_state(ws, st);
        return;
    }
    if (opt.start != kUnvisited) {
        st.start = opt.start;
        st.phase = kWideFinal;
    } else {
        st.start = M.n / 2;
        st.phase = kWideSearch;
        st.passes = 1;
    }
    if (read_status(M.res) != 0 || !wide_begin_pass<B>(M, st, opt.reverse != 0))
        wide_finish(M, st, read_status(M.res) != 0 ? kOk : kNeedTeam, 142);
    if (threadIdx.x == 0)
        store_state(ws, st);
}

template <int B>
__global__ void __launch_bounds__(B) k_wide_init(MatrixView M)
{
    init_nodes<B>(M, blockIdx.x, gridDim.x);
}

// After a level step: the next level, or the end of a pass.  Block-wide, by
// the last CTA of the place kernel (every other CTA of the step is done).
template <int B>
__device__ void wide_advance(const MatrixView& M, WideState* ws, const unsigned long long* tot, uint32_t G,
                             const Options& opt, unsigned long long* tmp, uint32_t* bcast)
{
    WideState st = load_state(ws);
    const uint32_t t = threadIdx.x;
    const uint32_t n = M.n;
    if (read_status(M.res) != 0) {
        if (t == 0) {
            st.phase = kWideDone;
            store_state(ws, st);
        }
        return;
    }
    unsigned long long cnt = 0, esum = 0;
    for (uint32_t r = t; r < G; r += B) {
        const unsigned long long u = __ldcg(tot + r);
        cnt += u & 0xFFFFFFFFull;
        esum += u >> 32;
    }
    block_reduce_sum2<B>(cnt, esum, tmp);
    st.steps += 1;
    if (cnt > 0) {
        st.last_start = st.b;
        st.a = st.b;
        st.b += (uint32_t)cnt;
        st.Ka = st.Kb;
        st.Kb += (uint32_t)esum;
        st.L += 1;
        if (st.b > n)
            wide_finish(M, st, kErrCheck, 143);
        if (t == 0)
            store_state(ws, st);
        return;
    }
    // the pass has ended: placed st.b nodes in st.L + 1 levels
    const uint32_t placed = st.b, nl = st.L + 1, ls = st.last_start;
    if (t == 0)
        __stcg(&ws->prev_levels, nl);
    if (st.phase == kWideFinal) {
        if (t == 0) {
            if (placed != n) {
                set_status(M.res, kErrDisconnected, 1);
                M.res->placed = placed;
            } else {
                M.res->start = st.start;
                M.res->passes = st.passes;
                M.res->ecc = st.ecc;
                M.res->levels = nl;
                M.res->placed = placed;
            }
        }
        st.phase = kWideDone;
    } else if (placed != n) {
        wide_finish(M, st, kErrDisconnected, 0);
    } else {
        const uint32_t dist = nl - 1;
        bool go = true;
        if (dist == st.lastdist) {
            st.ecc = dist;
            if (opt.mode == kModeStartOnly) {
                if (t == 0) {
                    M.res->start = st.start;
                    M.res->passes = st.passes;
                    M.res->ecc = st.ecc;
                    M.res->placed = n;
                }
                st.phase = kWideDone;
                go = false;
            } else {
                st.phase = kWideFinal;  // the ordered pass from the same start
            }
        } else {
            if (t == 0)
                bcast[0] = next_peripheral_start(M, opt.outnodes, ls);
            __syncthreads();
            st.start = bcast[0];
            st.lastdist = dist;
            st.passes += 1;
            if (st.passes > n + 1) {  // eccentricities only grow; cannot happen on a valid run
                wide_finish(M, st, kErrCheck, 3);
                go = false;
            }
        }
        if (go && !wide_begin_pass<B>(M, st, opt.reverse != 0))
            wide_finish(M, st, kNeedTeam, 144);
    }
    __syncthreads();
    if (t == 0)
        store_state(ws, st);
}

// Places the `count` children staged at M.stage[at..] at positions P0.. with
// edge ids K0 + their staged edge offsets, and claims their edges: what
// Chunk::place_staged computes, with 16 lanes per child so that a row is read
// by consecutive lanes and each child's record is one broadcast load.
template <int B>
__device__ void wide_place_children(const MatrixView& M, uint32_t base, uint32_t at, uint32_t count, uint32_t P0,
                                    uint32_t K0, bool write_perm, bool reverse)
{
    constexpr uint32_t kLanes = 16;
    const uint32_t sub = threadIdx.x & (kLanes - 1);
    for (uint32_t i = threadIdx.x / kLanes; i < count; i += B / kLanes) {
        uint4 r = make_uint4(0u, 0u, 0u, 0u);
        if (PB_CHECK(M.res, (uint64_t)at + i < M.nnz, 146))
            r = __ldcg(reinterpret_cast<const uint4*>(M.stage) + at + i);
        const uint32_t pos = P0 + i;
        const uint32_t eb = K0 + r.w;
        if (sub == 0 && PB_CHECK(M.res, pos < M.n, 147)) {
            __stcg(reinterpret_cast<uint4*>(M.rec) + pos, make_uint4(r.x, r.y, r.z, eb));
            if (write_perm)
                M.perm[reverse ? M.n - 1 - pos : pos] = r.x;
        }
        const uint32_t kb = base - 1u - eb;
        for (uint32_t k = sub; k < r.z; k += kLanes) {
            if (PB_CHECK(M.res, (uint64_t)r.y + k < M.nnz, 148)) {
                const uint32_t d = ld_ro(M.ci + r.y + k);
                if (PB_CHECK(M.res, d < M.n, 149))
                    atomicMax(claim_ptr(M, d), kb - k);
            }
        }
    }
}

// B threads per CTA, the same number of CTAs as the collect (the CTAs' runs
// match); no chunk buffers, so B can be twice the collect's threads.
template <int B>
__global__ void __launch_bounds__(B) k_wide_place(MatrixView M, WideState* ws, const unsigned long long* tot,
                                                  Options opt, uint32_t fused)
{
    __shared__ struct {
        unsigned long long tmp64[2 * (B / 32) + 2];
        uint32_t bcast[2];
    } s;
    const WideState st = load_state(ws);
    if (st.phase == kWideDone)
        return;  // every CTA reads the same phase
    const uint32_t R = blockIdx.x, G = gridDim.x;
    if (read_status(M.res) == 0) {
        unsigned long long pc = 0, pe = 0;
        for (uint32_t r = threadIdx.x; r < R; r += B) {
            const unsigned long long u = __ldcg(tot + r);
            pc += u & 0xFFFFFFFFull;
            pe += u >> 32;
        }
        block_reduce_sum2<B>(pc, pe, s.tmp64);
        const uint32_t cnt = (uint32_t)(__ldcg(tot + R) & 0xFFFFFFFFull);
        if (cnt > 0) {
            uint32_t p0, p1;
            cta_run(st, R, G, p0, p1);
            const uint32_t stage_base = __ldcg(&reinterpret_cast<const uint4*>(M.rec)[p0].w) - st.Ka;
            wide_place_children<B>(M, st.base, stage_base, cnt, st.b + (uint32_t)pc, st.Kb + (uint32_t)pe,
                                   st.phase == kWideFinal, opt.reverse != 0);
        }
    }
    if (!fused)
        return;  // k_wide_advance follows
    // the last CTA to finish advances the state
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s.bcast[1] = atomicAdd(&ws->ticket, 1u) == G - 1 ? 1u : 0u;
    }
    __syncthreads();
    if (s.bcast[1] == 0)
        return;
    __threadfence();
    if (threadIdx.x == 0)
        ws->ticket = 0;
    wide_advance<B>(M, ws, tot, G, opt, s.tmp64, s.bcast);
}

template <int B>
__global__ void __launch_bounds__(B) k_wide_advance(MatrixView M, WideState* ws, const unsigned long long* tot,
                                                    uint32_t G, Options opt)
{
    __shared__ unsigned long long tmp[2 * (B / 32) + 2];
    __shared__ uint32_t bcast[1];
    if (load_state(ws).phase == kWideDone)
        return;
    wide_advance<B>(M, ws, tot, G, opt, tmp, bcast);
}

// inv[rec[pos].node] = pos (Cuthill-McKee positions) for the bandwidth rows.
__global__ void __launch_bounds__(256) k_wide_inverse(MatrixView M, uint32_t* inv)
{
    if (read_status(M.res) != 0)
        return;
    for (uint64_t pos = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; pos < M.n;
         pos += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = __ldcg(&reinterpret_cast<const uint4*>(M.rec)[pos].x);
        if (PB_CHECK(M.res, v < M.n, 145))
            inv[v] = (uint32_t)pos;
    }
}

namespace {
constexpr int kWideB = 256, kWideEmax = 1024;
constexpr int kPlaceB = 512;  // threads of the place kernel's CTAs
}

int wide_ctas_per_sm()
{
    int occ = 0;
    const size_t smem = sizeof(Smem<kWideB, kWideEmax>);
    if (cudaFuncSetAttribute(k_wide_collect<kWideB, kWideEmax>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
        return 0;
    // the place kernel needs no co-residency (its last CTA takes a ticket),
    // so the collect's occupancy alone sets the number of CTAs
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_wide_collect<kWideB, kWideEmax>, kWideB, smem) !=
        cudaSuccess)
        return 0;
    return std::max(1, occ);
}

uint32_t wide_emax() { return (uint32_t)kWideEmax; }

cudaError_t launch_wide_start(const MatrixView& M, const Options& opt, WideState* ws, int sms, cudaStream_t st)
{
    const int blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)M.n + kWideB - 1) / kWideB,
                                                                      (uint64_t)sms * 8));
    k_wide_init<kWideB><<<blocks, kWideB, 0, st>>>(M);
    k_wide_begin<kWideB><<<1, kWideB, 0, st>>>(M, ws, opt);
    return cudaGetLastError();
}

cudaError_t launch_wide_steps(const MatrixView& M, const Options& opt, WideState* ws, unsigned long long* tot,
                              int ctas, int steps, bool fused, cudaStream_t st)
{
    const size_t smem = sizeof(Smem<kWideB, kWideEmax>);
    for (int i = 0; i < steps; ++i) {
        k_wide_collect<kWideB, kWideEmax><<<ctas, kWideB, smem, st>>>(M, ws, tot);
        k_wide_place<kPlaceB><<<ctas, kPlaceB, 0, st>>>(M, ws, tot, opt, fused ? 1u : 0u);
        if (!fused)
            k_wide_advance<kWideB><<<1, kWideB, 0, st>>>(M, ws, tot, (uint32_t)ctas, opt);
    }
    return cudaGetLastError();
}

cudaError_t launch_wide_bandwidth(const MatrixView& M, uint32_t* inv, int sms, cudaStream_t st)
{
    const int blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)M.n + 255) / 256, (uint64_t)sms * 8));
    k_wide_inverse<<<blocks, 256, 0, st>>>(M, inv);
    return launch_bw_rows(M.rp, M.ci, M.n, inv, M.res, sms, st);
}

}  // namespace pbrcm
