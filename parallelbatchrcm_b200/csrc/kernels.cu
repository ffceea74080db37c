// kernels.cu -- sm_100a kernels of the engine and their host launchers.
//
//   k_validate        one pass over row_ptr / col_idx (coalesced): CSR sanity
//                     and the largest valence (decides whether hub scratch is
//                     needed); a bad CSR never reaches the engine.
//   k_reorder_team    one matrix, all CTAs of a cooperative launch: start
//                     search + CM pass + reverse + bandwidth in one launch
//                     (agg: 2 words per CTA for the level all-gather, then
//                     one barrier flag word per CTA + phantom; all zeroed
//                     before the launch together with the GridSync words).
//   k_bw_*            bandwidth / profile of a caller permutation.
// The batch kernels (k_reorder_batch, k_reorder_cluster) are in pool.cuh,
// one translation unit per pool shape (pool_p0.cu .. pool_p4.cu).
#include <algorithm>
#include <cstdio>

#include "engine.cuh"
#include "kernels.h"

namespace pbrcm {

// ---------------------------------------------------------------------------
__device__ void validate_one(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci, uint32_t n,
                             uint32_t nnz, DevResult* res, uint64_t tid, uint64_t stride)
{
    __shared__ uint32_t s_max[32];
    uint32_t mx = 0;
    bool bad = false;
    for (uint64_t i = tid; i < n; i += stride) {
        const uint32_t a = rp[i], b = rp[i + 1];
        if (b < a || b > nnz)
            bad = true;
        else
            mx = max(mx, b - a);
    }
    if (tid == 0 && (rp[0] != 0 || rp[n] != nnz))
        bad = true;
    for (uint64_t k = tid; k < nnz; k += stride)
        if (ci[k] >= n)
            bad = true;
    if (bad)
        set_status(res, kErrArg, 200);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        mx = max(mx, __shfl_xor_sync(kFull, mx, o));
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0)
        s_max[w] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t m = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i)
            m = max(m, s_max[i]);
        atomicMax(&res->maxdeg, m);
    }
}

__global__ void __launch_bounds__(256) k_validate(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                                                  uint32_t n, uint32_t nnz, DevResult* res)
{
    validate_one(rp, ci, n, nnz, res, (uint64_t)blockIdx.x * blockDim.x + threadIdx.x,
                 (uint64_t)gridDim.x * blockDim.x);
}


template <int B, int EMAX>
__global__ void __launch_bounds__(B, 1) k_reorder_team(MatrixView M, Options opt, GridSync* gs,
                                                        unsigned long long* agg)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    auto& s = *reinterpret_cast<Smem<B, EMAX>*>(smem_raw);
    if (skip_matrix<EMAX>(M, blockIdx.x == 0 && threadIdx.x == 0))
        return;
    Team team;
    team.gs = gridDim.x > 1 ? gs : nullptr;
    team.flags = reinterpret_cast<unsigned int*>(agg + 2 * gridDim.x);
    team.size = gridDim.x;
    team.rank = blockIdx.x;
    team.expected = gridDim.x + opt.phantom;
    team.mode = opt.barrier;
    team.target = 0;
    team.epoch = 0;
    team.wait_ns = opt.wait_ns;
    team.res = M.res;
    bind_group<B>(team, s);
    reorder_matrix<B, EMAX>(s, M, team, agg, opt);
}

// ---------------------------------------------------------------------------
// Bandwidth of a caller permutation: inverse (with bijection check), then rows.
__global__ void __launch_bounds__(256) k_bw_inverse(const uint32_t* __restrict__ perm, uint32_t n, uint32_t* inv,
                                                    DevResult* res)
{
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = perm[k];
        if (v >= n || atomicCAS(inv + v, kUnvisited, (uint32_t)k) != kUnvisited)
            set_status(res, kErrArg, 300);
    }
}

__global__ void __launch_bounds__(256) k_bw_rows(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                                                 uint32_t n, const uint32_t* __restrict__ inv, DevResult* res)
{
    __shared__ unsigned long long tmp[18];
    unsigned long long bw = 0, bw0 = 0, plo = 0, phi = 0;
    if (read_status(res) == 0) {
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
             i += (uint64_t)gridDim.x * blockDim.x) {
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
            const unsigned long long b1 = me >= mnr ? (unsigned long long)(me - mnr) : 0ull;
            const unsigned long long b2 = mxr >= me ? (unsigned long long)(mxr - me) : 0ull;
            bw = max(bw, max(b1, b2));
            plo += b1;
            phi += b2;
            const uint32_t c0 = ci[a], c1 = ci[e - 1];
            const unsigned long long i0 = i >= c0 ? i - c0 : 0, i1 = c1 >= i ? c1 - i : 0;
            bw0 = max(bw0, max(i0, i1));
        }
    }
    bw = block_reduce_max<256, unsigned long long>(bw, tmp);
    bw0 = block_reduce_max<256, unsigned long long>(bw0, tmp);
    block_reduce_sum2<256>(plo, phi, tmp);
    if (threadIdx.x == 0) {
        atomicMax(&res->bandwidth, bw);
        atomicMax(&res->initial_bw, bw0);
        atomicAdd(&res->profile_lo, plo);
        atomicAdd(&res->profile_hi, phi);
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
namespace {

// The one-matrix team kernel of one shape.
template <int B, int EMAX>
struct Variant {
    static size_t smem() { return sizeof(Smem<B, EMAX>); }
    static cudaError_t prepare()
    {
        static cudaError_t once = cudaFuncSetAttribute(k_reorder_team<B, EMAX>,
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem());
        return once;
    }
    static int team_max_ctas(int sms)
    {
        if (prepare() != cudaSuccess)
            return 0;
        int nb = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_reorder_team<B, EMAX>, B, smem()) != cudaSuccess)
            return 0;
        return nb * sms;
    }
    static cudaError_t team(const MatrixView& M, const Options& opt, GridSync* gs, unsigned long long* agg, int ctas,
                            cudaStream_t st)
    {
        cudaError_t e = prepare();
        if (e != cudaSuccess)
            return e;
        MatrixView m = M;
        Options o = opt;
        void* args[] = {&m, &o, &gs, &agg};
        return cudaLaunchCooperativeKernel((const void*)k_reorder_team<B, EMAX>, dim3(ctas), dim3(B), args, smem(),
                                           st);
    }
};

}  // namespace

const VariantInfo kVariants[kNumVariants] = {
    {128, 512},
    {256, 1024},
    {512, 2048},
};

const PoolInfo kPools[kNumPools] = {
    {512, 2048, 512, 2048},
    {512, 2048, 256, 1024},
    {512, 2048, 128, 512},
    {512, 2048, 64, 256},
    {128, 512, 128, 512},
    {256, 512, 256, 512},
    {256, 1024, 256, 1024},
    {512, 2048, 256, 2048},
};

#define PBRCM_DISPATCH(v, CALL)                     \
    switch (v) {                                    \
    case 0: return Variant<128, 512>::CALL;         \
    case 1: return Variant<256, 1024>::CALL;        \
    case 2: return Variant<512, 2048>::CALL;        \
    default: break;                                 \
    }

// the pool shapes' entry points (pool_p<N>.cu, one translation unit each)
extern const PoolFns kPoolFns0, kPoolFns1, kPoolFns2, kPoolFns3, kPoolFns4, kPoolFns5, kPoolFns6, kPoolFns7;
static const PoolFns* const kPoolTable[kNumPools] = {&kPoolFns0, &kPoolFns1, &kPoolFns2, &kPoolFns3,
                                                     &kPoolFns4, &kPoolFns5, &kPoolFns6, &kPoolFns7};

bool batch_pool_ok(int p)
{
    return p >= 0 && p < kNumPools && p != 4;
}

bool session_pool_ok(int p)
{
    return p >= 0 && p < kNumPools && kPools[p].block == kPools[p].group;
}

size_t variant_smem(int v)
{
    switch (v) {
    case 0: return sizeof(Smem<128, 512>);
    case 1: return sizeof(Smem<256, 1024>);
    case 2: return sizeof(Smem<512, 2048>);
    default: return 0;
    }
}

int team_max_ctas(int v, int sms)
{
    PBRCM_DISPATCH(v, team_max_ctas(sms));
    return 0;
}

int batch_max_ctas(int p, int sms)
{
    return p >= 0 && p < kNumPools ? kPoolTable[p]->batch_max_ctas(sms) : 0;
}

int solo_max_ctas(int p, int sms)
{
    return p >= 0 && p < kNumPools ? kPoolTable[p]->solo_max_ctas(sms) : 0;
}

cudaError_t launch_solo(int p, const BatchJob* jobs, const BatchSlot* slots, uint32_t nslots, uint32_t* counter,
                        const Options& opt, int ctas, cudaStream_t st)
{
    if (p < 0 || p >= kNumPools)
        return cudaErrorInvalidValue;
    return kPoolTable[p]->solo(jobs, slots, nslots, counter, opt, ctas, st);
}

cudaError_t launch_team(int v, const MatrixView& M, const Options& opt, GridSync* gs, unsigned long long* agg,
                        int ctas, cudaStream_t st)
{
    PBRCM_DISPATCH(v, team(M, opt, gs, agg, ctas, st));
    return cudaErrorInvalidValue;
}

cudaError_t launch_batch(int p, const BatchJob* jobs, const BatchSlot* slots, uint32_t nslots, uint32_t* counter,
                         const Options& opt, int ctas, bool cooperative, cudaStream_t st)
{
    if (p < 0 || p >= kNumPools)
        return cudaErrorInvalidValue;
    return kPoolTable[p]->batch(jobs, slots, nslots, counter, opt, ctas, cooperative, st);
}

int cluster_max_active(int p, int csize)
{
    return p >= 0 && p < kNumPools ? kPoolTable[p]->cluster_max_active(csize) : 0;
}

cudaError_t launch_cluster(int p, const BatchJob* jobs, uint32_t nbig, const BatchSlot* slots, uint32_t nslots,
                           uint32_t* counters, const Options& copt, const Options& opt, int csize, int nclusters,
                           cudaStream_t st)
{
    if (p < 0 || p >= kNumPools)
        return cudaErrorInvalidValue;
    return kPoolTable[p]->cluster(jobs, nbig, slots, nslots, counters, copt, opt, csize, nclusters, st);
}

cudaError_t launch_validate(const uint32_t* rp, const uint32_t* ci, uint32_t n, uint32_t nnz, DevResult* res,
                            int sms, cudaStream_t st)
{
    uint64_t work = (uint64_t)n + nnz;
    int blocks = (int)std::min<uint64_t>((work + 255) / 256, (uint64_t)sms * 8);
    if (blocks < 1)
        blocks = 1;
    k_validate<<<blocks, 256, 0, st>>>(rp, ci, n, nnz, res);
    return cudaGetLastError();
}


void launch_perm_inverse(const uint32_t* perm, uint32_t n, uint32_t* inv, DevResult* res, int blocks,
                         cudaStream_t st)
{
    k_bw_inverse<<<blocks, 256, 0, st>>>(perm, n, inv, res);
}

cudaError_t launch_bw_rows(const uint32_t* rp, const uint32_t* ci, uint32_t n, const uint32_t* inv, DevResult* res,
                           int sms, cudaStream_t st)
{
    int blocks = (int)std::min<uint64_t>(((uint64_t)n + 255) / 256, (uint64_t)sms * 8);
    if (blocks < 1)
        blocks = 1;
    k_bw_rows<<<blocks, 256, 0, st>>>(rp, ci, n, inv, res);
    return cudaGetLastError();
}

cudaError_t launch_bandwidth(const uint32_t* rp, const uint32_t* ci, uint32_t n, const uint32_t* perm, uint32_t* inv,
                             DevResult* res, int sms, cudaStream_t st)
{
    int blocks = (int)std::min<uint64_t>(((uint64_t)n + 255) / 256, (uint64_t)sms * 8);
    if (blocks < 1)
        blocks = 1;
    cudaError_t e = cudaMemsetAsync(inv, 0xFF, sizeof(uint32_t) * (size_t)n, st);
    if (e != cudaSuccess)
        return e;
    k_bw_inverse<<<blocks, 256, 0, st>>>(perm, n, inv, res);
    k_bw_rows<<<blocks, 256, 0, st>>>(rp, ci, n, inv, res);
    return cudaGetLastError();
}

}  // namespace pbrcm
