// noalloc.cu -- pbrcm_reorder_device_noalloc: one full reorder of a
// device-resident matrix that allocates no memory at all.
//
// Why: some callers cannot call cudaMalloc while they run -- for example a
// host application whose device memory is owned by its own pool (a
// framework's caching allocator, or a fixed budget reserved at start-up), or
// code that must not let an allocation synchronise the device in the middle
// of its work.  For them this entry point keeps every piece of scratch the
// engine needs (node table, queue records, barrier words, result) in one
// file-scope device array, reserved when the library is loaded and held by
// every GPU that loads it until the process exits.  The caller still passes
// the CSR and the output buffer, both on the device.
//
// Limits: at most kNoAllocMaxNodes nodes, and no row longer than the team
// kernel's chunk (kNoAllocMaxValence); larger inputs are rejected with
// PBRCM_ERR_ARG before anything runs.
//
// Sharing: every call on a device uses the same array and leaves its
// contents behind; the words that must start at zero are cleared at the start
// of each call.  Calls that overlap on the GPU (two streams, or two host
// threads) race on the array, so callers must serialise them.
//
// Set-up: the first call on a device, with that device current, looks up the
// array's device address (cudaGetSymbolAddress; in host code the array's
// name is only a host-side stand-in) and the launch shape; that first call
// should come before any stream capture.  The looked-up address belongs to
// the device's current context: after a cudaDeviceReset the process must not
// call this entry point again.
//
// Engine: the one-matrix team kernel without the parts that need more
// scratch -- no speculative final pass beside the start search (second
// queue-record array), no staging of multi-chunk levels (2 nnz records) and
// no hub path (rows over kNoAllocMaxValence are refused) -- so it is slower
// than pbrcm_reorder_device on matrices with wide levels; same result.
// result->device_ms is the reorder kernel's time from the engine's own
// %globaltimer stamps.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/pbrcm.h"
#include "context.h"
#include "engine.cuh"
#include "kernels.h"
#include "types.h"

namespace pbrcm {
namespace {

constexpr uint32_t kNoAllocMaxNodes = 1u << 20;
constexpr int kNoAllocB = 256;     // team kernel shape (threads per CTA)
constexpr int kNoAllocEmax = 1024; // edges per chunk; also the longest row accepted
constexpr uint32_t kNoAllocMaxValence = kNoAllocEmax;
constexpr int kNoAllocMaxCtas = 1024;

// [DevResult | GridSync | team words | node table | queue records]
constexpr size_t kOffRes = 0;
constexpr size_t kOffGs = 256;
constexpr size_t kOffWords = kOffGs + 256;
constexpr size_t kWordsBytes = 16 * (size_t)kNoAllocMaxCtas + 4 * ((size_t)kNoAllocMaxCtas + 8);
constexpr size_t kOffNode = (kOffWords + kWordsBytes + 255) & ~(size_t)255;
constexpr size_t kOffRec = kOffNode + 16 * (size_t)kNoAllocMaxNodes;
constexpr size_t kScratchBytes = kOffRec + 16 * (size_t)kNoAllocMaxNodes;

static_assert(sizeof(DevResult) <= kOffGs, "DevResult overlaps the GridSync words");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// The team kernel of kernels.cu, restated for this file's launch: same engine,
// its scratch pointers all inside g_noalloc_scratch.
__global__ void __launch_bounds__(kNoAllocB, 1) k_reorder_team_noalloc(MatrixView M, Options opt, GridSync* gs,
                                                                      unsigned long long* words)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    auto& s = *reinterpret_cast<Smem<kNoAllocB, kNoAllocEmax>*>(smem_raw);
    if (read_status(M.res) != 0)
        return;
    if (M.res->maxdeg > kNoAllocMaxValence) {
        if (blockIdx.x == 0 && threadIdx.x == 0)
            set_status(M.res, kErrArg, 400);
        return;
    }
    Team team;
    team.gs = gridDim.x > 1 ? gs : nullptr;
    team.flags = reinterpret_cast<unsigned int*>(words + 2 * gridDim.x);
    team.size = gridDim.x;
    team.rank = blockIdx.x;
    team.expected = gridDim.x + opt.phantom;
    team.mode = 0;
    team.target = 0;
    team.epoch = 0;
    team.wait_ns = opt.wait_ns;
    team.res = M.res;
    bind_group<kNoAllocB>(team, s);
    reorder_matrix<kNoAllocB, kNoAllocEmax>(s, M, team, words, opt);
}

struct DeviceSetup {
    bool ready = false;
    int32_t rc = PBRCM_OK;
    unsigned char* base = nullptr;  // device address of g_noalloc_scratch
    int sms = 0;
    int ctas = 0;
    int max_smem = 0;  // dynamic shared memory the shared-memory engine may take
};

std::mutex g_setup_mu;
DeviceSetup g_setup[64];

// Once per device, with that device current.  A set-up that fails is not
// kept: the next call tries again.
int32_t setup_device(int dev, DeviceSetup*& out)
{
    if (dev < 0 || dev >= 64)
        return PBRCM_ERR_ARG;
    std::lock_guard<std::mutex> lk(g_setup_mu);
    DeviceSetup& d = g_setup[dev];
    if (!d.ready) {
        d.rc = PBRCM_OK;
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) {
            d.rc = PBRCM_ERR_CUDA;
        } else {
            d.base = static_cast<unsigned char*>(p);
            const size_t smem = sizeof(Smem<kNoAllocB, kNoAllocEmax>);
            int nb = 0, coop = 0;
            if (cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
                cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop ||
                cudaFuncSetAttribute(k_reorder_team_noalloc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem) != cudaSuccess ||
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_reorder_team_noalloc, kNoAllocB, smem) !=
                    cudaSuccess ||
                nb < 1) {
                d.rc = PBRCM_ERR_CUDA;
            } else {
                d.ctas = std::min(std::min(nb * d.sms, d.sms), kNoAllocMaxCtas);
                int optin = 0;
                if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess)
                    d.max_smem = optin - 2048;  // room for its static shared memory
            }
        }
        if (d.rc != PBRCM_OK)
            cudaGetLastError();  // clear the failed call's error for the caller
        d.ready = d.rc == PBRCM_OK;
    }
    out = &d;
    return d.rc;
}

}  // namespace
}  // namespace pbrcm

using namespace pbrcm;

extern "C" int32_t pbrcm_reorder_device_noalloc(const uint32_t* d_row_ptr, const uint32_t* d_col_idx, uint32_t n,
                                                uint64_t nnz, const pbrcm_options* opts, uint32_t* d_perm_out,
                                                pbrcm_result* result, void* stream)
{
    const auto t0 = std::chrono::steady_clock::now();
    if (!d_row_ptr || (!d_col_idx && nnz) || !d_perm_out || n == 0 || nnz > kMaxNnz)
        return PBRCM_ERR_ARG;
    if (n > kNoAllocMaxNodes)
        return PBRCM_ERR_ARG;  // beyond the reserved scratch: at most 2^20 nodes
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
        return PBRCM_ERR_CUDA;
    DeviceSetup* d = nullptr;
    int32_t rc = setup_device(dev, d);
    if (rc != PBRCM_OK)
        return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned char* S = d->base;
    DevResult* res = reinterpret_cast<DevResult*>(S + kOffRes);
    GridSync* gs = reinterpret_cast<GridSync*>(S + kOffGs);
    unsigned long long* words = reinterpret_cast<unsigned long long*>(S + kOffWords);
    // the words that must start at zero: result, barrier state, team words
    if (cudaMemsetAsync(S, 0, kOffWords + team_words_bytes(d->ctas), st) != cudaSuccess)
        return PBRCM_ERR_CUDA;
    MatrixView M{};
    M.rp = d_row_ptr;
    M.ci = d_col_idx;
    M.n = n;
    M.nnz = (uint32_t)nnz;
    M.node = reinterpret_cast<NodeEntry*>(S + kOffNode);
    M.rec = reinterpret_cast<PosRec*>(S + kOffRec);
    M.perm = d_perm_out;
    M.hub = nullptr;
    M.res = res;
    Options opt = make_options(opts, kModeFull);
    // a matrix that fits one CTA's shared memory: the shared-memory engine,
    // which needs no scratch beyond the result words (it checks the CSR
    // itself); a row longer than its chunks goes on to the team below
    const int rg = resident_default_group(n, nnz);
    if (opt.phantom == 0 && d->max_smem > 0 && resident_smem(rg, n, (uint32_t)nnz, false) <= (size_t)d->max_smem) {
        DevResult h;
        if (cudaMemsetAsync(res, 0, sizeof(DevResult), st) != cudaSuccess ||
            launch_resident(rg, d_row_ptr, d_col_idx, n, (uint32_t)nnz, d_perm_out, res, opt, d->max_smem, st) !=
                cudaSuccess ||
            cudaMemcpyAsync(&h, res, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return PBRCM_ERR_CUDA;
        if (h.status != kNeedTeam) {
            h.engine = 2;
            fill_result(h, opt, result);
            if (result) {
                result->device_ms = h.t_end > h.t_begin ? (float)((h.t_end - h.t_begin) * 1e-6) : 0.f;
                result->total_ms =
                    std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
            }
            return map_status(h.status);
        }
        if (cudaMemsetAsync(S, 0, kOffWords + team_words_bytes(d->ctas), st) != cudaSuccess)
            return PBRCM_ERR_CUDA;
    }
    opt.solo_parents = 2 * kNoAllocB;
    opt.solo_edges = 2 * kNoAllocEmax;
    opt.barrier = 0;
    if (launch_validate(d_row_ptr, d_col_idx, n, (uint32_t)nnz, res, d->sms, st) != cudaSuccess)
        return PBRCM_ERR_CUDA;
    void* args[] = {&M, &opt, &gs, &words};
    if (cudaLaunchCooperativeKernel((const void*)k_reorder_team_noalloc, dim3(d->ctas), dim3(kNoAllocB), args,
                                    sizeof(Smem<kNoAllocB, kNoAllocEmax>), st) != cudaSuccess)
        return PBRCM_ERR_CUDA;
    DevResult h;
    if (cudaMemcpyAsync(&h, res, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return PBRCM_ERR_CUDA;
    fill_result(h, opt, result);
    if (result) {
        // the engine's own %globaltimer stamps (no event to create)
        result->device_ms = h.t_end > h.t_begin ? (float)((h.t_end - h.t_begin) * 1e-6) : 0.f;
        result->total_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return map_status(h.status);
}
