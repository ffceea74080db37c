// batch.cpp -- many independent matrices in one persistent launch
// (pbrcm_reorder_batch / pbrcm_reorder_batch_device).
//
// Layout: one device arena per call holds, per matrix, its CSR (host-input
// form only), claim[n], rec[n] and perm[n], each 16-byte aligned.  A job
// table of MatrixView descriptors, sorted by nnz descending so that the
// biggest matrices start first, drives k_reorder_batch: every CTA takes the
// next job from an atomic counter and runs the whole reorder of that matrix
// (start search, CM pass, reverse, bandwidth) with a one-CTA team.  Matrices
// above the team cutoff run first, one cooperative team launch each.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <numeric>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/pbrcm.h"
#include "context.h"
#include "kernels.h"
#include "types.h"

using namespace pbrcm;

namespace {

inline size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

struct Slot {
    size_t rp, ci, claim, rec, perm;  // arena offsets (rp/ci unused for device input)
};

int env_int(const char* name, int dflt)
{
    const char* v = std::getenv(name);
    return v && *v ? std::atoi(v) : dflt;
}

// Shared driver; `host` selects whether mats[] point to host or device memory.
int32_t run_batch(Context& C, const pbrcm_matrix* mats, uint32_t count, const pbrcm_options* opts,
                  pbrcm_result* results, cudaStream_t st, bool host)
{
    auto t0 = std::chrono::steady_clock::now();
    Options opt = make_options(opts, kModeFull);
    for (uint32_t j = 0; j < count; ++j) {
        const pbrcm_matrix& m = mats[j];
        if (!m.row_ptr || (!m.col_idx && m.nnz) || !m.perm_out || m.n == 0 || m.n == 0xFFFFFFFFu ||
            m.nnz >= 0xFFFFFFFFull)
            return PBRCM_ERR_ARG;
    }
    // arena layout
    std::vector<Slot> slot(count);
    size_t off = 0;
    for (uint32_t j = 0; j < count; ++j) {
        const pbrcm_matrix& m = mats[j];
        if (host) {
            slot[j].rp = off;
            off = align16(off + 4 * ((size_t)m.n + 1));
            slot[j].ci = off;
            off = align16(off + 4 * (size_t)m.nnz);
        }
        slot[j].claim = off;
        off = align16(off + 4 * (size_t)m.n);
        slot[j].rec = off;
        off = align16(off + 16 * (size_t)m.n);
        if (host) {
            slot[j].perm = off;
            off = align16(off + 4 * (size_t)m.n);
        }
    }
    if (off > C.cap_arena) {
        if (C.d_arena)
            cudaFree(C.d_arena);
        C.d_arena = nullptr;
        C.cap_arena = 0;
        if (cudaMalloc(&C.d_arena, off) != cudaSuccess)
            return PBRCM_ERR_OOM;
        C.cap_arena = off;
    }
    if (count > C.cap_jobs) {
        if (C.d_jobs)
            cudaFree(C.d_jobs);
        if (C.d_bres)
            cudaFree(C.d_bres);
        C.d_jobs = nullptr;
        C.d_bres = nullptr;
        C.cap_jobs = 0;
        if (cudaMalloc(&C.d_jobs, sizeof(MatrixView) * count) != cudaSuccess ||
            cudaMalloc(&C.d_bres, sizeof(DevResult) * count) != cudaSuccess)
            return PBRCM_ERR_OOM;
        C.cap_jobs = count;
    }
    if (!C.d_counter) {
        if (cudaMalloc(&C.d_counter, sizeof(uint32_t) * 4) != cudaSuccess)
            return PBRCM_ERR_OOM;
        C.cap_counter = 4;
    }
    // copies in
    unsigned char* A = C.d_arena;
    if (host) {
        for (uint32_t j = 0; j < count; ++j) {
            const pbrcm_matrix& m = mats[j];
            if (cudaMemcpyAsync(A + slot[j].rp, m.row_ptr, 4 * ((size_t)m.n + 1), cudaMemcpyHostToDevice, st) !=
                    cudaSuccess ||
                (m.nnz && cudaMemcpyAsync(A + slot[j].ci, m.col_idx, 4 * (size_t)m.nnz, cudaMemcpyHostToDevice,
                                          st) != cudaSuccess))
                return PBRCM_ERR_CUDA;
        }
    }
    // job table, biggest first; the cutoff sends very large matrices to teams
    const uint64_t cutoff = (uint64_t)env_int("PBRCM_BATCH_TEAM_CUTOFF_N", 1 << 20);
    std::vector<uint32_t> order(count);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t b) { return mats[a].nnz > mats[b].nnz; });
    std::vector<MatrixView> jobs(count);
    for (uint32_t q = 0; q < count; ++q) {
        const uint32_t j = order[q];
        const pbrcm_matrix& m = mats[j];
        MatrixView M{};
        M.rp = host ? reinterpret_cast<const uint32_t*>(A + slot[j].rp) : m.row_ptr;
        M.ci = host ? reinterpret_cast<const uint32_t*>(A + slot[j].ci) : m.col_idx;
        M.n = m.n;
        M.nnz = (uint32_t)m.nnz;
        M.claim = reinterpret_cast<uint32_t*>(A + slot[j].claim);
        M.rec = reinterpret_cast<PosRec*>(A + slot[j].rec);
        M.perm = host ? reinterpret_cast<uint32_t*>(A + slot[j].perm) : m.perm_out;
        M.hub = nullptr;
        M.res = C.d_bres + q;
        jobs[q] = M;
    }
    uint32_t nteam = 0;
    while (nteam < count && mats[order[nteam]].n > cutoff)
        ++nteam;
    if (cudaMemcpyAsync(C.d_jobs, jobs.data(), sizeof(MatrixView) * count, cudaMemcpyHostToDevice, st) !=
            cudaSuccess ||
        cudaMemsetAsync(C.d_bres, 0, sizeof(DevResult) * count, st) != cudaSuccess ||
        cudaMemsetAsync(C.d_counter, 0, sizeof(uint32_t), st) != cudaSuccess)
        return PBRCM_ERR_CUDA;
    if (launch_validate_batch(C.d_jobs, count, C.sms, st) != cudaSuccess)
        return PBRCM_ERR_CUDA;
    cudaEventRecord(C.ev0, st);
    // big ones: one team launch each
    for (uint32_t q = 0; q < nteam; ++q) {
        if (cudaMemsetAsync(C.d_gs, 0, sizeof(GridSync), st) != cudaSuccess ||
            launch_team(C.team_variant, jobs[q], opt, C.d_gs, C.d_agg, C.team_ctas, st) != cudaSuccess)
            return PBRCM_ERR_CUDA;
    }
    if (nteam < count) {
        // the counter starts at nteam: those jobs are done already
        uint32_t start = nteam;
        if (cudaMemcpyAsync(C.d_counter, &start, sizeof(uint32_t), cudaMemcpyHostToDevice, st) != cudaSuccess)
            return PBRCM_ERR_CUDA;
        int ctas = std::min<int>(batch_max_ctas(C.batch_variant, C.sms), (int)(count - nteam));
        if (ctas < 1)
            ctas = 1;
        if (launch_batch(C.batch_variant, C.d_jobs, count, C.d_counter, opt, ctas, st) != cudaSuccess)
            return PBRCM_ERR_CUDA;
    }
    cudaEventRecord(C.ev1, st);
    std::vector<DevResult> res(count);
    if (cudaMemcpyAsync(res.data(), C.d_bres, sizeof(DevResult) * count, cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return PBRCM_ERR_CUDA;
    float dms = 0.f;
    cudaEventElapsedTime(&dms, C.ev0, C.ev1);
    // matrices with a hub row rerun on the team path with hub scratch
    for (uint32_t q = 0; q < count; ++q) {
        if (res[q].status != kNeedHub)
            continue;
        const MatrixView& M = jobs[q];
        if (!C.ensure_hub(M.nnz))
            return PBRCM_ERR_OOM;
        MatrixView H = M;
        H.hub = C.d_hub;
        if (cudaMemsetAsync(M.res, 0, sizeof(DevResult), st) != cudaSuccess ||
            cudaMemsetAsync(C.d_gs, 0, sizeof(GridSync), st) != cudaSuccess ||
            launch_validate(M.rp, M.ci, M.n, M.nnz, M.res, C.sms, st) != cudaSuccess ||
            launch_team(C.team_variant, H, opt, C.d_gs, C.d_agg, C.team_ctas, st) != cudaSuccess ||
            cudaMemcpyAsync(&res[q], M.res, sizeof(DevResult), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return PBRCM_ERR_CUDA;
    }
    int32_t worst = PBRCM_OK;
    for (uint32_t q = 0; q < count; ++q) {
        const uint32_t j = order[q];
        if (host && res[q].status == kOk) {
            if (cudaMemcpyAsync(mats[j].perm_out, jobs[q].perm, 4 * (size_t)mats[j].n, cudaMemcpyDeviceToHost,
                                st) != cudaSuccess)
                return PBRCM_ERR_CUDA;
        }
        if (results) {
            fill_result(res[q], opt, &results[j]);
            results[j].device_ms = dms;
        }
        if (res[q].status != kOk && worst == PBRCM_OK)
            worst = map_status(res[q].status);
    }
    if (cudaStreamSynchronize(st) != cudaSuccess)
        return PBRCM_ERR_CUDA;
    if (results) {
        float tms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
        for (uint32_t j = 0; j < count; ++j)
            results[j].total_ms = tms;
    }
    return worst;
}

}  // namespace

#define PBRCM_CTX2(ctx)                                      \
    if (!ctx) {                                              \
        int32_t rc_ = pbrcm_context_create(-1, &ctx_local); \
        if (rc_ != PBRCM_OK)                                 \
            return rc_;                                      \
        ctx = ctx_local;                                     \
    }

extern "C" {

int32_t pbrcm_reorder_batch(pbrcm_context* ctx, const pbrcm_matrix* mats, uint32_t count, const pbrcm_options* opts,
                            pbrcm_result* results)
{
    if (!mats && count)
        return PBRCM_ERR_ARG;
    if (count == 0)
        return PBRCM_OK;
    pbrcm_context* ctx_local = nullptr;
    PBRCM_CTX2(ctx);
    int32_t rc;
    {
        std::lock_guard<std::mutex> lk(ctx->ctx.mu);
        cudaSetDevice(ctx->ctx.device);
        rc = run_batch(ctx->ctx, mats, count, opts, results, ctx->ctx.stream, true);
    }
    if (ctx_local)
        pbrcm_context_destroy(ctx_local);
    return rc;
}

int32_t pbrcm_reorder_batch_device(pbrcm_context* ctx, const pbrcm_matrix* mats, uint32_t count,
                                   const pbrcm_options* opts, pbrcm_result* results, void* stream)
{
    if (!mats && count)
        return PBRCM_ERR_ARG;
    if (count == 0)
        return PBRCM_OK;
    pbrcm_context* ctx_local = nullptr;
    PBRCM_CTX2(ctx);
    int32_t rc;
    {
        std::lock_guard<std::mutex> lk(ctx->ctx.mu);
        cudaSetDevice(ctx->ctx.device);
        rc = run_batch(ctx->ctx, mats, count, opts, results,
                       stream ? (cudaStream_t)stream : ctx->ctx.stream, false);
    }
    if (ctx_local)
        pbrcm_context_destroy(ctx_local);
    return rc;
}

}  // extern "C"
