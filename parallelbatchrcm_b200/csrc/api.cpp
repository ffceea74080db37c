// api.cpp -- C ABI of libpbrcm (include/pbrcm.h): contexts, single-matrix and
// batched reorders, start search and bandwidth.  Host C++ over the CUDA
// runtime; all device work is in kernels.cu.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/pbrcm.h"
#include "context.h"
#include "kernels.h"
#include "types.h"

using namespace pbrcm;

namespace pbrcm {

const char* kVersion = "pbrcm-b200 0.1 (sm_100a)";

// ---------------------------------------------------------------------------
int32_t map_status(uint32_t s)
{
    switch (s) {
    case kOk: return PBRCM_OK;
    case kErrArg: return PBRCM_ERR_ARG;
    case kErrDisconnected: return PBRCM_ERR_DISCONNECTED;
    case kErrTimeout: return PBRCM_ERR_TIMEOUT;
    case kErrCheck: return PBRCM_ERR_CHECK;
    default: return PBRCM_ERR_CHECK;
    }
}

Options make_options(const pbrcm_options* o, uint32_t mode)
{
    pbrcm_options d;
    pbrcm_default_options(&d);
    if (!o)
        o = &d;
    Options opt{};
    opt.start = o->start_node;
    opt.reverse = o->reverse ? 1u : 0u;
    opt.want_bw = o->want_bandwidth ? 1u : 0u;
    opt.outnodes = o->peripheral_nodes ? o->peripheral_nodes : 32u;
    opt.wait_ns = (unsigned long long)(o->wait_limit_ms ? o->wait_limit_ms : 2000u) * 1000000ull;
    opt.phantom = (o->debug_flags & PBRCM_DEBUG_PHANTOM_CTA) ? 1u : 0u;
    opt.mode = mode;
    opt.solo_edges = 0;
    opt.solo_parents = 0;
    return opt;
}

void apply_team_shape(const Context& C, Options& opt)
{
    opt.solo_edges = C.solo_edges;
    opt.solo_parents = C.solo_parents;
    opt.barrier = C.barrier;
    opt.spec_from = C.spec_from;
}

void fill_result(const DevResult& r, const Options& opt, pbrcm_result* out)
{
    if (!out)
        return;
    out->status = map_status(r.status);
    out->start_node = r.start;
    out->peripheral_passes = r.passes;
    out->eccentricity = r.ecc;
    out->levels = r.levels;
    out->placed = r.placed;
    out->engine = r.engine;
    if (opt.want_bw && r.status == kOk && opt.mode == kModeFull) {
        out->bandwidth = (int64_t)r.bandwidth;
        out->initial_bandwidth = (int64_t)r.initial_bw;
        out->profile = opt.reverse ? r.profile_hi : r.profile_lo;
    } else {
        out->bandwidth = -1;
        out->initial_bandwidth = -1;
        out->profile = 0;
    }
}

// ---------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------
static int env_int(const char* name, int dflt)
{
    const char* v = std::getenv(name);
    return v && *v ? std::atoi(v) : dflt;
}

int32_t Context::init(int dev)
{
    if (dev < 0) {
        if (cudaGetDevice(&dev) != cudaSuccess)
            return PBRCM_ERR_CUDA;
    }
    device = dev;
    if (cudaSetDevice(dev) != cudaSuccess)
        return PBRCM_ERR_CUDA;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess)
        return PBRCM_ERR_CUDA;
    sms = prop.multiProcessorCount;
    if (!prop.cooperativeLaunch)
        return PBRCM_ERR_CUDA;
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess)
        return PBRCM_ERR_CUDA;
    if (cudaEventCreate(&ev0) != cudaSuccess || cudaEventCreate(&ev1) != cudaSuccess)
        return PBRCM_ERR_CUDA;
    // host-buffer batches copy their inputs on a second stream while the
    // batch kernel already runs
    if (cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming) != cudaSuccess)
        return PBRCM_ERR_CUDA;
    if (cudaMallocHost(&h_one, sizeof(uint32_t)) != cudaSuccess)
        return PBRCM_ERR_OOM;
    *h_one = 1u;
    if (cudaMalloc(&d_res, sizeof(DevResult)) != cudaSuccess || cudaMalloc(&d_gs, kTeamParts * sizeof(GridSync)) != cudaSuccess)
        return PBRCM_ERR_OOM;
    if (cudaMallocHost(&h_res, sizeof(DevResult)) != cudaSuccess ||
        cudaMallocHost(&h_aux, 64) != cudaSuccess)
        return PBRCM_ERR_OOM;
    // team shape: variant and CTA count (PBRCM_TEAM_VARIANT / PBRCM_TEAM_CTAS override)
    team_variant = env_int("PBRCM_TEAM_VARIANT", 1);
    if (team_variant < 0 || team_variant >= kNumVariants)
        team_variant = 1;
    int maxc = team_max_ctas(team_variant, sms);
    if (maxc <= 0)
        return PBRCM_ERR_CUDA;
    team_maxc = maxc;
    team_ctas = env_int("PBRCM_TEAM_CTAS", 0);
    if (team_ctas <= 0 || team_ctas > maxc)
        team_ctas = std::min(maxc, sms);
    // levels of one chunk run on CTA 0 alone (measured against 2 chunks: the
    // 128^3 grid 10.55 -> 10.36 ms, a 1000^2 grid 58.9 -> 50.4 ms, a 1M-node
    // RGG 6.97 -> 6.87 ms; smaller bounds are slower again)
    solo_parents = (uint32_t)env_int("PBRCM_SOLO_PARENTS", kVariants[team_variant].block);
    solo_edges = (uint32_t)env_int("PBRCM_SOLO_EDGES", kVariants[team_variant].emax);
    barrier = (uint32_t)env_int("PBRCM_BARRIER", 0) ? 1u : 0u;
    spec_from = (uint32_t)std::max(0, env_int("PBRCM_SPEC_FROM", 3));
    // wide, shallow graphs: PBRCM_WIDE_DIV (0: never), PBRCM_WIDE_MIN,
    // PBRCM_ENGINE=wide to run the level-synchronous engine first, =team for
    // the team engine alone
    wide_div = (uint32_t)std::max(0, env_int("PBRCM_WIDE_DIV", 16));
    wide_min = (uint32_t)std::max(1, env_int("PBRCM_WIDE_MIN", 1 << 18));
    if (const char* e = std::getenv("PBRCM_ENGINE")) {
        wide_force = std::string(e) == "wide";
        team_force = std::string(e) == "team";
    }
    wide_fused = env_int("PBRCM_WIDE_FUSED", 1) != 0;
    wide_batch_pass = env_int("PBRCM_WIDE_BATCH_PASS", 1) != 0;
    wide_ctas = wide_ctas_per_sm() * sms;
    // small matrices: the shared-memory engine (PBRCM_RESIDENT_GROUP: 32,
    // 64, 128 or 256 threads a group, 0 off; unset: by the matrix, see
    // run_single)
    resident_group = env_int("PBRCM_RESIDENT_GROUP", -1);
    if (resident_group != -1 && !resident_group_ok(resident_group))
        resident_group = 0;
    resident_max_smem = (int)prop.sharedMemPerBlockOptin - 2048;  // room for its static shared memory
    // batch / serving shape: built-in defaults (measured on the 4,096-matrix
    // mixed batch on a B200: the solo batch kernel with three 256-thread
    // CTAs per SM, 82 ms; 2 x 256 threads per CTA, 86 ms with the solo
    // kernel and 89-95 ms with the general one; 1 x 512, 102 ms; 2 x 256
    // with 2,048-edge chunks, 109 ms), or a tuning file written by
    // pbrcm_autotune for this device shape and library version
    // (PBRCM_TUNING); a PBRCM_* knob below still overrides a single setting
    pbrcm_tuning tn;
    std::memset(&tn, 0, sizeof(tn));
    tn.batch_pool = 6;
    tn.batch_kernel = 1;
    // no cluster teams by default: with the solo engine one group takes even
    // the biggest matrices of the mixed batch faster than a cluster team of
    // the engine does (100 ms against 106 ms for the 4,096-matrix batch)
    tn.cluster_size = 1;
    tn.cluster_max = 16;
    tn.cluster_nnz = 1u << 18;
    tn.session_cutoff_n = 1u << 18;
    tn.session_pool = 0;
    tn.session_team_nnz = 1u << 20;
    tn.session_cluster_max = 16;
    if (const char* tp = std::getenv("PBRCM_TUNING")) {
        if (load_tuning_file(tp, sms, &tn))
            tuned = 1;
    }
    batch_pool = env_int("PBRCM_BATCH_POOL", (int)tn.batch_pool);
    if (!batch_pool_ok(batch_pool))
        batch_pool = 6;
    session_cutoff_n = (uint32_t)std::max(1, env_int("PBRCM_SESSION_CUTOFF_N", (int)tn.session_cutoff_n));
    session_pool = env_int("PBRCM_SESSION_POOL", (int)tn.session_pool);
    if (!session_pool_ok(session_pool))
        session_pool = 0;
    session_team_nnz = (uint32_t)std::max(1, env_int("PBRCM_SESSION_TEAM_NNZ", (int)tn.session_team_nnz));
    session_cluster_max = std::max(0, std::min(16, env_int("PBRCM_SESSION_CLUSTER_MAX", (int)tn.session_cluster_max)));
    solo = env_int("PBRCM_SOLO", 1) != 0;
    batch_solo_kernel = env_int("PBRCM_BATCH_SOLO_KERNEL", (int)tn.batch_kernel) != 0;
    batch_graphs = env_int("PBRCM_BATCH_GRAPHS", 1) != 0;
    if (cudaMalloc(&d_agg, kTeamParts * team_part_bytes(maxc)) != cudaSuccess)
        return PBRCM_ERR_OOM;
    // cluster teams of the batch path (PBRCM_BATCH_CLUSTER* override)
    // measured on the mixed 1,024-matrix batch: pairs for the 16 biggest
    // matrices cut its makespan by ~16 %; larger clusters or more of them
    // cost more CTA-time than the tail they remove
    cluster_size = env_int("PBRCM_BATCH_CLUSTER", (int)tn.cluster_size);
    cluster_nnz = (uint64_t)std::max(1, env_int("PBRCM_BATCH_CLUSTER_NNZ", (int)tn.cluster_nnz));
    cluster_max = env_int("PBRCM_BATCH_CLUSTERS", (int)tn.cluster_max);
    cluster_solo_parents = (uint32_t)env_int("PBRCM_CLUSTER_SOLO_PARENTS", kPools[batch_pool].block);
    cluster_solo_edges = (uint32_t)env_int("PBRCM_CLUSTER_SOLO_EDGES", kPools[batch_pool].emax);
    return PBRCM_OK;
}

Context::~Context()
{
    if (device >= 0)
        cudaSetDevice(device);
    if (stream)
        cudaStreamSynchronize(stream);
    for (void* p : {(void*)d_wide, (void*)d_pw, (void*)d_rp, (void*)d_ci, (void*)d_node, (void*)d_perm, (void*)d_rec, (void*)d_rec2, (void*)d_stage, (void*)d_hub,
                    (void*)d_res, (void*)d_gs, (void*)d_agg, (void*)d_jobs, (void*)d_slots, (void*)d_counter, (void*)d_bres,
                    (void*)d_arena})
        if (p)
            cudaFree(p);
    if (bgraph.exec)
        cudaGraphExecDestroy(bgraph.exec);
    for (void* p : {(void*)h_jobs, (void*)h_slots, (void*)h_bres, (void*)bgraph.h_jobs, (void*)bgraph.h_slots})
        if (p)
            cudaFreeHost(p);
    if (d_ready)
        cudaFree(d_ready);
    if (h_one)
        cudaFreeHost(h_one);
    if (ev_fork)
        cudaEventDestroy(ev_fork);
    if (ev_join)
        cudaEventDestroy(ev_join);
    if (copy_stream) {
        cudaStreamSynchronize(copy_stream);
        cudaStreamDestroy(copy_stream);
    }
    if (h_res)
        cudaFreeHost(h_res);
    if (h_aux)
        cudaFreeHost(h_aux);
    if (ev0)
        cudaEventDestroy(ev0);
    if (ev1)
        cudaEventDestroy(ev1);
    if (stream)
        cudaStreamDestroy(stream);
}

template <typename T>
static bool grow(T*& p, size_t& cap, size_t need)
{
    if (need <= cap && p)
        return true;
    if (p)
        cudaFree(p);
    p = nullptr;
    cap = 0;
    size_t want = std::max(need, (size_t)1);
    if (cudaMalloc(&p, sizeof(T) * want) != cudaSuccess) {
        p = nullptr;
        return false;
    }
    cap = want;
    return true;
}

bool Context::ensure_single(uint32_t n, uint64_t nnz, bool inputs)
{
    if (inputs && (!grow(d_rp, cap_rp, (size_t)n + 1) || !grow(d_ci, cap_ci, (size_t)nnz)))
        return false;
    return grow(d_node, cap_node, n) && grow(d_rec, cap_rec, n) && grow(d_rec2, cap_rec2, n) &&
           grow(d_stage, cap_stage, 2 * std::max<uint64_t>(nnz, 1)) && grow(d_perm, cap_perm, n);
}

bool Context::ensure_hub(uint64_t nnz) { return grow(d_hub, cap_hub, 4 * (size_t)std::max<uint64_t>(nnz, 1)); }

static size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

// The level-synchronous engine: level steps in batches, one read of the
// state between batches.  While no pass has finished the batches grow 8, 16,
// 32, ...; after that a batch is the rest of a pass as long as the last one
// (the final pass, from the same start as the last search pass, has exactly
// its levels).  A matrix still running after kWideMaxSteps steps (its levels
// are many, not wide) goes back to the team.
static constexpr int kWideMaxSteps = 1024;

bool Context::run_wide(const MatrixView& M, const Options& opt, cudaStream_t st)
{
    const size_t o_tot = 256, o_inv = o_tot + al256(8 * (size_t)wide_ctas);
    if (!grow(d_wide, cap_wide, o_inv + 4 * (size_t)M.n))
        return false;
    WideState* ws = reinterpret_cast<WideState*>(d_wide);
    unsigned long long* tot = reinterpret_cast<unsigned long long*>(d_wide + o_tot);
    if (cudaMemsetAsync(ws, 0, sizeof(WideState), st) != cudaSuccess ||
        launch_wide_start(M, opt, ws, sms, st) != cudaSuccess)
        return false;
    WideState* hs = reinterpret_cast<WideState*>(h_aux);
    static_assert(sizeof(WideState) <= 64, "the state is read back through the 64-byte pinned words");
    int total = 0, grow_batch = 8;
    bool done = false;
    while (total < kWideMaxSteps) {
        int batch = grow_batch;
        if (wide_batch_pass && total > 0 && hs->prev_levels > 0)
            batch = std::max(2, (int)hs->prev_levels + 1 - (int)hs->L);
        batch = std::min(batch, kWideMaxSteps - total);
        if (launch_wide_steps(M, opt, ws, tot, wide_ctas, batch, wide_fused, st) != cudaSuccess ||
            cudaMemcpyAsync(hs, ws, sizeof(WideState), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return false;
        total += batch;
        grow_batch *= 2;
        if (hs->phase == kWideDone) {
            done = true;
            break;
        }
    }
    if (!done) {
        const uint32_t code = kNeedTeam;
        return cudaMemcpyAsync(&M.res->status, &code, sizeof(code), cudaMemcpyHostToDevice, st) == cudaSuccess &&
               cudaStreamSynchronize(st) == cudaSuccess;
    }
    if (opt.want_bw && opt.mode == kModeFull &&
        launch_wide_bandwidth(M, reinterpret_cast<uint32_t*>(d_wide + o_inv), sms, st) != cudaSuccess)
        return false;
    return true;
}

// Runs start search (+ CM + bandwidth) on device buffers already in place.
// Enqueues on `st` and synchronises.  The team engine runs first; it is
// rerun with hub scratch when a row is longer than its chunks take, and it
// hands a matrix whose first pass meets a level of at least
// max(n / wide_div, wide_min) nodes to the level-synchronous engine (rows
// permitting; that engine hands back the rare matrix it cannot finish).
int32_t Context::run_single(const uint32_t* rp, const uint32_t* ci, uint32_t n, uint64_t nnz, uint32_t* perm,
                            const Options& opt, cudaStream_t st, DevResult* out, float* dev_ms)
{
    // a matrix whose CSR and workspace fit one CTA's shared memory: the
    // shared-memory engine, which checks the CSR itself; a row longer than
    // its chunks sends the matrix on to the engines below
    // (not when an engine is forced, nor under the phantom-CTA test hook,
    // which tests the team's barrier)
    // group size unless set: by the matrix (resident_default_group)
    const int rg = resident_group >= 0 ? resident_group : resident_default_group(n, nnz);
    if (rg > 0 && !wide_force && !team_force && opt.phantom == 0 && n >= 1 &&
        resident_smem(rg, n, (uint32_t)nnz, false) <= (size_t)resident_max_smem) {
        if (cudaMemsetAsync(d_res, 0, sizeof(DevResult), st) != cudaSuccess)
            return PBRCM_ERR_CUDA;
        cudaEventRecord(ev0, st);
        if (launch_resident(rg, rp, ci, n, (uint32_t)nnz, perm, d_res, opt, resident_max_smem, st) !=
            cudaSuccess)
            return PBRCM_ERR_CUDA;
        cudaEventRecord(ev1, st);
        if (cudaMemcpyAsync(h_res, d_res, sizeof(DevResult), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return PBRCM_ERR_CUDA;
        if (h_res->status != kNeedTeam) {
            if (dev_ms)
                cudaEventElapsedTime(dev_ms, ev0, ev1);
            *out = *h_res;
            out->engine = 2;
            return PBRCM_OK;
        }
    }
    bool with_hub = false;
    bool try_wide = wide_ctas > 0 && wide_div != 0 && n > 1 && !team_force;
    bool wide_first = try_wide && wide_force;
    for (int attempt = 0; attempt < 4; ++attempt) {
        MatrixView M{};
        M.rp = rp;
        M.ci = ci;
        M.n = n;
        M.nnz = (uint32_t)nnz;
        M.node = d_node;
        M.rec = d_rec;
        M.rec2 = d_rec2;
        M.stage = d_stage;
        M.perm = perm;
        M.hub = with_hub ? d_hub : nullptr;
        M.res = d_res;
        if (cudaMemsetAsync(d_res, 0, sizeof(DevResult), st) != cudaSuccess ||
            cudaMemsetAsync(d_gs, 0, kTeamParts * sizeof(GridSync), st) != cudaSuccess ||
            cudaMemsetAsync(d_agg, 0, kTeamParts * team_part_bytes(team_ctas), st) != cudaSuccess)
            return PBRCM_ERR_CUDA;
        if (launch_validate(rp, ci, n, (uint32_t)nnz, d_res, sms, st) != cudaSuccess)
            return PBRCM_ERR_CUDA;
        if (attempt == 0)
            cudaEventRecord(ev0, st);  // every attempt counts in the device time
        bool wide_ran = false;
        if (wide_first) {
            // the engine needs every row within one chunk: read the valences
            if (cudaMemcpyAsync(h_res, d_res, sizeof(DevResult), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess)
                return PBRCM_ERR_CUDA;
            if (h_res->status == kOk && h_res->maxdeg <= wide_emax()) {
                if (!run_wide(M, opt, st))
                    return PBRCM_ERR_CUDA;
                wide_ran = true;
            }
        }
        if (!wide_ran) {
            Options o = opt;
            apply_team_shape(*this, o);
            o.wide_at = try_wide ? std::max(n / wide_div, wide_min) : 0u;
            if (launch_team(team_variant, M, o, d_gs, d_agg, team_ctas, st) != cudaSuccess)
                return PBRCM_ERR_CUDA;
        }
        cudaEventRecord(ev1, st);
        if (cudaMemcpyAsync(h_res, d_res, sizeof(DevResult), cudaMemcpyDeviceToHost, st) != cudaSuccess)
            return PBRCM_ERR_CUDA;
        if (cudaStreamSynchronize(st) != cudaSuccess)
            return PBRCM_ERR_CUDA;
        if (dev_ms)
            cudaEventElapsedTime(dev_ms, ev0, ev1);
        *out = *h_res;
        out->engine = wide_ran ? 1u : 0u;
        if (out->status == kNeedHub && !with_hub) {
            if (!ensure_hub(nnz))
                return PBRCM_ERR_OOM;
            with_hub = true;
            continue;
        }
        if (out->status == kNeedWide) {
            // the team met a wide level: the level-synchronous engine, if
            // every row fits its chunks, else the team without the hand-over
            wide_first = out->maxdeg <= wide_emax();
            try_wide = wide_first;
            continue;
        }
        if (out->status == kNeedTeam) {
            wide_first = false;
            try_wide = false;
            continue;
        }
        break;
    }
    // every hand-over sequence ends within the four attempts (hub, then wide
    // or team, then hub again); an internal code still standing means the
    // hand-over logic went round in a circle: a check failure of its own
    // (where 900 + the code's offset), not a CSR check's
    if (out->status == kNeedHub || out->status == kNeedWide || out->status == kNeedTeam) {
        out->where = 900u + (out->status - (uint32_t)kNeedHub);
        out->status = kErrCheck;
    }
    return PBRCM_OK;
}

// inv (n) | scan partials | mid-row list (n) | long-row list | counters
size_t Context::permute_work_bytes(uint32_t n, uint64_t nnz)
{
    return 2 * al256(4 * (size_t)n) + al256(4 * (size_t)scan_partials_count(n)) +
           al256(4 * (size_t)permute_long_cap(n, nnz)) + 256;
}

// B = P A P^T into out_*, after the CSR check on the same stream (the
// permutation kernels bound every access themselves, so they need not wait
// for its verdict); one synchronisation of `st`, two if a row has more than
// 1,024 entries and the long-row scratch has to be allocated first.
int32_t Context::run_permute(const uint32_t* rp, const uint32_t* ci, const void* vals, uint32_t val_bytes, uint32_t n,
                             uint64_t nnz, const uint32_t* perm, uint32_t* out_rp, uint32_t* out_ci, void* out_vals,
                             uint32_t* out_map, unsigned char* work, cudaStream_t st)
{
    size_t o = 0;
    uint32_t* inv = reinterpret_cast<uint32_t*>(work + o);
    o += al256(4 * (size_t)n);
    uint32_t* partials = reinterpret_cast<uint32_t*>(work + o);
    o += al256(4 * (size_t)scan_partials_count(n));
    uint32_t* mids = reinterpret_cast<uint32_t*>(work + o);
    o += al256(4 * (size_t)n);
    uint32_t* longs = reinterpret_cast<uint32_t*>(work + o);
    o += al256(4 * (size_t)permute_long_cap(n, nnz));
    uint32_t* counters = reinterpret_cast<uint32_t*>(work + o);
    const uint32_t cap_long = permute_long_cap(n, nnz);
    uint32_t* scratch = d_hub != nullptr && cap_hub >= 4 * (size_t)std::max<uint64_t>(nnz, 1) ? d_hub : nullptr;
    if (cudaMemsetAsync(d_res, 0, sizeof(DevResult), st) != cudaSuccess ||
        launch_validate(rp, ci, n, (uint32_t)nnz, d_res, sms, st) != cudaSuccess ||
        launch_permute(rp, ci, vals, val_bytes, n, (uint32_t)nnz, perm, inv, out_rp, out_ci, out_vals, out_map,
                       partials, mids, longs, cap_long, counters, scratch, d_res, sms, st) != cudaSuccess ||
        cudaMemcpyAsync(h_res, d_res, sizeof(DevResult), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(h_aux, counters, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return PBRCM_ERR_CUDA;
    if (h_res->status != kOk)
        return map_status(h_res->status);
    if (h_aux[1] > 0 && scratch == nullptr) {
        if (!ensure_hub(nnz))
            return PBRCM_ERR_OOM;
        if (launch_permute_long(rp, ci, vals, val_bytes, n, (uint32_t)nnz, perm, inv, out_rp, out_ci, out_vals,
                                out_map, longs, cap_long, counters, d_hub, d_res, sms, st) != cudaSuccess ||
            cudaMemcpyAsync(h_res, d_res, sizeof(DevResult), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return PBRCM_ERR_CUDA;
    }
    return map_status(h_res->status);
}

// parent (n) | scan partials | counters
size_t Context::connect_work_bytes(uint32_t n)
{
    return al256(4 * (size_t)n) + al256(4 * (size_t)scan_partials_count(n)) + 256;
}

// The loader's connectivity repair into out_* after the CSR check on the same
// stream (the repair kernels clamp every row range themselves); one
// synchronisation of `st`.
int32_t Context::run_connect(const uint32_t* rp, const uint32_t* ci, uint32_t n, uint64_t nnz, uint32_t* out_rp,
                             uint32_t* out_ci, uint64_t cap, uint64_t* nnz_out, uint32_t* links_out,
                             unsigned char* work, cudaStream_t st)
{
    uint32_t* parent = reinterpret_cast<uint32_t*>(work);
    uint32_t* partials = reinterpret_cast<uint32_t*>(work + al256(4 * (size_t)n));
    uint32_t* counters =
        reinterpret_cast<uint32_t*>(work + al256(4 * (size_t)n) + al256(4 * (size_t)scan_partials_count(n)));
    if (cudaMemsetAsync(d_res, 0, sizeof(DevResult), st) != cudaSuccess ||
        launch_validate(rp, ci, n, (uint32_t)nnz, d_res, sms, st) != cudaSuccess ||
        launch_connect(rp, ci, n, (uint32_t)nnz, out_rp, out_ci, cap, parent, partials, counters, sms, st) !=
            cudaSuccess ||
        cudaMemcpyAsync(h_res, d_res, sizeof(DevResult), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(h_aux, counters, 3 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return PBRCM_ERR_CUDA;
    if (h_res->status != kOk)
        return map_status(h_res->status);
    if (h_aux[2] != 0)
        return PBRCM_ERR_ARG;  // column out of range, unsorted row or not symmetric
    if (h_aux[0] >= n)
        return PBRCM_ERR_FORMAT;  // no entry at all
    const uint64_t need = nnz + 2ull * h_aux[1];
    *nnz_out = need;
    if (links_out)
        *links_out = h_aux[1];
    return need > kMaxNnz || need > cap ? PBRCM_ERR_ARG : PBRCM_OK;
}

static int32_t check_sizes(uint32_t n, uint64_t nnz)
{
    if (n == 0 || n == 0xFFFFFFFFu || nnz > kMaxNnz)
        return PBRCM_ERR_ARG;
    return PBRCM_OK;
}

}  // namespace pbrcm

// ---------------------------------------------------------------------------
// process-wide default context (per device)
// ---------------------------------------------------------------------------
static std::mutex g_default_mu;
static std::vector<pbrcm_context*> g_default;

static pbrcm_context* default_context(int32_t* rc)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        *rc = PBRCM_ERR_CUDA;
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_default_mu);
    if ((int)g_default.size() <= dev)
        g_default.resize(dev + 1, nullptr);
    if (!g_default[dev]) {
        pbrcm_context* c = nullptr;
        *rc = pbrcm_context_create(dev, &c);
        if (*rc != PBRCM_OK)
            return nullptr;
        g_default[dev] = c;
    }
    *rc = PBRCM_OK;
    return g_default[dev];
}

#define PBRCM_CTX(ctx)                               \
    int32_t rc_ctx_ = PBRCM_OK;                      \
    if (!ctx)                                        \
        ctx = default_context(&rc_ctx_);             \
    if (!ctx)                                        \
        return rc_ctx_;                              \
    std::lock_guard<std::mutex> lk_(ctx->ctx.mu);    \
    cudaSetDevice(ctx->ctx.device);

extern "C" {

void pbrcm_default_options(pbrcm_options* o)
{
    if (!o)
        return;
    std::memset(o, 0, sizeof(*o));
    o->reverse = 1;
    o->start_node = PBRCM_AUTO_START;
    o->stable = 1;
    o->want_bandwidth = 1;
    o->peripheral_nodes = 32;
    o->wait_limit_ms = 2000;
}

const char* pbrcm_version(void) { return pbrcm::kVersion; }

const char* pbrcm_status_string(int32_t s)
{
    switch (s) {
    case PBRCM_OK: return "ok";
    case PBRCM_ERR_ARG: return "invalid argument";
    case PBRCM_ERR_DISCONNECTED: return "graph not connected";
    case PBRCM_ERR_TIMEOUT: return "device wait timed out";
    case PBRCM_ERR_OOM: return "out of memory";
    case PBRCM_ERR_CUDA: return "CUDA error";
    case PBRCM_ERR_IO: return "I/O error";
    case PBRCM_ERR_FORMAT: return "format error";
    case PBRCM_ERR_CHECK: return "device check failed";
    case PBRCM_ERR_BUSY: return "over memory cap";
    case PBRCM_ERR_NOT_FOUND: return "unknown ticket";
    default: return "unknown status";
    }
}

int32_t pbrcm_context_create(int32_t device, pbrcm_context** out)
{
    if (!out)
        return PBRCM_ERR_ARG;
    *out = nullptr;
    auto* c = new (std::nothrow) pbrcm_context();
    if (!c)
        return PBRCM_ERR_OOM;
    int32_t rc = c->ctx.init(device);
    if (rc != PBRCM_OK) {
        delete c;
        return rc;
    }
    *out = c;
    return PBRCM_OK;
}

void pbrcm_context_destroy(pbrcm_context* c) { delete c; }

int32_t pbrcm_reorder(pbrcm_context* ctx, const uint32_t* row_ptr, const uint32_t* col_idx, uint32_t n, uint64_t nnz,
                      const pbrcm_options* opts, uint32_t* perm_out, pbrcm_result* result)
{
    auto t0 = std::chrono::steady_clock::now();
    if (!row_ptr || (!col_idx && nnz) || !perm_out)
        return PBRCM_ERR_ARG;
    if (int32_t rc = check_sizes(n, nnz))
        return rc;
    PBRCM_CTX(ctx);
    Context& C = ctx->ctx;
    if (!C.ensure_single(n, nnz, true))
        return PBRCM_ERR_OOM;
    Options opt = make_options(opts, kModeFull);
    cudaStream_t st = C.stream;
    if (cudaMemcpyAsync(C.d_rp, row_ptr, sizeof(uint32_t) * ((size_t)n + 1), cudaMemcpyHostToDevice, st) !=
            cudaSuccess ||
        (nnz && cudaMemcpyAsync(C.d_ci, col_idx, sizeof(uint32_t) * nnz, cudaMemcpyHostToDevice, st) != cudaSuccess))
        return PBRCM_ERR_CUDA;
    DevResult r{};
    float dms = 0.f;
    int32_t rc = C.run_single(C.d_rp, C.d_ci, n, nnz, C.d_perm, opt, st, &r, &dms);
    if (rc != PBRCM_OK)
        return rc;
    if (r.status == kOk) {
        if (cudaMemcpyAsync(perm_out, C.d_perm, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return PBRCM_ERR_CUDA;
    }
    fill_result(r, opt, result);
    if (result) {
        result->device_ms = dms;
        result->total_ms =
            std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return map_status(r.status);
}

int32_t pbrcm_reorder_device(pbrcm_context* ctx, const uint32_t* d_row_ptr, const uint32_t* d_col_idx, uint32_t n,
                             uint64_t nnz, const pbrcm_options* opts, uint32_t* d_perm_out, pbrcm_result* result,
                             void* stream)
{
    auto t0 = std::chrono::steady_clock::now();
    if (!d_row_ptr || (!d_col_idx && nnz) || !d_perm_out)
        return PBRCM_ERR_ARG;
    if (int32_t rc = check_sizes(n, nnz))
        return rc;
    PBRCM_CTX(ctx);
    Context& C = ctx->ctx;
    if (!C.ensure_single(n, nnz, false))
        return PBRCM_ERR_OOM;
    Options opt = make_options(opts, kModeFull);
    cudaStream_t st = stream ? (cudaStream_t)stream : C.stream;
    DevResult r{};
    float dms = 0.f;
    int32_t rc = C.run_single(d_row_ptr, d_col_idx, n, nnz, d_perm_out, opt, st, &r, &dms);
    if (rc != PBRCM_OK)
        return rc;
    fill_result(r, opt, result);
    if (result) {
        result->device_ms = dms;
        result->total_ms =
            std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return map_status(r.status);
}

int32_t pbrcm_permute_device(pbrcm_context* ctx, const uint32_t* d_row_ptr, const uint32_t* d_col_idx,
                             const void* d_vals, uint32_t val_bytes, uint32_t n, uint64_t nnz, const uint32_t* d_perm,
                             uint32_t* d_row_ptr_out, uint32_t* d_col_idx_out, void* d_vals_out, uint32_t* d_map_out,
                             void* stream)
{
    if (!d_row_ptr || (!d_col_idx && nnz) || !d_perm || !d_row_ptr_out || (!d_col_idx_out && nnz) ||
        (val_bytes != 0 && val_bytes != 4 && val_bytes != 8) || (val_bytes && nnz && (!d_vals || !d_vals_out)))
        return PBRCM_ERR_ARG;
    if (int32_t rc = check_sizes(n, nnz))
        return rc;
    PBRCM_CTX(ctx);
    Context& C = ctx->ctx;
    if (!grow(C.d_pw, C.cap_pw, Context::permute_work_bytes(n, nnz)))
        return PBRCM_ERR_OOM;
    cudaStream_t st = stream ? (cudaStream_t)stream : C.stream;
    return C.run_permute(d_row_ptr, d_col_idx, d_vals, val_bytes, n, nnz, d_perm, d_row_ptr_out, d_col_idx_out,
                         d_vals_out, d_map_out, C.d_pw, st);
}

int32_t pbrcm_connect_device(pbrcm_context* ctx, const uint32_t* d_row_ptr, const uint32_t* d_col_idx, uint32_t n,
                             uint64_t nnz, uint32_t* d_row_ptr_out, uint32_t* d_col_idx_out, uint64_t cap_nnz_out,
                             uint64_t* nnz_out, uint32_t* links_out, void* stream)
{
    if (!d_row_ptr || (!d_col_idx && nnz) || !d_row_ptr_out || (!d_col_idx_out && cap_nnz_out) || !nnz_out)
        return PBRCM_ERR_ARG;
    if (int32_t rc = check_sizes(n, nnz))
        return rc;
    if (nnz == 0)
        return PBRCM_ERR_FORMAT;
    PBRCM_CTX(ctx);
    Context& C = ctx->ctx;
    if (!grow(C.d_pw, C.cap_pw, Context::connect_work_bytes(n)))
        return PBRCM_ERR_OOM;
    cudaStream_t st = stream ? (cudaStream_t)stream : C.stream;
    return C.run_connect(d_row_ptr, d_col_idx, n, nnz, d_row_ptr_out, d_col_idx_out, cap_nnz_out, nnz_out, links_out,
                         C.d_pw, st);
}

int32_t pbrcm_permute(pbrcm_context* ctx, const uint32_t* row_ptr, const uint32_t* col_idx, const void* vals,
                      uint32_t val_bytes, uint32_t n, uint64_t nnz, const uint32_t* perm, uint32_t* row_ptr_out,
                      uint32_t* col_idx_out, void* vals_out, uint32_t* map_out)
{
    if (!row_ptr || (!col_idx && nnz) || !perm || !row_ptr_out || (!col_idx_out && nnz) ||
        (val_bytes != 0 && val_bytes != 4 && val_bytes != 8) || (val_bytes && nnz && (!vals || !vals_out)))
        return PBRCM_ERR_ARG;
    if (int32_t rc = check_sizes(n, nnz))
        return rc;
    PBRCM_CTX(ctx);
    Context& C = ctx->ctx;
    const size_t vb = val_bytes ? (size_t)val_bytes * nnz : 0;
    // work | in: rp, ci, perm, vals | out: rp, ci, vals, map
    const size_t w = al256(Context::permute_work_bytes(n, nnz));
    const size_t o_rp = w, o_ci = o_rp + al256(4 * ((size_t)n + 1)), o_pm = o_ci + al256(4 * nnz),
                 o_v = o_pm + al256(4 * (size_t)n), o_orp = o_v + al256(vb), o_oci = o_orp + al256(4 * ((size_t)n + 1)),
                 o_ov = o_oci + al256(4 * nnz), o_map = o_ov + al256(vb), total = o_map + al256(4 * nnz);
    if (!grow(C.d_pw, C.cap_pw, total))
        return PBRCM_ERR_OOM;
    unsigned char* D = C.d_pw;
    cudaStream_t st = C.stream;
    if (cudaMemcpyAsync(D + o_rp, row_ptr, 4 * ((size_t)n + 1), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        (nnz && cudaMemcpyAsync(D + o_ci, col_idx, 4 * nnz, cudaMemcpyHostToDevice, st) != cudaSuccess) ||
        cudaMemcpyAsync(D + o_pm, perm, 4 * (size_t)n, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        (vb && cudaMemcpyAsync(D + o_v, vals, vb, cudaMemcpyHostToDevice, st) != cudaSuccess))
        return PBRCM_ERR_CUDA;
    int32_t rc = C.run_permute(reinterpret_cast<uint32_t*>(D + o_rp), reinterpret_cast<uint32_t*>(D + o_ci),
                               vb ? D + o_v : nullptr, val_bytes, n, nnz, reinterpret_cast<uint32_t*>(D + o_pm),
                               reinterpret_cast<uint32_t*>(D + o_orp), reinterpret_cast<uint32_t*>(D + o_oci),
                               vb ? D + o_ov : nullptr, map_out ? reinterpret_cast<uint32_t*>(D + o_map) : nullptr, D,
                               st);
    if (rc != PBRCM_OK)
        return rc;
    if (cudaMemcpyAsync(row_ptr_out, D + o_orp, 4 * ((size_t)n + 1), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        (nnz && cudaMemcpyAsync(col_idx_out, D + o_oci, 4 * nnz, cudaMemcpyDeviceToHost, st) != cudaSuccess) ||
        (vb && cudaMemcpyAsync(vals_out, D + o_ov, vb, cudaMemcpyDeviceToHost, st) != cudaSuccess) ||
        (map_out && nnz && cudaMemcpyAsync(map_out, D + o_map, 4 * nnz, cudaMemcpyDeviceToHost, st) != cudaSuccess) ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return PBRCM_ERR_CUDA;
    return PBRCM_OK;
}

int32_t pbrcm_find_peripheral(pbrcm_context* ctx, const uint32_t* row_ptr, const uint32_t* col_idx, uint32_t n,
                              uint64_t nnz, uint32_t* start_out, uint32_t* passes_out, uint32_t* ecc_out)
{
    if (!row_ptr || (!col_idx && nnz) || !start_out)
        return PBRCM_ERR_ARG;
    if (int32_t rc = check_sizes(n, nnz))
        return rc;
    PBRCM_CTX(ctx);
    Context& C = ctx->ctx;
    if (!C.ensure_single(n, nnz, true))
        return PBRCM_ERR_OOM;
    pbrcm_options o;
    pbrcm_default_options(&o);
    Options opt = make_options(&o, kModeStartOnly);
    cudaStream_t st = C.stream;
    if (cudaMemcpyAsync(C.d_rp, row_ptr, sizeof(uint32_t) * ((size_t)n + 1), cudaMemcpyHostToDevice, st) !=
            cudaSuccess ||
        (nnz && cudaMemcpyAsync(C.d_ci, col_idx, sizeof(uint32_t) * nnz, cudaMemcpyHostToDevice, st) != cudaSuccess))
        return PBRCM_ERR_CUDA;
    DevResult r{};
    int32_t rc = C.run_single(C.d_rp, C.d_ci, n, nnz, C.d_perm, opt, st, &r, nullptr);
    if (rc != PBRCM_OK)
        return rc;
    *start_out = r.start;
    if (passes_out)
        *passes_out = r.passes;
    if (ecc_out)
        *ecc_out = r.ecc;
    return map_status(r.status);
}

int32_t pbrcm_bandwidth(pbrcm_context* ctx, const uint32_t* row_ptr, const uint32_t* col_idx, uint32_t n,
                        uint64_t nnz, const uint32_t* perm, int64_t* bandwidth, int64_t* initial_bandwidth,
                        uint64_t* profile)
{
    if (!row_ptr || (!col_idx && nnz) || !perm)
        return PBRCM_ERR_ARG;
    if (int32_t rc = check_sizes(n, nnz))
        return rc;
    PBRCM_CTX(ctx);
    Context& C = ctx->ctx;
    if (!C.ensure_single(n, nnz, true))
        return PBRCM_ERR_OOM;
    cudaStream_t st = C.stream;
    if (cudaMemcpyAsync(C.d_rp, row_ptr, sizeof(uint32_t) * ((size_t)n + 1), cudaMemcpyHostToDevice, st) !=
            cudaSuccess ||
        (nnz && cudaMemcpyAsync(C.d_ci, col_idx, sizeof(uint32_t) * nnz, cudaMemcpyHostToDevice, st) !=
                    cudaSuccess) ||
        cudaMemcpyAsync(C.d_perm, perm, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemsetAsync(C.d_res, 0, sizeof(DevResult), st) != cudaSuccess)
        return PBRCM_ERR_CUDA;
    if (launch_validate(C.d_rp, C.d_ci, n, (uint32_t)nnz, C.d_res, C.sms, st) != cudaSuccess ||
        launch_bandwidth(C.d_rp, C.d_ci, n, C.d_perm, reinterpret_cast<uint32_t*>(C.d_node), C.d_res, C.sms, st) !=
            cudaSuccess ||
        cudaMemcpyAsync(C.h_res, C.d_res, sizeof(DevResult), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return PBRCM_ERR_CUDA;
    const DevResult& r = *C.h_res;
    if (r.status != kOk)
        return map_status(r.status);
    if (bandwidth)
        *bandwidth = (int64_t)r.bandwidth;
    if (initial_bandwidth)
        *initial_bandwidth = (int64_t)r.initial_bw;
    if (profile)
        *profile = r.profile_lo;
    return PBRCM_OK;
}

}  // extern "C"
