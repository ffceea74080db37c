// context.h -- per-device state behind a pbrcm_context.
#pragma once

#include <cstddef>
#include <cstdint>
#include <memory>
#include <mutex>
#include <vector>

#include <cuda_runtime.h>

#include "types.h"

namespace pbrcm {

struct Context {
    std::mutex mu;
    int device = -1;
    int sms = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int team_variant = 1;   // kernel shape of the one-matrix team
    int team_ctas = 0;      // CTAs of the one-matrix team
    int batch_pool = 6;     // shape of the batch kernels (kPools: CTA and group sizes)
    bool solo = true;       // batch: one-group jobs run the solo engine where it applies (PBRCM_SOLO=0: never)
    // batch without teams: the solo batch kernel (no team engine code, fewer
    // registers, more CTAs per SM) in place of the general one
    // (PBRCM_BATCH_SOLO_KERNEL=0: never)
    bool batch_solo_kernel = true;
    uint32_t solo_edges = 0;    // levels at most this big run on one CTA
    uint32_t solo_parents = 0;
    uint32_t barrier = 0;       // team barrier implementation
    uint32_t spec_from = 3;     // speculative split from this search pass on (team-dominated matrices)
    int team_maxc = 0;          // co-resident CTAs of the team kernel
    // the level-synchronous engine for wide, shallow graphs (wide.cu): a
    // first-pass level of at least max(n / wide_div, wide_min) nodes hands
    // the matrix over; wide_force runs it first (rows permitting)
    uint32_t wide_div = 16, wide_min = 1u << 18;
    bool wide_force = false;
    bool team_force = false;  // PBRCM_ENGINE=team: no shared-memory engine, no hand-over
    bool wide_fused = true;        // the place kernel's last CTA advances the level state
    bool wide_batch_pass = true;   // batches sized by the last pass's levels (else 8, 16, 32, ...)
    int wide_ctas = 0;  // CTAs per level step (0: engine unavailable)
    // the shared-memory engine (resident.cu) for matrices whose CSR and
    // workspace fit one CTA's shared memory: group size (32, 64, 128, 256;
    // 0 off; -1 chosen per matrix)
    int resident_group = -1;
    int resident_max_smem = 0;  // dynamic shared memory a CTA may take
    // batches: the biggest matrices go to thread-block-cluster teams
    int cluster_size = 1;             // CTAs per cluster (0 or 1: off)
    uint64_t cluster_nnz = 1u << 18;  // matrices with at least this many entries
    int cluster_max = 16;             // cap on the matrices given a cluster (0: one per co-resident cluster)
    uint32_t cluster_solo_parents = 0, cluster_solo_edges = 0;  // solo level bounds inside a cluster
    // serving: a request of more nodes runs on a cooperative team
    uint32_t session_cutoff_n = 1u << 18;
    int session_pool = 0;  // serving: kPools shape of the one-CTA requests (512-thread CTAs: on the
                           // Poisson mix 264 reorders/s against 219 for 256-thread CTAs)
    uint32_t session_team_nnz = 1u << 20;  // serving: entries per team CTA
    int session_cluster_max = 16;          // serving: largest cluster team (0: cooperative teams only)
    // where the batch / serving shape came from: 0 built-in defaults, 1 a
    // tuning file, 2 pbrcm_autotune or pbrcm_tuning_set
    uint32_t tuned = 0;

    // single-matrix buffers (grow only)
    uint32_t* d_rp = nullptr;
    size_t cap_rp = 0;
    uint32_t* d_ci = nullptr;
    size_t cap_ci = 0;
    NodeEntry* d_node = nullptr;
    size_t cap_node = 0;
    uint32_t* d_perm = nullptr;
    size_t cap_perm = 0;
    PosRec* d_rec = nullptr;
    size_t cap_rec = 0;
    PosRec* d_rec2 = nullptr;  // queue records of the speculative ordered pass
    size_t cap_rec2 = 0;
    PosRec* d_stage = nullptr;  // staged children of multi-chunk team levels (2 nnz)
    size_t cap_stage = 0;
    uint32_t* d_hub = nullptr;
    size_t cap_hub = 0;
    DevResult* d_res = nullptr;
    DevResult* h_res = nullptr;
    uint32_t* h_aux = nullptr;  // pinned words read back with a result
    GridSync* d_gs = nullptr;
    unsigned long long* d_agg = nullptr;
    unsigned char* d_wide = nullptr;  // WideState | per-CTA totals | inverse permutation (n)
    size_t cap_wide = 0;

    // matrix permutation workspace (grow only)
    unsigned char* d_pw = nullptr;
    size_t cap_pw = 0;

    // batch buffers (grow only)
    BatchJob* d_jobs = nullptr;
    size_t cap_jobs = 0;
    BatchSlot* d_slots = nullptr;
    size_t cap_slots = 0;
    uint32_t* d_counter = nullptr;
    size_t cap_counter = 0;
    DevResult* d_bres = nullptr;
    size_t cap_bres = 0;
    unsigned char* d_arena = nullptr;
    size_t cap_arena = 0;
    // host-buffer batches: inputs copied in waves on copy_stream, each wave
    // followed by a copy of *h_one into its ready word d_ready[w]
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    uint32_t* d_ready = nullptr;
    size_t cap_ready = 0;
    uint32_t* h_one = nullptr;
    // pinned staging of a batch's job list and results (grow only)
    BatchJob* h_jobs = nullptr;
    size_t cap_hjobs = 0;
    BatchSlot* h_slots = nullptr;
    size_t cap_hslots = 0;
    DevResult* h_bres = nullptr;
    size_t cap_hbres = 0;
    // batches on device buffers, or on host buffers that are all pinned, are
    // captured as one CUDA graph (job list and copies in, kernel, results
    // and permutations out) and replayed while the same buffers, sizes,
    // options and shape come back (PBRCM_BATCH_GRAPHS=0: never)
    bool batch_graphs = true;
    // serving sessions' pinned staging pool, shared by the context's sessions
    // (created by the first session; type private to session.cpp)
    std::shared_ptr<void> session_pinned;
    struct BatchGraph {
        uint64_t key = 0;
        cudaGraphExec_t exec = nullptr;
        std::vector<uint32_t> order;  // job q -> matrix index
        std::vector<BatchJob> jobs;
        uint64_t replays = 0;
        // the job list the graph uploads (pinned, owned by the graph)
        BatchJob* h_jobs = nullptr;
        size_t cap_jobs = 0;
        BatchSlot* h_slots = nullptr;
        size_t cap_slots = 0;
    } bgraph;

    int32_t init(int dev);
    ~Context();
    bool ensure_single(uint32_t n, uint64_t nnz, bool inputs);
    bool ensure_hub(uint64_t nnz);
    int32_t run_permute(const uint32_t* rp, const uint32_t* ci, const void* vals, uint32_t val_bytes, uint32_t n,
                        uint64_t nnz, const uint32_t* perm, uint32_t* out_rp, uint32_t* out_ci, void* out_vals,
                        uint32_t* out_map, unsigned char* work, cudaStream_t st);
    static size_t permute_work_bytes(uint32_t n, uint64_t nnz);
    int32_t run_connect(const uint32_t* rp, const uint32_t* ci, uint32_t n, uint64_t nnz, uint32_t* out_rp,
                        uint32_t* out_ci, uint64_t cap, uint64_t* nnz_out, uint32_t* links_out, unsigned char* work,
                        cudaStream_t st);
    static size_t connect_work_bytes(uint32_t n);
    int32_t run_single(const uint32_t* rp, const uint32_t* ci, uint32_t n, uint64_t nnz, uint32_t* perm,
                       const Options& opt, cudaStream_t st, DevResult* out, float* dev_ms);
    // the level-synchronous engine on M (node table, passes, bandwidth);
    // false on a CUDA error; M.res holds the outcome (kNeedTeam: use the team)
    bool run_wide(const MatrixView& M, const Options& opt, cudaStream_t st);
};

// The many-matrix driver (batch.cpp); `host` selects whether mats[] point
// to host or device memory.
int32_t run_batch(Context& C, const struct pbrcm_matrix* mats, uint32_t count, const struct pbrcm_options* opts,
                  struct pbrcm_result* results, cudaStream_t st, bool host);
// The shape settings a tuning holds (tune.cpp): read by Context::init from
// the file named by PBRCM_TUNING when its key matches this device and
// library, before the environment knobs (which still override).
bool load_tuning_file(const char* path, int sms, struct pbrcm_tuning* out);

int32_t map_status(uint32_t s);
Options make_options(const struct pbrcm_options* o, uint32_t mode);
void apply_team_shape(const Context& C, Options& opt);
void fill_result(const DevResult& r, const Options& opt, struct pbrcm_result* out);

}  // namespace pbrcm

struct pbrcm_context {
    pbrcm::Context ctx;
};
