// kernels.h -- host-callable launchers of the engine kernels (kernels.cu).
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

#include "types.h"

namespace pbrcm {

// Kernel shape variants: threads per CTA (B) and edges per chunk (EMAX).
struct VariantInfo {
    int block;
    int emax;
};
constexpr int kNumVariants = 3;
extern const VariantInfo kVariants[kNumVariants];

// Shapes of the batch kernels ("pools"): CTAs of `block` threads (a
// cluster team of whole CTAs chunks `emax` edges per CTA) split into groups
// of `group` threads that reorder one matrix each (`gemax` edges per chunk).
struct PoolInfo {
    int block;
    int emax;
    int group;
    int gemax;
};
constexpr int kNumPools = 8;
extern const PoolInfo kPools[kNumPools];
// Shapes a batch may use (all but 4, the session's 128-thread CTA) and
// shapes a session may give a one-request CTA (one group per CTA).
bool batch_pool_ok(int p);
bool session_pool_ok(int p);

// Entry points of one pool shape (see launch_batch / launch_cluster).
struct PoolFns {
    int (*batch_max_ctas)(int sms);
    int (*cluster_max_active)(int csize);
    cudaError_t (*batch)(const BatchJob* jobs, const BatchSlot* slots, uint32_t nslots, uint32_t* counter,
                         const Options& opt, int ctas, bool cooperative, cudaStream_t st);
    cudaError_t (*cluster)(const BatchJob* jobs, uint32_t nbig, const BatchSlot* slots, uint32_t nslots,
                           uint32_t* counters, const Options& copt, const Options& opt, int csize, int nclusters,
                           cudaStream_t st);
    int (*solo_max_ctas)(int sms);
    cudaError_t (*solo)(const BatchJob* jobs, const BatchSlot* slots, uint32_t nslots, uint32_t* counter,
                        const Options& opt, int ctas, cudaStream_t st);
};

size_t variant_smem(int v);
int team_max_ctas(int v, int sms);   // co-resident CTAs of the team kernel
int batch_max_ctas(int p, int sms);  // co-resident CTAs of pool p's batch kernel
// Pool p's solo batch kernel (only one-group jobs with edge records, no
// teams): co-resident CTAs (0: the shape has none) and the launch.
int solo_max_ctas(int p, int sms);
cudaError_t launch_solo(int p, const BatchJob* jobs, const BatchSlot* slots, uint32_t nslots, uint32_t* counter,
                        const Options& opt, int ctas, cudaStream_t st);

// The shared-memory engine (resident.cu): one CTA of two groups of g
// threads (32, 64, 128 or 256) holds the matrix in shared memory and runs the
// whole reorder.  resident_smem: dynamic shared memory for one (spec false)
// or two workspaces; the launch takes two when they fit max_smem.  Rows of
// more than kResidentMaxRow entries are refused on the device (kNeedTeam).
constexpr uint32_t kResidentMaxRow = 512;
bool resident_group_ok(int g);
// Group size by the matrix: 256 threads above six entries a row (3-D meshes
// and denser: wider levels), else 128 (on a B200: the 64^2 grid 0.34 ms with
// 128, 0.38 with 256; a 16^3 grid 0.25 against 0.22 ms, a 3,000-node random
// geometric graph 0.47 against 0.39).
inline int resident_default_group(uint32_t n, uint64_t nnz) { return nnz > 6 * (uint64_t)n ? 256 : 128; }
size_t resident_smem(int g, uint32_t n, uint32_t nnz, bool spec);
cudaError_t launch_resident(int g, const uint32_t* rp, const uint32_t* ci, uint32_t n, uint32_t nnz, uint32_t* perm,
                            DevResult* res, const Options& opt, int max_smem, cudaStream_t st);

cudaError_t launch_validate(const uint32_t* rp, const uint32_t* ci, uint32_t n, uint32_t nnz, DevResult* res,
                            int sms, cudaStream_t st);
cudaError_t launch_team(int v, const MatrixView& M, const Options& opt, GridSync* gs, unsigned long long* agg,
                        int ctas, cudaStream_t st);
// pool p's batch kernel; cooperative: required when some job has a team of
// more than one group
cudaError_t launch_batch(int p, const BatchJob* jobs, const BatchSlot* slots, uint32_t nslots, uint32_t* counter,
                         const Options& opt, int ctas, bool cooperative, cudaStream_t st);
// A batch in thread-block clusters: jobs[0..nbig) one per cluster (team
// options copt), then the one-group slots by pool p's groups (opt);
// counters[0..1] zeroed per launch.
int cluster_max_active(int p, int csize);  // co-resident clusters of that size
cudaError_t launch_cluster(int p, const BatchJob* jobs, uint32_t nbig, const BatchSlot* slots, uint32_t nslots,
                           uint32_t* counters, const Options& copt, const Options& opt, int csize, int nclusters,
                           cudaStream_t st);
// inv[perm[k]] = k over a zeroed-to-0xFF inv; a non-permutation posts
// kErrArg (kernels.cu)
void launch_perm_inverse(const uint32_t* perm, uint32_t n, uint32_t* inv, DevResult* res, int blocks,
                         cudaStream_t st);
// B = P A P^T (permute.cu): row_ptr_out (n+1), col_idx_out (nnz), values of
// val_bytes 0 / 4 / 8 and the source map (nullable) from row_ptr, col_idx,
// values and perm.  Workspace: inv (n), partials (scan_partials_count(n)),
// mid_rows (n), long_rows (cap_long = permute_long_cap(n, nnz)), counters
// (2), scratch (4 * nnz, only needed when a row has more than 1,024
// entries; else nullptr and cap_long 0).
cudaError_t launch_permute(const uint32_t* rp, const uint32_t* ci, const void* vals, uint32_t val_bytes, uint32_t n,
                           uint32_t nnz, const uint32_t* perm, uint32_t* inv, uint32_t* out_rp, uint32_t* out_ci,
                           void* out_vals, uint32_t* out_map, uint32_t* partials, uint32_t* mid_rows,
                           uint32_t* long_rows, uint32_t cap_long, uint32_t* counters, uint32_t* scratch,
                           DevResult* res, int sms, cudaStream_t st);
// the long rows launch_permute listed (counters[1]) when it had no scratch
cudaError_t launch_permute_long(const uint32_t* rp, const uint32_t* ci, const void* vals, uint32_t val_bytes,
                                uint32_t n, uint32_t nnz, const uint32_t* perm, const uint32_t* inv,
                                const uint32_t* out_rp, uint32_t* out_ci, void* out_vals, uint32_t* out_map,
                                const uint32_t* long_rows, uint32_t cap_long, const uint32_t* counters,
                                uint32_t* scratch, DevResult* res, int sms, cudaStream_t st);
uint32_t scan_partials_count(uint32_t n);
// in-place inclusive scan of data[0..m) (permute.cu); partials holds
// scan_partials_count(m) words
cudaError_t launch_scan(uint32_t* data, uint64_t m, uint32_t* partials, cudaStream_t st);
// The loader's connectivity repair (connect.cu): out_rp (n+1) and out_ci
// (writes at or past cap dropped) from a symmetric CSR with sorted rows.
// Workspace: parent (n), partials (scan_partials_count(n)), counters (4):
// [0] first non-empty row, [1] links added, [2] check flags (1 column out of
// range, 2 row not sorted, 4 not symmetric, 8 union limit).
cudaError_t launch_connect(const uint32_t* rp, const uint32_t* ci, uint32_t n, uint32_t nnz, uint32_t* out_rp,
                           uint32_t* out_ci, uint64_t cap, uint32_t* parent, uint32_t* partials, uint32_t* counters,
                           int sms, cudaStream_t st);
uint32_t permute_long_cap(uint32_t n, uint64_t nnz);
constexpr uint32_t kPermuteWarpRow = 1024;  // longest row of the warp path
cudaError_t launch_bandwidth(const uint32_t* rp, const uint32_t* ci, uint32_t n, const uint32_t* perm, uint32_t* inv,
                             DevResult* res, int sms, cudaStream_t st);
// bandwidth, initial bandwidth and profiles from an inverse permutation
cudaError_t launch_bw_rows(const uint32_t* rp, const uint32_t* ci, uint32_t n, const uint32_t* inv, DevResult* res,
                           int sms, cudaStream_t st);
// The level-synchronous engine (wide.cu).  launch_wide_start fills the node
// table and starts the first pass; launch_wide_steps enqueues `steps` level
// steps (each a no-op once ws->phase is kWideDone; fused: the place
// kernel's last CTA advances the state, else a one-CTA kernel after it);
// launch_wide_bandwidth
// writes the bandwidth and profiles of the result (inv: n words).  `ctas` CTAs
// per step (wide_ctas_per_sm() x SMs fills the GPU once); rows must be at
// most wide_emax() long.
int wide_ctas_per_sm();
uint32_t wide_emax();
cudaError_t launch_wide_start(const MatrixView& M, const Options& opt, WideState* ws, int sms, cudaStream_t st);
cudaError_t launch_wide_steps(const MatrixView& M, const Options& opt, WideState* ws, unsigned long long* tot,
                              int ctas, int steps, bool fused, cudaStream_t st);
cudaError_t launch_wide_bandwidth(const MatrixView& M, uint32_t* inv, int sms, cudaStream_t st);

}  // namespace pbrcm
