/*
 * pbrcm.h -- C ABI of the B200 Reverse Cuthill-McKee engine (libpbrcm.so).
 *
 * Drop-in boundary for the GPU_BATCH path of GPUPeople/ParallelBatchRCM.
 * Plain pointers and sizes only; no CUDA or C++ types in the signatures
 * (streams are passed as void*).  Every call returns a pbrcm_status; nothing
 * throws or exits.
 *
 * Conventions shared by every entry point
 *  - A matrix is a square CSR pattern: row_ptr[n+1] and col_idx[nnz], uint32,
 *    as the reference's CSR<T> holds it (include/CSR.h:43-75 there).  Values
 *    are never read.  Rows may hold the diagonal and duplicate entries; the
 *    valence of a node is its row length (include/Graph.h:57-60).
 *  - The result is a permutation perm[k] = original node at new position k.
 *    With reverse = 0 it is the Cuthill-McKee order the reference returns
 *    (its -r flag is parsed but never applied, src/main.cpp:250); with
 *    reverse = 1 it is that order reversed (RCM).  The permutation is
 *    bit-identical to the reference's serial stable CPU RCM
 *    (src/rcm_cpu.cpp:57-104, rcm_seq<true>) from the same start node.
 *  - The automatic start node is the reference's pseudo-peripheral node
 *    (src/simple_peripheral.cpp:92-141, findPeripheral with 32 output
 *    nodes), computed on the GPU.
 *  - Bandwidth is the reference's computeBandwidth (src/main.cpp:143-184);
 *    initial bandwidth its checkBandwidth (src/main.cpp:114-129).  Profile
 *    (envelope) has no counterpart in the reference: sum over rows r of the
 *    reordered matrix of r minus its smallest column, clamped at 0.
 *  - The graph must be connected (the reference's loader connects it,
 *    include/Graph.h:160-263; pbrcm_load_mtx does the same).  A disconnected
 *    input returns PBRCM_ERR_DISCONNECTED instead of the reference's endless
 *    spin.
 */
#ifndef PBRCM_H
#define PBRCM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define PBRCM_API __attribute__((visibility("default")))
#else
#define PBRCM_API
#endif

#define PBRCM_AUTO_START 0xFFFFFFFFu

typedef enum pbrcm_status {
    PBRCM_OK = 0,
    PBRCM_ERR_ARG = 1,          /* bad argument or size out of range */
    PBRCM_ERR_DISCONNECTED = 2, /* BFS from the start did not reach every node */
    PBRCM_ERR_TIMEOUT = 3,      /* a bounded device-side wait ran out */
    PBRCM_ERR_OOM = 4,          /* device or host allocation failed */
    PBRCM_ERR_CUDA = 5,         /* a CUDA runtime call failed */
    PBRCM_ERR_IO = 6,           /* file could not be opened or read */
    PBRCM_ERR_FORMAT = 7,       /* malformed MatrixMarket / .hicsr input */
    PBRCM_ERR_CHECK = 8,        /* a device-side bounds check fired */
    PBRCM_ERR_BUSY = 9,         /* admission refused: over the memory cap */
    PBRCM_ERR_NOT_FOUND = 10    /* unknown ticket */
} pbrcm_status;

/* Options of one reorder (the reference's CLI flags, src/main.cpp:245-256). */
typedef struct pbrcm_options {
    uint32_t reverse;         /* -r: 1 = RCM (reversed CM order), 0 = CM order */
    uint32_t start_node;      /* -s: explicit start, or PBRCM_AUTO_START */
    uint32_t stable;          /* -b: accepted for compatibility; the result is
                                 always the stable order (std::sort's tie order
                                 in the reference's non-stable path is
                                 implementation-defined, src/rcm_cpu.cpp:96) */
    uint32_t want_bandwidth;  /* -w: compute bandwidth, initial bandwidth, profile */
    uint32_t peripheral_nodes;/* nodes kept per BFS pass (0 = 32, the reference default) */
    uint32_t wait_limit_ms;   /* bound of every device-side wait (0 = 2000 ms) */
    uint32_t debug_flags;     /* test hooks, 0 in production (PBRCM_DEBUG_*) */
    uint32_t reserved;
} pbrcm_options;

/* debug_flags: a grid barrier that waits for one CTA more than the launch has,
 * so that the bounded wait runs out and PBRCM_ERR_TIMEOUT comes back. */
#define PBRCM_DEBUG_PHANTOM_CTA 0x1u

typedef struct pbrcm_result {
    int32_t status;              /* pbrcm_status of this matrix */
    uint32_t start_node;         /* start actually used */
    uint32_t peripheral_passes;  /* BFS passes of the start search (0 if given) */
    uint32_t eccentricity;       /* eccentricity of the start from the search */
    uint32_t levels;             /* BFS levels of the final order */
    uint32_t placed;             /* nodes placed (n when connected) */
    int64_t bandwidth;           /* of the result (-1 if not asked) */
    int64_t initial_bandwidth;   /* of the input as stored (-1 if not asked) */
    uint64_t profile;            /* of the result (0 if not asked) */
    float device_ms;             /* device time of the reorder launch(es) */
    float total_ms;              /* host wall time of the call */
    uint32_t engine;             /* 0: team engine (one cooperative launch); 1: level-synchronous
                                    engine for wide, shallow graphs; 2: shared-memory engine for
                                    matrices that fit one CTA's shared memory (same result) */
    uint32_t reserved;
} pbrcm_result;

/* Default options: reverse=1, automatic start, stable=1, want_bandwidth=1. */
PBRCM_API void pbrcm_default_options(pbrcm_options* opts);

/* Library version string. */
PBRCM_API const char* pbrcm_version(void);

/* Human-readable name of a status code. */
PBRCM_API const char* pbrcm_status_string(int32_t status);

/* ---------------------------------------------------------------------- */
/* Context: device, stream and a growing device workspace reused by calls.  */
/* ---------------------------------------------------------------------- */
typedef struct pbrcm_context pbrcm_context;

/* Creates a context on `device` (the caller's current device if < 0). */
PBRCM_API int32_t pbrcm_context_create(int32_t device, pbrcm_context** ctx);
PBRCM_API void pbrcm_context_destroy(pbrcm_context* ctx);

/*
 * One reorder from HOST buffers.  Replaces GPU_BATCH::rcm<T>
 * (include/rcm_gpu_batch.h:40-41, src/device/rcm_gpu_batch.cu:42-112): copies
 * the CSR to the device, runs start search + CM + reverse + bandwidth in one
 * persistent launch, copies perm back.  perm_out holds n entries.
 * ctx may be NULL (a process-wide context on the current device is used).
 */
PBRCM_API int32_t pbrcm_reorder(pbrcm_context* ctx, const uint32_t* row_ptr, const uint32_t* col_idx,
                      uint32_t n, uint64_t nnz, const pbrcm_options* opts, uint32_t* perm_out,
                      pbrcm_result* result);

/*
 * One reorder on DEVICE-resident buffers, enqueued on `stream` (a
 * cudaStream_t, NULL = the context's stream); d_perm_out receives n entries.
 * Synchronises the stream before returning so that `result` is filled.
 */
PBRCM_API int32_t pbrcm_reorder_device(pbrcm_context* ctx, const uint32_t* d_row_ptr, const uint32_t* d_col_idx,
                             uint32_t n, uint64_t nnz, const pbrcm_options* opts, uint32_t* d_perm_out,
                             pbrcm_result* result, void* stream);

/*
 * Start-node search alone.  Replaces SimplePeripheral::findPeripheral
 * (include/simple_peripheral.h:46) on the GPU.  Host buffers.
 */
PBRCM_API int32_t pbrcm_find_peripheral(pbrcm_context* ctx, const uint32_t* row_ptr, const uint32_t* col_idx,
                              uint32_t n, uint64_t nnz, uint32_t* start_out, uint32_t* passes_out,
                              uint32_t* ecc_out);

/*
 * Bandwidth / profile of a permutation.  Replaces computeBandwidth
 * (src/main.cpp:143-184) on the GPU; also returns checkBandwidth
 * (src/main.cpp:114-129) of the input and the profile.  Host buffers.
 * Returns PBRCM_ERR_ARG if perm is not a bijection (checkPermutation,
 * src/main.cpp:186-226).
 */
PBRCM_API int32_t pbrcm_bandwidth(pbrcm_context* ctx, const uint32_t* row_ptr, const uint32_t* col_idx,
                        uint32_t n, uint64_t nnz, const uint32_t* perm, int64_t* bandwidth,
                        int64_t* initial_bandwidth, uint64_t* profile);

/*
 * One full reorder of a DEVICE-resident matrix that allocates nothing.  No
 * counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc while they run (a host application whose device memory is
 * owned by its own pool or by a budget fixed at start-up, or code that must
 * not let an allocation synchronise the device mid-flight).  All scratch
 * lives in a static device array reserved when the library is loaded (about
 * 32 MiB on every GPU that loads it, held until exit).  Limits: n <= 2^20
 * nodes and no row longer than 1024 entries; larger inputs return
 * PBRCM_ERR_ARG.  The first call on a device looks up the array's address and
 * should come before any stream capture.  Every call shares the array, so
 * calls that overlap on the GPU race: serialise them.  Same options, result
 * and permutation as pbrcm_reorder_device; synchronises `stream` (a
 * cudaStream_t, NULL = the legacy default stream) before returning.
 */
PBRCM_API int32_t pbrcm_reorder_device_noalloc(const uint32_t* d_row_ptr, const uint32_t* d_col_idx, uint32_t n,
                                               uint64_t nnz, const pbrcm_options* opts, uint32_t* d_perm_out,
                                               pbrcm_result* result, void* stream);

/* ---------------------------------------------------------------------- */
/* Many matrices in one persistent launch.                                 */
/* ---------------------------------------------------------------------- */
typedef struct pbrcm_matrix {
    const uint32_t* row_ptr;  /* n+1 entries */
    const uint32_t* col_idx;  /* nnz entries */
    uint32_t n;
    uint32_t reserved;
    uint64_t nnz;
    uint32_t* perm_out;       /* n entries */
} pbrcm_matrix;

/*
 * Reorders `count` independent matrices (HOST buffers) with one persistent
 * launch: the CSRs are packed into one device arena and copied in waves
 * while the kernel already reorders the ones that have arrived; every CTA
 * runs several thread groups, one matrix each, and the biggest matrices run
 * on thread-block-cluster teams (the shape is the context's tuning: see
 * pbrcm_autotune).  results[i] receives matrix i's result; its device_ms is
 * the time from the batch's first matrix taken to matrix i's result.  The
 * reference has no batched form; each permutation equals the single-matrix
 * result.
 */
PBRCM_API int32_t pbrcm_reorder_batch(pbrcm_context* ctx, const pbrcm_matrix* mats, uint32_t count,
                            const pbrcm_options* opts, pbrcm_result* results);

/* Same on device-resident CSRs and device perm buffers (pointers in `mats`
 * are device pointers; `mats` itself is a host array). */
PBRCM_API int32_t pbrcm_reorder_batch_device(pbrcm_context* ctx, const pbrcm_matrix* mats, uint32_t count,
                                   const pbrcm_options* opts, pbrcm_result* results, void* stream);

/* ---------------------------------------------------------------------- */
/* Autotuner of the batch and serving shapes.                              */
/* ---------------------------------------------------------------------- */

/*
 * The shape settings of the batched and serving paths.  They replace the
 * reference's compile-time constants (include/rcm_gpu_batch_params.h:36-46:
 * BlockSizePow, MaxElementsPerThreadPow, QueueSize, Overalloc), which set
 * one batch shape for every input; here they are measured per device.
 */
typedef struct pbrcm_tuning {
    uint32_t batch_pool;       /* thread groups of the batch kernel, one matrix each:
                                  0 = 1 x 512 threads per CTA, 1 = 2 x 256, 2 = 4 x 128,
                                  3 = 8 x 64, 5 / 6 = 256-thread CTAs with 512 / 1024-edge
                                  chunks, 7 = 2 x 256 with 2048-edge chunks */
    uint32_t batch_kernel;     /* 0: the general batch kernel; 1: the solo batch kernel where
                                  every job is one group's (no teams, no clusters): the
                                  one-group engine alone, fewer registers, more CTAs per SM */
    uint32_t cluster_size;     /* CTAs of a cluster team for the biggest matrices (1 = none) */
    uint32_t cluster_max;      /* at most this many matrices of a batch get a cluster team */
    uint32_t cluster_nnz;      /* ... and only those with at least this many entries */
    uint32_t session_cutoff_n; /* serving: requests with more nodes run on a cooperative team */
    uint32_t session_pool;     /* serving: CTA shape of the other requests (0 = 512 threads,
                                  5 = 256 threads, three per SM, 4 = 128 threads, four per SM) */
    uint32_t session_team_nnz; /* serving: a team request gets one CTA per this many entries */
    uint32_t session_cluster_max; /* serving: largest thread-block-cluster team (0 = cooperative
                                  teams only) */
    uint32_t sms;              /* streaming multiprocessors of the device it was measured on */
    uint32_t trials;           /* settings measured */
    uint32_t source;           /* 0 built-in defaults, 1 a tuning file, 2 measured or set */
    float default_ms;          /* calibration batch with the settings the tuner started from */
    float best_ms;             /* ... with the chosen settings */
    float session_default_ms;  /* calibration serving replay: makespan before / after */
    float session_best_ms;
} pbrcm_tuning;

/*
 * Measures the batch shapes on `mats` (a calibration batch on HOST buffers,
 * e.g. a sample of the caller's own workload): the thread-group shape, the
 * cluster-team size, count and threshold, then the serving cutoff (a replay
 * of the batch through a session), each against the current best.  Every
 * setting tried must give bit-identical permutations (it returns
 * PBRCM_ERR_CHECK otherwise).  The chosen settings become the context's;
 * with cache_path they are also written there, keyed by the device's SM
 * count and the library version, for pbrcm_tuning_load or the PBRCM_TUNING
 * environment variable (read by pbrcm_context_create; the PBRCM_* knobs
 * still override single settings).  `out` (nullable) receives them.
 */
PBRCM_API int32_t pbrcm_autotune(pbrcm_context* ctx, const pbrcm_matrix* mats, uint32_t count,
                                 const pbrcm_options* opts, const char* cache_path, pbrcm_tuning* out);

/* The context's current settings. */
PBRCM_API int32_t pbrcm_tuning_get(pbrcm_context* ctx, pbrcm_tuning* out);
/* Sets them (out-of-range values return PBRCM_ERR_ARG, nothing changed). */
PBRCM_API int32_t pbrcm_tuning_set(pbrcm_context* ctx, const pbrcm_tuning* t);
/* Applies a cache file written by pbrcm_autotune; PBRCM_ERR_NOT_FOUND if it
 * is missing or was measured on another device shape or library version. */
PBRCM_API int32_t pbrcm_tuning_load(pbrcm_context* ctx, const char* path);

/* ---------------------------------------------------------------------- */
/* Serving session: continuous batching of reorder requests.               */
/* ---------------------------------------------------------------------- */
typedef struct pbrcm_session pbrcm_session;

typedef struct pbrcm_session_config {
    uint64_t memory_cap_bytes; /* admission cap on device bytes in flight (0 = 120 GB) */
    uint32_t max_inflight;     /* most requests on the device at once (0 = 4096) */
    uint32_t streams;          /* concurrent device streams (0 = 8) */
    uint32_t reserved[4];
} pbrcm_session_config;

PBRCM_API int32_t pbrcm_session_create(pbrcm_context* ctx, const pbrcm_session_config* cfg, pbrcm_session** s);
PBRCM_API void pbrcm_session_destroy(pbrcm_session* s);

/*
 * Submits one request (HOST buffers, copied before return).  Returns
 * PBRCM_ERR_BUSY if the request alone exceeds the memory cap; otherwise the
 * request is queued and admitted as soon as memory and slots allow.
 */
PBRCM_API int32_t pbrcm_session_submit(pbrcm_session* s, const uint32_t* row_ptr, const uint32_t* col_idx,
                             uint32_t n, uint64_t nnz, const pbrcm_options* opts, uint64_t* ticket);

/*
 * Polls a ticket: returns PBRCM_OK with perm_out (n entries) and result
 * filled once done (*done = 1), or *done = 0 if still running.  A finished
 * ticket is released by the first poll that returns it.
 */
PBRCM_API int32_t pbrcm_session_poll(pbrcm_session* s, uint64_t ticket, uint32_t* perm_out, pbrcm_result* result,
                           int32_t* done);

/* Blocks until every submitted request has finished. */
PBRCM_API int32_t pbrcm_session_drain(pbrcm_session* s);

/* Latency / throughput counters since creation. */
typedef struct pbrcm_session_stats {
    uint64_t submitted, completed;
    uint64_t bytes_in_flight, peak_bytes_in_flight;
    double p50_ms, p99_ms, max_ms;     /* submit -> completion latency */
    double busy_s;                     /* wall time from first submit to last completion */
} pbrcm_session_stats;

PBRCM_API int32_t pbrcm_session_stats_get(pbrcm_session* s, pbrcm_session_stats* st);

/* ---------------------------------------------------------------------- */
/* Input boundary: MatrixMarket loader with the reference's semantics.     */
/* ---------------------------------------------------------------------- */

/*
 * Loads a MatrixMarket `coordinate` file like Graph<T>::load
 * (include/Graph.h:266-332: COO.cpp:89-199 parse, CSR.cpp:170-200 sort by
 * (row, col), prepareRCM symmetrize + connect) without writing .hicsr cache
 * files.  *row_ptr and *col_idx are malloc'd; free them with pbrcm_free.
 */
PBRCM_API int32_t pbrcm_load_mtx(const char* path, uint32_t* n, uint64_t* nnz, uint32_t** row_ptr,
                       uint32_t** col_idx);

/* prepareRCM (include/Graph.h:74-264) on a caller CSR; outputs malloc'd. */
PBRCM_API int32_t pbrcm_prepare_csr(const uint32_t* row_ptr, const uint32_t* col_idx, uint32_t n, uint64_t nnz,
                          int32_t check_symmetry, uint64_t* nnz_out, uint32_t** row_ptr_out,
                          uint32_t** col_idx_out);

PBRCM_API void pbrcm_free(void* p);

/*
 * The reference's binary CSR cache, `.hicsr` (storeCSR / loadCSR,
 * src/CSR.cpp:57-168; Graph<T>::load keeps `<file>.hicsr` and
 * `<file>.rcm.hicsr` next to a MatrixMarket input, include/Graph.h:266-332).
 * pbrcm_load_hicsr reads either; *row_ptr, *col_idx and (if vals is not NULL)
 * *vals are malloc'd (free with pbrcm_free), *val_bytes is 4 (float) or 8
 * (double).  pbrcm_store_hicsr writes one the reference can read; without
 * values (val_bytes 0) every value is float 1.0.
 */
PBRCM_API int32_t pbrcm_load_hicsr(const char* path, uint32_t* n, uint64_t* nnz, uint32_t** row_ptr,
                                   uint32_t** col_idx, void** vals, uint32_t* val_bytes);
PBRCM_API int32_t pbrcm_store_hicsr(const char* path, uint32_t n, uint64_t nnz, const uint32_t* row_ptr,
                                    const uint32_t* col_idx, const void* vals, uint32_t val_bytes);

/* ---------------------------------------------------------------------- */
/* Output boundary: the reordered matrix (the reference's `-o`).           */
/* ---------------------------------------------------------------------- */

/*
 * B = P A P^T for a permutation perm (perm[k] = original row at position k):
 * row i of B is row perm[i] of A with every column c renamed to the position
 * of c, entries sorted by the new column (duplicate entries of A keep their
 * order).  Replaces CuSolverRCM::reorder (include/device/rcm_cusolver.cuh:
 * 154-185: cusolverSpXcsrpermHost with p = q = perm, then the values shuffled
 * through its map).  vals / vals_out: nnz values of val_bytes = 4 or 8 bytes
 * each, moved with their entries (val_bytes = 0: no values, both may be
 * NULL).  map_out (nullable, nnz): the entry of A each entry of B came from.
 * row_ptr_out has n + 1 entries.  A perm that is not a permutation of 0..n-1
 * returns PBRCM_ERR_ARG.
 */
PBRCM_API int32_t pbrcm_permute(pbrcm_context* ctx, const uint32_t* row_ptr, const uint32_t* col_idx,
                                const void* vals, uint32_t val_bytes, uint32_t n, uint64_t nnz, const uint32_t* perm,
                                uint32_t* row_ptr_out, uint32_t* col_idx_out, void* vals_out, uint32_t* map_out);

/* The same on device buffers, enqueued on `stream` (a cudaStream_t; NULL =
 * the context's stream), which is synchronised before returning. */
PBRCM_API int32_t pbrcm_permute_device(pbrcm_context* ctx, const uint32_t* d_row_ptr, const uint32_t* d_col_idx,
                                       const void* d_vals, uint32_t val_bytes, uint32_t n, uint64_t nnz,
                                       const uint32_t* d_perm, uint32_t* d_row_ptr_out, uint32_t* d_col_idx_out,
                                       void* d_vals_out, uint32_t* d_map_out, void* stream);

/*
 * The connectivity repair of the reference's loader (Graph<T>::prepareRCM,
 * include/Graph.h:160-263) on device buffers: every component is joined to
 * the rest by the links that loader adds -- with minn the first non-empty
 * row, (m - 1, m) for each component whose smallest node m > 0 is not in
 * minn's, and (0, minn) when row 0 is empty -- both directions inserted at
 * their sorted place.  The input is the symmetric pattern the loader has at
 * that point (every row sorted by column, as pbrcm_load_mtx and the
 * reference's convert leave it); a column out of range, an unsorted row or a
 * missing transposed entry returns PBRCM_ERR_ARG, a matrix without entries
 * PBRCM_ERR_FORMAT.  An empty row is a component of its own (the reference
 * never finishes on one; pbrcm_prepare_csr links it the same way).
 * Outputs: d_row_ptr_out (n + 1) and d_col_idx_out (cap_nnz_out entries;
 * nnz + 2 (n - 1) always suffices); *nnz_out = the output's entry count and
 * *links_out (nullable) = the links added.  A connected matrix comes back
 * unchanged.  With cap_nnz_out below *nnz_out the call returns PBRCM_ERR_ARG
 * with *nnz_out set (the output is incomplete; call again with room).
 * Enqueued on `stream` (NULL = the context's stream), synchronised before
 * returning.
 */
PBRCM_API int32_t pbrcm_connect_device(pbrcm_context* ctx, const uint32_t* d_row_ptr, const uint32_t* d_col_idx,
                                       uint32_t n, uint64_t nnz, uint32_t* d_row_ptr_out, uint32_t* d_col_idx_out,
                                       uint64_t cap_nnz_out, uint64_t* nnz_out, uint32_t* links_out, void* stream);

/*
 * Writes a CSR as a MatrixMarket file in the reference's format (storeMTX,
 * src/COO.cpp:213-251: "coordinate real general", 1-based "row col value"
 * lines, values printed like std::to_string).  val_bytes 4 = float, 8 =
 * double; 0 writes "coordinate pattern general" without values.
 */
PBRCM_API int32_t pbrcm_store_mtx(const char* path, uint32_t n, uint64_t nnz, const uint32_t* row_ptr,
                                  const uint32_t* col_idx, const void* vals, uint32_t val_bytes);

#ifdef __cplusplus
}
#endif

#endif /* PBRCM_H */
