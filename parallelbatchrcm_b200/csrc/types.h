// types.h -- plain data shared by the engine's device code and host code.
#pragma once

#include <cstddef>
#include <cstdint>

#if defined(__CUDACC__)
#define PBRCM_HD __host__ __device__
#else
#define PBRCM_HD
#endif

namespace pbrcm {

constexpr uint32_t kUnvisited = 0xFFFFFFFFu;
constexpr uint32_t kFull = 0xFFFFFFFFu;

enum : uint32_t {
    kOk = 0,
    kErrArg = 1,
    kErrDisconnected = 2,
    kErrTimeout = 3,
    kErrCheck = 8,
    kNeedHub = 100,   // internal: relaunch with hub scratch
    kNeedWide = 101,  // internal: the first pass met a wide level; run the level-synchronous engine
    kNeedTeam = 102,  // internal: the level-synchronous engine cannot take this matrix; run the team
};

// One record per queue position: node, row start, valence, edge id base.
struct alignas(16) PosRec {
    uint32_t node, rs, deg, ebase;
};

// One entry per node: claim key (see engine.cuh), row start, valence and,
// after the final pass, the node's position (inverse permutation).  Claim,
// row start and valence share one 16-byte load.
struct alignas(16) NodeEntry {
    uint32_t claim, rs, deg, inv;
};

// Grid-team synchronisation words, zeroed before every cooperative launch.
//   count      monotonic barrier counter: every CTA adds 1 per barrier and
//              waits until it reaches (barriers so far) x (team size)
//   epoch      bumped by CTA 0 when it hands a run of small levels ("solo"
//              levels it processed alone) back to the whole team
//   heartbeat  bumped by CTA 0 once per solo level (keeps the waiters' bounded
//              wait from running out while CTA 0 makes progress)
//   st[]       the level state CTA 0 publishes with the epoch
struct alignas(128) GridSync {
    unsigned int count;
    unsigned int pad0[31];
    unsigned int epoch;
    unsigned int heartbeat;
    unsigned int st[14];
    unsigned int pad1[16];
};

// Device-side result of one matrix.
struct alignas(16) DevResult {
    uint32_t status;
    uint32_t where;  // diagnostic code of a failed wait / check
    uint32_t start;
    uint32_t passes;
    uint32_t ecc;
    uint32_t levels;
    uint32_t placed;
    uint32_t maxdeg;   // largest valence (written by the validation kernel)
    uint32_t engine;   // set by the host: 0 team engine, 1 level-synchronous engine
    uint32_t pad_;
    unsigned long long bandwidth;      // max |inv[i]-inv[j]|
    unsigned long long initial_bw;
    unsigned long long profile_lo;     // sum inv[i] - min(inv[row])   (CM order)
    unsigned long long profile_hi;     // sum max(inv[row]) - inv[i]   (reversed order)
    unsigned long long t_begin;        // %globaltimer (ns) when the engine took the matrix
    unsigned long long t_end;          // %globaltimer (ns) when its result was written
};

// One matrix as the engine sees it.
struct MatrixView {
    const uint32_t* __restrict__ rp;   // n+1
    const uint32_t* __restrict__ ci;   // nnz
    uint32_t n;
    uint32_t nnz;                      // <= kMaxNnz (checked by the host)
    NodeEntry* node;                   // n
    PosRec* rec;                       // n
    uint32_t* perm;                    // n   output
    uint32_t* hub;                     // 4 * nnz hub scratch, or nullptr if no hub can occur
    DevResult* res;
    PosRec* rec2;                      // n: queue records of the speculative ordered pass, or nullptr
    uint32_t cf;                       // claim word of NodeEntry this pass uses (0 claim, 3 inv)
    PosRec* stage;                     // 2 nnz: ranked children of multi-chunk team levels (the
                                       // speculative half uses the second nnz), or nullptr
};

constexpr uint64_t kMaxNnz = 0xFFFFFFF0ull;

// The one-group engine of the batch kernels (solo.cuh) keeps a matrix's
// visited set in shared memory: matrices of at most this many nodes.
constexpr uint32_t kSoloMaxN = 1u << 18;
// Its 8-byte edge and queue records hold a node in 20 bits and a valence in
// 12: matrices of at most this many nodes (and rows of at most 4,095).
constexpr uint32_t kSoloMaxNodes = 1u << 20;

// Bytes of the per-launch team words of a cooperative launch of `ctas` CTAs:
// 2 x u64 per CTA for the level all-gather, then one u32 barrier flag per
// CTA (plus room for the phantom test CTA).
inline size_t team_words_bytes(int ctas)
{
    return 16 * (size_t)(ctas > 0 ? ctas : 1) + 4 * ((size_t)(ctas > 0 ? ctas : 1) + 8);
}

// A single-matrix team launch gets kTeamParts sets of team words and
// GridSyncs: part 0 for the whole team, parts 1 and 2 for its two halves
// while they run a start-search pass and the speculative ordered pass side
// by side.  Parts are team_part_bytes apart.
constexpr int kTeamParts = 3;
PBRCM_HD inline size_t team_part_bytes(int ctas)
{
    return (16 * (size_t)(ctas > 0 ? ctas : 1) + 4 * ((size_t)(ctas > 0 ? ctas : 1) + 8) + 255) & ~(size_t)255;
}

// One matrix of a batch: its view, its team size (CTAs that reorder it
// together) and, for teams, its own barrier words.
struct BatchJob {
    MatrixView M;
    uint32_t team;
    uint32_t pad;
    GridSync* gs;                 // team > 1: zeroed GridSync of this job
    unsigned long long* words;    // team > 1: zeroed team_words_bytes(team)
    const uint32_t* ready;        // nonzero once the matrix's CSR is in device memory (written by a
                                  // host-to-device copy after the CSR's copies); nullptr: already there
    uint2* e2;                    // nnz edge records for the one-group engine (solo.cuh), or nullptr
    uint32_t* inv;                // n words (the solo engine's inverse permutation)
    uint32_t* gvis;               // ceil(n / 32) words: the solo engine's visited bitmap when n > kSoloMaxN
};

// One entry of the batch work list: member `rank` of job `job`'s team.
struct BatchSlot {
    uint32_t job, rank;
};

struct Options {
    uint32_t start;         // kUnvisited = automatic
    uint32_t reverse;
    uint32_t want_bw;
    uint32_t outnodes;      // peripheral: nodes kept per pass (32)
    unsigned long long wait_ns;
    uint32_t phantom;       // extra CTAs a grid barrier waits for (test hook)
    uint32_t mode;          // kModeFull, or kModeStartOnly: stop after the start search
    uint32_t solo_edges;    // a level with at most this many edges runs on CTA 0 alone
    uint32_t solo_parents;  // ... and at most this many parents
    uint32_t barrier;       // team barrier: 0 counter, 1 flag array
    uint32_t spec_from;     // speculative split from this search pass on (0: only for solo-dominated matrices)
    uint32_t wide_at;       // first BFS pass (key base 2 nnz + 3): a level of at least this many nodes
                            // hands the matrix to the level-synchronous engine (kNeedWide; 0 = never)
    unsigned long long data_wait_ns;  // batch kernels: bound of the wait for a matrix's CSR to arrive
};

// State of the level-synchronous engine (wide.cu), one per matrix in device
// memory: the level being expanded and the start-search bookkeeping, advanced
// by one kernel after every level.
enum : uint32_t { kWideSearch = 0, kWideFinal = 1, kWideDone = 2 };
struct alignas(16) WideState {
    uint32_t a, b, Ka, Kb;       // frontier positions [a, b), its edge ids [Ka, Kb)
    uint32_t L, last_start;      // level index in the pass, first position of the newest level
    uint32_t phase;              // kWideSearch / kWideFinal / kWideDone
    uint32_t base;               // key base of the pass
    uint32_t start, passes, ecc, lastdist;
    uint32_t pid;                // pass number in the claim key space
    uint32_t steps;              // level steps run (bounded by the host)
    uint32_t ticket;             // CTAs of the place kernel done with this step
    uint32_t prev_levels;        // levels of the last finished pass (the host sizes its batches by it)
};

constexpr uint32_t kModeFull = 0;
constexpr uint32_t kModeStartOnly = 1;

}  // namespace pbrcm
