// types.h -- plain data shared by the engine's device code and host code.
#pragma once

#include <cstdint>

namespace pbrcm {

constexpr uint32_t kUnvisited = 0xFFFFFFFFu;
constexpr uint32_t kFull = 0xFFFFFFFFu;

enum : uint32_t {
    kOk = 0,
    kErrArg = 1,
    kErrDisconnected = 2,
    kErrTimeout = 3,
    kErrCheck = 8,
    kNeedHub = 100,  // internal: relaunch with hub scratch
};

// One record per queue position: node, row start, valence, edge base.
struct alignas(16) PosRec {
    uint32_t node, rs, deg, ebase;
};

// Grid barrier state: reset to zero before every cooperative launch.
struct alignas(128) GridSync {
    unsigned int arrive;
    unsigned int gen;
    unsigned int pad[30];
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
    unsigned long long bandwidth;      // max |inv[i]-inv[j]|
    unsigned long long initial_bw;
    unsigned long long profile_lo;     // sum inv[i] - min(inv[row])   (CM order)
    unsigned long long profile_hi;     // sum max(inv[row]) - inv[i]   (reversed order)
};

// One matrix as the engine sees it.
struct MatrixView {
    const uint32_t* __restrict__ rp;   // n+1
    const uint32_t* __restrict__ ci;   // nnz
    uint32_t n;
    uint32_t nnz;                      // < 2^32 - 1 (checked by the host)
    uint32_t* claim;                   // n   (reused as the inverse permutation)
    PosRec* rec;                       // n
    uint32_t* perm;                    // n   output
    uint32_t* hub;                     // 4 * nnz hub scratch, or nullptr if no hub can occur
    DevResult* res;
};

struct Options {
    uint32_t start;         // kUnvisited = automatic
    uint32_t reverse;
    uint32_t want_bw;
    uint32_t outnodes;      // peripheral: nodes kept per pass (32)
    unsigned long long wait_ns;
    uint32_t phantom;       // extra CTAs a grid barrier waits for (test hook)
    uint32_t mode;          // kModeFull, or kModeStartOnly: stop after the start search
};

constexpr uint32_t kModeFull = 0;
constexpr uint32_t kModeStartOnly = 1;

}  // namespace pbrcm
