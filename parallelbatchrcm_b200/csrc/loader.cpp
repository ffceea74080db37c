// loader.cpp -- MatrixMarket input with the reference loader's semantics.
//
// Graph<T>::load (include/Graph.h:266-332) = loadMTX (src/COO.cpp:89-199) ->
// convert COO->CSR sorted by (row, col), duplicates kept (src/CSR.cpp:170-200)
// -> prepareRCM(!symmetric) (include/Graph.h:74-264): symmetry repair for
// non-symmetric files, then a connectivity repair that links every further
// component.  The reference also writes .hicsr cache files next to the input
// and prefers a stale cache on the next run; this loader writes nothing.
//
// Differences, all on inputs where the reference misbehaves:
//  - an index of 0 or past the declared size, or more entries than declared,
//    is PBRCM_ERR_FORMAT (the reference writes out of bounds);
//  - a linked node that no entry leads back to (an empty row) is marked
//    visited (the reference's connectivity loop never ends on it).
#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/pbrcm.h"

namespace {

struct CsrBuf {
    uint32_t n = 0;
    std::vector<uint32_t> rp, ci;
};

// Sorts each row's columns (rows are short: insertion sort; long rows:
// std::sort).
void sort_rows(CsrBuf& out)
{
    for (uint32_t r = 0; r < out.n; ++r) {
        uint32_t* b = out.ci.data() + out.rp[r];
        uint32_t* e = out.ci.data() + out.rp[r + 1];
        if (e - b > 32) {
            std::sort(b, e);
            continue;
        }
        for (uint32_t* i = b + 1; i < e; ++i) {
            const uint32_t v = *i;
            uint32_t* j = i;
            while (j > b && *(j - 1) > v) {
                *j = *(j - 1);
                --j;
            }
            *j = v;
        }
    }
}

// COO (row, col) pairs, in one or more runs -> CSR sorted by (row, col),
// duplicates kept: a counting sort by row, then each row's columns sorted.
void coo_to_csr(uint32_t n, const std::vector<const std::vector<uint64_t>*>& runs, CsrBuf& out)
{
    out.n = n;
    out.rp.assign((size_t)n + 1, 0);
    size_t total = 0;
    for (const auto* run : runs) {
        total += run->size();
        for (uint64_t k : *run)
            out.rp[(k >> 32) + 1]++;
    }
    for (uint32_t i = 0; i < n; ++i)
        out.rp[i + 1] += out.rp[i];
    out.ci.resize(total);
    std::vector<uint32_t> fill(out.rp.begin(), out.rp.end() - 1);
    for (const auto* run : runs)
        for (uint64_t k : *run)
            out.ci[fill[k >> 32]++] = (uint32_t)(k & 0xFFFFFFFFull);
    sort_rows(out);
}

void coo_to_csr(uint32_t n, std::vector<uint64_t>& keys, CsrBuf& out)
{
    coo_to_csr(n, std::vector<const std::vector<uint64_t>*>{&keys}, out);
}

inline uint64_t pair_key(uint32_t r, uint32_t c)
{
    uint32_t a = r < c ? r : c, b = r < c ? c : r;
    return ((uint64_t)a << 32) | b;
}

// prepareRCM (include/Graph.h:74-264).
int32_t prepare(CsrBuf& m, bool check_sym)
{
    const uint32_t n = m.n;
    if (check_sym && !m.ci.empty()) {
        // pairs {r,c}, r != c, stored an odd number of times are "missing"
        std::vector<uint64_t> keys;
        keys.reserve(m.ci.size());
        for (uint32_t r = 0; r < n; ++r)
            for (uint32_t k = m.rp[r]; k < m.rp[r + 1]; ++k)
                if (m.ci[k] != r)
                    keys.push_back(pair_key(r, m.ci[k]));
        std::sort(keys.begin(), keys.end());
        std::vector<uint64_t> odd;
        for (size_t i = 0; i < keys.size();) {
            size_t j = i;
            while (j < keys.size() && keys[j] == keys[i])
                ++j;
            if ((j - i) & 1)
                odd.push_back(keys[i]);
            i = j;
        }
        if (!odd.empty()) {
            std::vector<uint64_t> coo;
            coo.reserve(m.ci.size() + odd.size());
            for (uint32_t r = 0; r < n; ++r)
                for (uint32_t k = m.rp[r]; k < m.rp[r + 1]; ++k) {
                    const uint32_t c = m.ci[k];
                    coo.push_back(((uint64_t)r << 32) | c);
                    if (c != r && std::binary_search(odd.begin(), odd.end(), pair_key(r, c)))
                        coo.push_back(((uint64_t)c << 32) | r);
                }
            coo_to_csr(n, coo, m);
        }
    }
    // connectivity repair
    uint32_t minn = n;
    for (uint32_t r = 0; r < n; ++r)
        if (m.rp[r + 1] != m.rp[r]) {
            minn = r;
            break;
        }
    if (minn == n)
        return n ? PBRCM_ERR_FORMAT : PBRCM_OK;
    std::vector<uint8_t> vis(n, 0);
    std::vector<uint32_t> q;
    q.reserve(n);
    std::vector<std::pair<uint32_t, uint32_t>> links;
    size_t numv = 1, qh = 0;
    q.push_back(minn);
    vis[minn] = 1;
    uint32_t scan_from = 0, pending = 0xFFFFFFFFu;
    while (numv != n) {
        while (qh < q.size()) {
            const uint32_t v = q[qh++];
            for (uint32_t k = m.rp[v]; k < m.rp[v + 1]; ++k) {
                const uint32_t c = m.ci[k];
                if (!vis[c]) {
                    vis[c] = 1;
                    q.push_back(c);
                    ++numv;
                }
            }
        }
        if (pending != 0xFFFFFFFFu && !vis[pending]) {
            vis[pending] = 1;
            ++numv;
        }
        pending = 0xFFFFFFFFu;
        if (numv != n) {
            uint32_t i = scan_from;
            while (vis[i])
                ++i;
            scan_from = i;
            bool connected = false;
            for (uint32_t j = i; j > 0; --j)
                if (vis[j - 1]) {
                    links.emplace_back(j - 1, i);
                    connected = true;
                    break;
                }
            if (!connected)
                for (uint32_t j = i + 1; j < n; ++j)
                    if (vis[j]) {
                        links.emplace_back(i, j);
                        break;
                    }
            q.clear();
            qh = 0;
            q.push_back(i);
            pending = i;
        }
    }
    if (!links.empty()) {
        std::vector<uint64_t> coo;
        coo.reserve(m.ci.size() + 2 * links.size());
        for (uint32_t r = 0; r < n; ++r)
            for (uint32_t k = m.rp[r]; k < m.rp[r + 1]; ++k)
                coo.push_back(((uint64_t)r << 32) | m.ci[k]);
        for (auto& l : links) {
            coo.push_back(((uint64_t)l.second << 32) | l.first);
            coo.push_back(((uint64_t)l.first << 32) | l.second);
        }
        coo_to_csr(n, coo, m);
    }
    return PBRCM_OK;
}

// Fast unsigned / float token skipping for the MatrixMarket body.
inline const char* skip_ws(const char* p, const char* e)
{
    while (p < e && (*p == ' ' || *p == '\t' || *p == '\r'))
        ++p;
    return p;
}

inline bool parse_u64(const char*& p, const char* e, unsigned long long& v)
{
    p = skip_ws(p, e);
    if (p >= e || !std::isdigit((unsigned char)*p))
        return false;
    unsigned long long x = 0;
    while (p < e && std::isdigit((unsigned char)*p)) {
        x = x * 10 + (unsigned)(*p - '0');
        if (x > 0xFFFFFFFFFFFFull)
            return false;
        ++p;
    }
    v = x;
    return true;
}

// A value token must read as one number up to the next white space (the
// buffer ends in a NUL, so strtod stops at the latest there).
inline bool skip_number(const char*& p, const char* e)
{
    p = skip_ws(p, e);
    const char* s = p;
    while (p < e && !std::isspace((unsigned char)*p))
        ++p;
    if (p == s)
        return false;
    char* end = nullptr;
    std::strtod(s, &end);
    return end == p;
}

// Body lines [b, e) (b at a line start) -> (row, col) keys; counts entries.
struct ParseOut {
    std::vector<uint64_t> coo;
    unsigned long long entries = 0;
    int32_t rc = PBRCM_OK;
};

void parse_body(const char* b, const char* e, bool pattern, bool sym, unsigned long long nr, ParseOut& o)
{
    const char* p = b;
    while (p < e) {
        const char* nl = static_cast<const char*>(std::memchr(p, '\n', (size_t)(e - p)));
        const char* le = nl ? nl : e;
        const char* ls = p;
        p = nl ? nl + 1 : e;
        if (ls < le && *ls == '%')
            continue;
        const char* q = skip_ws(ls, le);
        if (q >= le)
            continue;
        unsigned long long r, c;
        if (!parse_u64(q, le, r) || !parse_u64(q, le, c) || (!pattern && !skip_number(q, le)) || r == 0 || c == 0 ||
            r > nr || c > nr) {
            o.rc = PBRCM_ERR_FORMAT;
            return;
        }
        ++o.entries;
        o.coo.push_back(((r - 1) << 32) | (c - 1));
        if (sym && r != c)
            o.coo.push_back(((c - 1) << 32) | (r - 1));
    }
}

int32_t load_mtx(const char* path, CsrBuf& out)
{
    FILE* f = std::fopen(path, "rb");
    if (!f)
        return PBRCM_ERR_IO;
    std::fseek(f, 0, SEEK_END);
    long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (sz < 0) {
        std::fclose(f);
        return PBRCM_ERR_IO;
    }
    std::string buf((size_t)sz, '\0');
    size_t got = std::fread(&buf[0], 1, (size_t)sz, f);
    std::fclose(f);
    if (got != (size_t)sz)
        return PBRCM_ERR_IO;
    const char* p = buf.data();
    const char* e = p + buf.size();
    auto next_line = [&](const char*& ls, const char*& le) -> bool {
        if (p >= e)
            return false;
        ls = p;
        const char* nl = static_cast<const char*>(std::memchr(p, '\n', (size_t)(e - p)));
        le = nl ? nl : e;
        p = nl ? nl + 1 : e;
        return true;
    };
    const char *ls, *le;
    if (!next_line(ls, le))
        return PBRCM_ERR_FORMAT;
    std::string header(ls, le);
    if (header.compare(0, 32, "%%MatrixMarket matrix coordinate") != 0)
        return PBRCM_ERR_FORMAT;
    char t0[64], t1[64], t2[64], dtype[64], symm[64];
    if (std::sscanf(header.c_str(), "%63s %63s %63s %63s %63s", t0, t1, t2, dtype, symm) != 5)
        return PBRCM_ERR_FORMAT;
    const bool pattern = std::strcmp(dtype, "pattern") == 0;
    if (!pattern && std::strcmp(dtype, "real") && std::strcmp(dtype, "integer") && std::strcmp(dtype, "complex"))
        return PBRCM_ERR_FORMAT;
    bool symmetric = false, hermitian = false;
    if (!std::strcmp(symm, "symmetric"))
        symmetric = true;
    else if (!std::strcmp(symm, "Hermitian"))
        hermitian = true;
    else if (std::strcmp(symm, "general"))
        return PBRCM_ERR_FORMAT;
    unsigned long long nr = 0, nc = 0, nz = 0;
    for (;;) {
        if (!next_line(ls, le))
            return PBRCM_ERR_FORMAT;
        if (ls < le && *ls == '%')
            continue;
        const char* q = ls;
        if (!parse_u64(q, le, nr) || !parse_u64(q, le, nc) || !parse_u64(q, le, nz))
            return PBRCM_ERR_FORMAT;
        break;
    }
    if (nr != nc || nr == 0 || nr >= 0xFFFFFFFFull)
        return PBRCM_ERR_FORMAT;
    // the body in parallel: chunks of whole lines, one thread each
    const size_t body = (size_t)(e - p);
    unsigned threads = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (body < (1u << 20))
        threads = 1;
    std::vector<const char*> cut(threads + 1);
    cut[0] = p;
    cut[threads] = e;
    for (unsigned t = 1; t < threads; ++t) {
        const char* c = p + body * t / threads;
        c = std::max(c, cut[t - 1]);
        const char* nl = c < e ? static_cast<const char*>(std::memchr(c, '\n', (size_t)(e - c))) : nullptr;
        cut[t] = nl ? nl + 1 : e;
    }
    std::vector<ParseOut> parts(threads);
    const bool sym = symmetric || hermitian;
    for (unsigned t = 0; t < threads; ++t)
        parts[t].coo.reserve((size_t)((cut[t + 1] - cut[t]) / 8) * (sym ? 2 : 1));
    if (threads == 1) {
        parse_body(cut[0], cut[1], pattern, sym, nr, parts[0]);
    } else {
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < threads; ++t)
            pool.emplace_back(parse_body, cut[t], cut[t + 1], pattern, sym, nr, std::ref(parts[t]));
        for (auto& th : pool)
            th.join();
    }
    unsigned long long entries = 0;
    std::vector<const std::vector<uint64_t>*> runs;
    for (auto& part : parts) {
        if (part.rc != PBRCM_OK)
            return part.rc;
        entries += part.entries;
        runs.push_back(&part.coo);
    }
    if (entries > nz)
        return PBRCM_ERR_FORMAT;  // more entries than the size line declares
    coo_to_csr((uint32_t)nr, runs, out);
    return prepare(out, !symmetric);
}

int32_t export_csr(CsrBuf& m, uint64_t* nnz, uint32_t** rp, uint32_t** ci)
{
    *rp = static_cast<uint32_t*>(std::malloc(sizeof(uint32_t) * ((size_t)m.n + 1)));
    *ci = static_cast<uint32_t*>(std::malloc(sizeof(uint32_t) * std::max<size_t>(m.ci.size(), 1)));
    if (!*rp || !*ci) {
        std::free(*rp);
        std::free(*ci);
        *rp = *ci = nullptr;
        return PBRCM_ERR_OOM;
    }
    std::memcpy(*rp, m.rp.data(), sizeof(uint32_t) * ((size_t)m.n + 1));
    if (!m.ci.empty())
        std::memcpy(*ci, m.ci.data(), sizeof(uint32_t) * m.ci.size());
    *nnz = m.ci.size();
    return PBRCM_OK;
}

}  // namespace

extern "C" {

int32_t pbrcm_load_mtx(const char* path, uint32_t* n, uint64_t* nnz, uint32_t** row_ptr, uint32_t** col_idx)
{
    if (!path || !n || !nnz || !row_ptr || !col_idx)
        return PBRCM_ERR_ARG;
    CsrBuf m;
    int32_t rc;
    try {
        rc = load_mtx(path, m);
    } catch (std::bad_alloc&) {
        return PBRCM_ERR_OOM;
    }
    if (rc != PBRCM_OK)
        return rc;
    *n = m.n;
    return export_csr(m, nnz, row_ptr, col_idx);
}

int32_t pbrcm_prepare_csr(const uint32_t* row_ptr, const uint32_t* col_idx, uint32_t n, uint64_t nnz,
                          int32_t check_symmetry, uint64_t* nnz_out, uint32_t** row_ptr_out, uint32_t** col_idx_out)
{
    if (!row_ptr || (!col_idx && nnz) || !nnz_out || !row_ptr_out || !col_idx_out || n == 0)
        return PBRCM_ERR_ARG;
    if (row_ptr[0] != 0 || row_ptr[n] != nnz)
        return PBRCM_ERR_ARG;
    CsrBuf m;
    try {
        m.n = n;
        m.rp.assign(row_ptr, row_ptr + (size_t)n + 1);
        m.ci.assign(col_idx, col_idx + nnz);
        for (uint32_t i = 0; i < n; ++i)
            if (m.rp[i + 1] < m.rp[i])
                return PBRCM_ERR_ARG;
        for (uint32_t c : m.ci)
            if (c >= n)
                return PBRCM_ERR_ARG;
        int32_t rc = prepare(m, check_symmetry != 0);
        if (rc != PBRCM_OK)
            return rc;
    } catch (std::bad_alloc&) {
        return PBRCM_ERR_OOM;
    }
    return export_csr(m, nnz_out, row_ptr_out, col_idx_out);
}

void pbrcm_free(void* p) { std::free(p); }

// The reference's binary CSR cache (.hicsr, src/CSR.cpp:57-168): a header
// of a 9-byte magic and eight u64 fields (type size, compressed direction,
// index size, fixed offset, offset size, rows, columns, non-zeros), the
// State<T> {scaling, transpose} record, then values, column ids, row offsets.
namespace {
const char kHiMagic[9] = {'H', 'i', 1, 'C', 'o', 'm', 'p', 's', 'd'};
struct HiHeader {
    char magic[9];
    char pad[7];
    uint64_t typesize, compresseddir, indexsize, fixedoffset, offsetsize, rows, cols, nnz;
};
static_assert(sizeof(HiHeader) == 80, "hicsr header layout");
size_t hi_state_bytes(uint64_t typesize) { return typesize == 8 ? 16 : 8; }  // {T scaling; bool transpose}
}  // namespace

int32_t pbrcm_load_hicsr(const char* path, uint32_t* n, uint64_t* nnz, uint32_t** row_ptr, uint32_t** col_idx,
                         void** vals, uint32_t* val_bytes)
{
    if (!path || !n || !nnz || !row_ptr || !col_idx)
        return PBRCM_ERR_ARG;
    std::FILE* f = std::fopen(path, "rb");
    if (!f)
        return PBRCM_ERR_NOT_FOUND;
    HiHeader h;
    unsigned char state[16];
    int32_t rc = PBRCM_OK;
    uint32_t *rp = nullptr, *ci = nullptr;
    void* v = nullptr;
    if (std::fread(&h, sizeof(h), 1, f) != 1 || std::memcmp(h.magic, kHiMagic, 9) != 0 ||
        (h.typesize != 4 && h.typesize != 8) || h.indexsize != 4 || h.offsetsize != 4 || h.compresseddir != 0 ||
        h.rows != h.cols || h.rows == 0 || h.rows >= 0xFFFFFFFFull || h.nnz > 0xFFFFFFF0ull ||
        std::fread(state, hi_state_bytes(h.typesize), 1, f) != 1) {
        rc = PBRCM_ERR_FORMAT;
    } else {
        rp = static_cast<uint32_t*>(std::malloc(4 * (h.rows + 1)));
        ci = static_cast<uint32_t*>(std::malloc(4 * std::max<uint64_t>(h.nnz, 1)));
        v = std::malloc(h.typesize * std::max<uint64_t>(h.nnz, 1));
        if (!rp || !ci || !v)
            rc = PBRCM_ERR_OOM;
        else if (std::fread(v, h.typesize, h.nnz, f) != h.nnz || std::fread(ci, 4, h.nnz, f) != h.nnz ||
                 std::fread(rp, 4, h.rows + 1, f) != h.rows + 1)
            rc = PBRCM_ERR_FORMAT;
        else if (rp[0] != 0 || rp[h.rows] != h.nnz)
            rc = PBRCM_ERR_FORMAT;
    }
    std::fclose(f);
    if (rc != PBRCM_OK) {
        std::free(rp);
        std::free(ci);
        std::free(v);
        return rc;
    }
    *n = (uint32_t)h.rows;
    *nnz = h.nnz;
    *row_ptr = rp;
    *col_idx = ci;
    if (vals) {
        *vals = v;
    } else {
        std::free(v);
    }
    if (val_bytes)
        *val_bytes = (uint32_t)h.typesize;
    return PBRCM_OK;
}

int32_t pbrcm_store_hicsr(const char* path, uint32_t n, uint64_t nnz, const uint32_t* row_ptr, const uint32_t* col_idx,
                          const void* vals, uint32_t val_bytes)
{
    if (!path || !row_ptr || (!col_idx && nnz) || (val_bytes != 0 && val_bytes != 4 && val_bytes != 8) ||
        (val_bytes && nnz && !vals) || row_ptr[n] != nnz)
        return PBRCM_ERR_ARG;
    HiHeader h;
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.magic, kHiMagic, 9);
    h.typesize = val_bytes ? val_bytes : 4;  // no values: float 1.0, the reference's pattern data
    h.indexsize = 4;
    h.offsetsize = 4;
    h.rows = h.cols = n;
    h.nnz = nnz;
    unsigned char state[16];
    std::memset(state, 0, sizeof(state));
    if (h.typesize == 8) {
        const double one = 1.0;
        std::memcpy(state, &one, 8);
    } else {
        const float one = 1.0f;
        std::memcpy(state, &one, 4);
    }
    std::FILE* f = std::fopen(path, "wb");
    if (!f)
        return PBRCM_ERR_IO;
    bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1 && std::fwrite(state, hi_state_bytes(h.typesize), 1, f) == 1;
    if (ok && val_bytes) {
        ok = std::fwrite(vals, val_bytes, nnz, f) == nnz;
    } else if (ok) {
        const float one = 1.0f;
        for (uint64_t k = 0; k < nnz && ok; ++k)
            ok = std::fwrite(&one, 4, 1, f) == 1;
    }
    ok = ok && std::fwrite(col_idx, 4, nnz, f) == nnz && std::fwrite(row_ptr, 4, (size_t)n + 1, f) == (size_t)n + 1;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? PBRCM_OK : PBRCM_ERR_IO;
}

int32_t pbrcm_store_mtx(const char* path, uint32_t n, uint64_t nnz, const uint32_t* row_ptr, const uint32_t* col_idx,
                        const void* vals, uint32_t val_bytes)
{
    if (!path || !row_ptr || (!col_idx && nnz) || (val_bytes != 0 && val_bytes != 4 && val_bytes != 8) ||
        (val_bytes && nnz && !vals) || row_ptr[n] != nnz)
        return PBRCM_ERR_ARG;
    std::FILE* f = std::fopen(path, "wb");
    if (!f)
        return PBRCM_ERR_IO;
    std::string buf;
    buf.reserve(1 << 22);
    buf += val_bytes ? "%%MatrixMarket matrix coordinate real general\n"
                     : "%%MatrixMarket matrix coordinate pattern general\n";
    buf += std::to_string(n) + " " + std::to_string(n) + " " + std::to_string(nnz) + "\n";
    bool ok = true;
    for (uint32_t r = 0; r < n && ok; ++r) {
        for (uint32_t k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
            buf += std::to_string((unsigned long)r + 1);
            buf += ' ';
            buf += std::to_string((unsigned long)col_idx[k] + 1);
            if (val_bytes == 4) {
                buf += ' ';
                buf += std::to_string(static_cast<const float*>(vals)[k]);
            } else if (val_bytes == 8) {
                buf += ' ';
                buf += std::to_string(static_cast<const double*>(vals)[k]);
            }
            buf += '\n';
        }
        if (buf.size() >= (1u << 22)) {
            ok = std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
            buf.clear();
        }
    }
    ok = ok && std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
    ok = (std::fclose(f) == 0) && ok;
    return ok ? PBRCM_OK : PBRCM_ERR_IO;
}

}  // extern "C"
