/*
 * pbrcm_oracle.c -- TEST INFRASTRUCTURE ONLY (the parity oracle).
 *
 * A plain-C, single-threaded restatement of the reference's CPU path for
 * Reverse Cuthill-McKee (GPUPeople/ParallelBatchRCM).  Only tests/,
 * __graft_entry__.smoke() and the cpu_baseline leg of bench.py may load this
 * file's shared library, and only as the checker.  Nothing in the product
 * (parallelbatchrcm_b200/, include/) links or calls it.
 *
 * Every function names the reference file:line range it restates.  Where the
 * reference has undefined behaviour (empty rows, a one-node graph, an
 * isolated row in the connectivity repair), the oracle defines the outcome and
 * says so next to the code; the product engine follows the same definitions.
 *
 * Parity of this restatement is pinned against the reference's own sources,
 * compiled unchanged into oracle/_ref/ by oracle/Makefile, through the golden
 * fixtures in tests/golden/ (tests/test_oracle_golden.py).
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <ctype.h>

#define ORC_OK 0
#define ORC_ERR_ARG (-1)
#define ORC_ERR_DISCONNECTED (-2)
#define ORC_ERR_IO (-3)
#define ORC_ERR_FORMAT (-4)
#define ORC_ERR_NOMEM (-5)

typedef struct {
    uint32_t key;
    uint32_t val;
} orc_kv;

/* Stable merge sort of (key,val) by key; ties keep their input order, as
 * std::stable_sort does in rcm_cpu.cpp:94-95. */
static void orc_stable_sort(orc_kv *a, orc_kv *tmp, size_t m)
{
    if (m < 2)
        return;
    if (m <= 16) {
        for (size_t i = 1; i < m; ++i) {
            orc_kv x = a[i];
            size_t j = i;
            while (j > 0 && a[j - 1].key > x.key) {
                a[j] = a[j - 1];
                --j;
            }
            a[j] = x;
        }
        return;
    }
    size_t h = m / 2;
    orc_stable_sort(a, tmp, h);
    orc_stable_sort(a + h, tmp, m - h);
    size_t i = 0, j = h, k = 0;
    while (i < h && j < m)
        tmp[k++] = (a[j].key < a[i].key) ? a[j++] : a[i++];
    while (i < h)
        tmp[k++] = a[i++];
    while (j < m)
        tmp[k++] = a[j++];
    memcpy(a, tmp, m * sizeof(orc_kv));
}

/*
 * Cuthill-McKee order from `start` (rcm_cpu.cpp:57-104, rcm_seq<STABLE=true>).
 * FIFO queue; each parent appends its still-unvisited neighbours in CSR-row
 * order, stable-sorted by valence = row length (Graph.h:57-60, includes the
 * diagonal and any duplicate entries).  With sort_by_degree == 0 the children
 * keep row order: that is the discovery order of the FIFO BFS in
 * simple_peripheral.cpp:44-90.  perm[k] = original node at new position k (the
 * reference's output is this CM order; its -r flag is parsed but never read,
 * main.cpp:250).  Returns the number of nodes placed (n when connected).
 */
int64_t orc_cm_order(uint32_t n, const uint32_t *rp, const uint32_t *ci, uint32_t start,
                     int sort_by_degree, uint32_t *perm)
{
    if (n == 0 || start >= n)
        return ORC_ERR_ARG;
    uint8_t *visited = (uint8_t *)calloc(n, 1);
    uint32_t maxdeg = 0;
    for (uint32_t v = 0; v < n; ++v)
        if (rp[v + 1] - rp[v] > maxdeg)
            maxdeg = rp[v + 1] - rp[v];
    orc_kv *tmpv = (orc_kv *)malloc(sizeof(orc_kv) * (size_t)(maxdeg + 1));
    orc_kv *tmps = (orc_kv *)malloc(sizeof(orc_kv) * (size_t)(maxdeg + 1));
    if (!visited || !tmpv || !tmps) {
        free(visited); free(tmpv); free(tmps);
        return ORC_ERR_NOMEM;
    }
    size_t head = 0, tail = 0;
    perm[tail++] = start;
    visited[start] = 1;
    while (head < tail) {
        uint32_t v = perm[head++];
        size_t m = 0;
        for (uint32_t k = rp[v]; k < rp[v + 1]; ++k) {
            uint32_t c = ci[k];
            if (!visited[c]) {
                visited[c] = 1;
                tmpv[m].key = rp[c + 1] - rp[c];
                tmpv[m].val = c;
                ++m;
            }
        }
        if (sort_by_degree)
            orc_stable_sort(tmpv, tmps, m);
        for (size_t i = 0; i < m; ++i)
            perm[tail++] = tmpv[i].val;
    }
    free(visited); free(tmpv); free(tmps);
    return (int64_t)tail;
}

/*
 * FIFO BFS of simple_peripheral.cpp:44-90 (findMaxDistance).  Keeps the last
 * `outputnodes` discovered nodes (never the start) with their distances, in
 * discovery order.  Returns the number recorded, or ORC_ERR_DISCONNECTED when
 * not every node is reached (the reference throws, :85-89).
 */
static int64_t orc_find_max_distance(uint32_t n, const uint32_t *rp, const uint32_t *ci,
                                     uint32_t start, uint32_t outputnodes, uint32_t *nodes,
                                     uint32_t *dists, uint32_t *qn, uint32_t *dist)
{
    for (uint32_t i = 0; i < n; ++i)
        dist[i] = 0xFFFFFFFFu;
    size_t to_visit = (size_t)n - 1;
    size_t head = 0, tail = 0, rec = 0;
    qn[tail++] = start;
    dist[start] = 0;
    while (head < tail) {
        uint32_t v = qn[head++];
        uint32_t nd = dist[v] + 1;
        for (uint32_t k = rp[v]; k < rp[v + 1]; ++k) {
            uint32_t c = ci[k];
            if (dist[c] == 0xFFFFFFFFu) {
                dist[c] = nd;
                qn[tail++] = c;
                if (--to_visit < outputnodes) {
                    nodes[rec] = c;
                    dists[rec] = nd;
                    ++rec;
                }
            }
        }
    }
    if (to_visit > 0)
        return ORC_ERR_DISCONNECTED;
    return (int64_t)rec;
}

/*
 * Pseudo-peripheral start node (simple_peripheral.cpp:92-141, findPeripheral,
 * outputnodes = 32 by default, simple_peripheral.h:46).  Starts at rows/2;
 * repeats the BFS until the largest recorded distance equals the previous one
 * (initially 0) and returns that BFS's start.  Otherwise the next start is,
 * among the recorded nodes from the first one at maximal distance, the last
 * one of minimal valence (:118-127: `min(...) == valence` also fires on ties).
 * A one-node graph records nothing (the reference then reads back() of an
 * empty vector); the oracle defines the result as node 0 after one pass.
 * iters_out = BFS passes run, ecc_out = eccentricity of the returned node.
 */
int64_t orc_peripheral(uint32_t n, const uint32_t *rp, const uint32_t *ci, uint32_t outputnodes,
                       uint32_t *iters_out, uint32_t *ecc_out)
{
    if (n == 0 || outputnodes == 0)
        return ORC_ERR_ARG;
    uint32_t *nodes = (uint32_t *)malloc(sizeof(uint32_t) * outputnodes);
    uint32_t *dists = (uint32_t *)malloc(sizeof(uint32_t) * outputnodes);
    uint32_t *qn = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)n);
    uint32_t *dist = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)n);
    if (!nodes || !dists || !qn || !dist) {
        free(nodes); free(dists); free(qn); free(dist);
        return ORC_ERR_NOMEM;
    }
    uint32_t lastdist = 0;
    uint32_t s = n / 2;
    uint32_t iters = 0, ecc = 0;
    int64_t ret = 0;
    for (;;) {
        ++iters;
        int64_t cnt = orc_find_max_distance(n, rp, ci, s, outputnodes, nodes, dists, qn, dist);
        if (cnt < 0) {
            ret = cnt;
            break;
        }
        if (cnt == 0) { /* one-node graph */
            ecc = 0;
            ret = s;
            break;
        }
        if (dists[cnt - 1] == lastdist) {
            ecc = lastdist;
            ret = s;
            break;
        }
        size_t index = 0;
        for (size_t i = 1; i < (size_t)cnt; ++i)
            if (dists[i] > dists[index])
                index = i;
        int64_t minval = INT64_MAX;
        for (size_t i = index; i < (size_t)cnt; ++i) {
            int64_t val = (int64_t)(rp[nodes[i] + 1] - rp[nodes[i]]);
            if (val <= minval) {
                minval = val;
                s = nodes[i];
            }
        }
        lastdist = dists[cnt - 1];
    }
    if (iters_out)
        *iters_out = iters;
    if (ecc_out)
        *ecc_out = ecc;
    free(nodes); free(dists); free(qn); free(dist);
    return ret;
}

/*
 * Bandwidth of the reordered matrix (main.cpp:143-184, computeBandwidth):
 * max over stored entries (i,j), diagonal included, of |invp[i] - invp[j]|.
 * Empty rows are skipped (the reference reads a stale buffer for them).
 */
int64_t orc_bandwidth(uint32_t n, const uint32_t *rp, const uint32_t *ci, const uint32_t *perm)
{
    if (n == 0)
        return -1;
    uint32_t *inv = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)n);
    if (!inv)
        return ORC_ERR_NOMEM;
    for (uint32_t k = 0; k < n; ++k)
        inv[perm[k]] = k;
    int64_t bw = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (rp[i] == rp[i + 1])
            continue;
        uint32_t mn = 0xFFFFFFFFu, mx = 0;
        for (uint32_t k = rp[i]; k < rp[i + 1]; ++k) {
            uint32_t p = inv[ci[k]];
            if (p < mn) mn = p;
            if (p > mx) mx = p;
        }
        int64_t r = inv[i];
        int64_t lo = r - (int64_t)mn, hi = (int64_t)mx - r;
        int64_t b = lo > hi ? lo : hi;
        if (b > bw)
            bw = b;
    }
    free(inv);
    return bw;
}

/*
 * Bandwidth of the input as stored (main.cpp:114-129, checkBandwidth): per
 * row, the first and last stored column against the row index.  Matches the
 * true bandwidth for the sorted rows the loader produces.  Empty rows skipped.
 */
int64_t orc_initial_bandwidth(uint32_t n, const uint32_t *rp, const uint32_t *ci)
{
    int64_t bw = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (rp[i] == rp[i + 1])
            continue;
        int64_t lo = (int64_t)i - (int64_t)ci[rp[i]];
        int64_t hi = (int64_t)ci[rp[i + 1] - 1] - (int64_t)i;
        int64_t b = lo > hi ? lo : hi;
        if (b > bw)
            bw = b;
    }
    return bw;
}

/* Max row length (main.cpp:131-140, maxValency). */
int64_t orc_max_valency(uint32_t n, const uint32_t *rp)
{
    int64_t m = 0;
    for (uint32_t i = 0; i < n; ++i)
        if ((int64_t)(rp[i + 1] - rp[i]) > m)
            m = rp[i + 1] - rp[i];
    return m;
}

/*
 * Profile (envelope size) of the reordered matrix: sum over rows r of the
 * permuted matrix of r - (smallest column in row r), clamped at 0.  The
 * reference has no profile; this definition is the project's own.
 */
uint64_t orc_profile(uint32_t n, const uint32_t *rp, const uint32_t *ci, const uint32_t *perm)
{
    uint32_t *inv = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)n);
    if (!inv)
        return 0;
    for (uint32_t k = 0; k < n; ++k)
        inv[perm[k]] = k;
    uint64_t prof = 0;
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t r = inv[i], mn = r;
        for (uint32_t k = rp[i]; k < rp[i + 1]; ++k) {
            uint32_t p = inv[ci[k]];
            if (p < mn) mn = p;
        }
        prof += (uint64_t)(r - mn);
    }
    free(inv);
    return prof;
}

/* Bijection check (main.cpp:186-226, checkPermutation).  0 = valid, -1 = not.
 * The reference accepts element == n (an off-by-one, :193); the oracle does not. */
int orc_check_permutation(uint32_t n, const uint32_t *perm)
{
    uint8_t *seen = (uint8_t *)calloc(n ? n : 1, 1);
    if (!seen)
        return ORC_ERR_NOMEM;
    int ok = 0;
    for (uint32_t k = 0; k < n; ++k) {
        if (perm[k] >= n || seen[perm[k]]) {
            ok = -1;
            break;
        }
        seen[perm[k]] = 1;
    }
    free(seen);
    return ok;
}

/* ------------------------------------------------------------------------ */
/* Loader semantics: COO -> CSR (CSR.cpp:170-200) and Graph::prepareRCM     */
/* (Graph.h:74-264).  Values are not carried: RCM reads structure only.     */
/* ------------------------------------------------------------------------ */

static int orc_cmp_u64(const void *a, const void *b)
{
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

/* COO -> CSR sorted by (row, col), duplicates kept (CSR.cpp:170-200).
 * rp must hold rows+1 entries, ci nnz entries. */
int orc_coo_to_csr(uint32_t rows, uint64_t nnz, const uint32_t *r, const uint32_t *c,
                   uint32_t *rp, uint32_t *ci)
{
    uint64_t *e = (uint64_t *)malloc(sizeof(uint64_t) * (nnz ? nnz : 1));
    if (!e)
        return ORC_ERR_NOMEM;
    for (uint64_t i = 0; i < nnz; ++i) {
        if (r[i] >= rows) {
            free(e);
            return ORC_ERR_ARG;
        }
        e[i] = ((uint64_t)r[i] << 32) | c[i];
    }
    qsort(e, nnz, sizeof(uint64_t), orc_cmp_u64);
    memset(rp, 0, sizeof(uint32_t) * ((size_t)rows + 1));
    for (uint64_t i = 0; i < nnz; ++i) {
        ci[i] = (uint32_t)(e[i] & 0xFFFFFFFFu);
        rp[(e[i] >> 32) + 1]++;
    }
    for (uint32_t i = 0; i < rows; ++i)
        rp[i + 1] += rp[i];
    free(e);
    return ORC_OK;
}

typedef struct {
    uint32_t n;
    uint64_t nnz;
    uint32_t *rp;
    uint32_t *ci;
    uint32_t added_entries;  /* entries created by the symmetry repair */
    uint32_t added_links;    /* component links created by the connectivity repair */
} orc_csr;

void orc_csr_free(orc_csr *m)
{
    if (!m)
        return;
    free(m->rp);
    free(m->ci);
    m->rp = m->ci = NULL;
}

/*
 * Graph::prepareRCM(check_sym) (Graph.h:74-264) on a square CSR with sorted
 * rows.  (1) When check_sym: every off-diagonal pair {r,c} stored an odd
 * number of times is "missing" (the toggle map of :79-100); each stored entry
 * of such a pair gets its mirror added, then the CSR is rebuilt (:104-146).
 * (2) BFS from the first non-empty row; whenever nodes stay unvisited, the
 * first unvisited node i is linked to the nearest visited node below it (else
 * above it) and the BFS continues from i (:160-232); the links are added in
 * both directions and the CSR rebuilt (:233-262).  The reference never marks
 * i itself visited, so when no stored entry leads back to i (an empty row, or
 * an asymmetric pattern) it loops forever; the oracle marks such an i visited
 * after its BFS.  A matrix with no stored entry at all is rejected.
 */
int orc_prepare_rcm(orc_csr *m, int check_sym)
{
    uint32_t n = m->n;
    m->added_entries = 0;
    m->added_links = 0;
    if (check_sym && m->nnz) {
        uint64_t cnt = 0;
        uint64_t *keys = (uint64_t *)malloc(sizeof(uint64_t) * m->nnz);
        if (!keys)
            return ORC_ERR_NOMEM;
        for (uint32_t r = 0; r < n; ++r)
            for (uint32_t k = m->rp[r]; k < m->rp[r + 1]; ++k) {
                uint32_t c = m->ci[k];
                if (c == r)
                    continue;
                uint32_t a = r < c ? r : c, b = r < c ? c : r;
                keys[cnt++] = ((uint64_t)a << 32) | b;
            }
        qsort(keys, cnt, sizeof(uint64_t), orc_cmp_u64);
        /* compact to the list of keys with odd multiplicity */
        uint64_t odd = 0;
        for (uint64_t i = 0; i < cnt;) {
            uint64_t j = i;
            while (j < cnt && keys[j] == keys[i])
                ++j;
            if ((j - i) & 1)
                keys[odd++] = keys[i];
            i = j;
        }
        if (odd) {
            uint64_t extra = 0;
            for (uint32_t r = 0; r < n; ++r)
                for (uint32_t k = m->rp[r]; k < m->rp[r + 1]; ++k) {
                    uint32_t c = m->ci[k];
                    if (c == r)
                        continue;
                    uint32_t a = r < c ? r : c, b = r < c ? c : r;
                    uint64_t key = ((uint64_t)a << 32) | b;
                    if (bsearch(&key, keys, odd, sizeof(uint64_t), orc_cmp_u64))
                        ++extra;
                }
            uint64_t nn = m->nnz + extra;
            uint32_t *cr = (uint32_t *)malloc(sizeof(uint32_t) * nn);
            uint32_t *cc = (uint32_t *)malloc(sizeof(uint32_t) * nn);
            if (!cr || !cc) {
                free(keys); free(cr); free(cc);
                return ORC_ERR_NOMEM;
            }
            uint64_t w = 0;
            for (uint32_t r = 0; r < n; ++r)
                for (uint32_t k = m->rp[r]; k < m->rp[r + 1]; ++k) {
                    uint32_t c = m->ci[k];
                    cr[w] = r; cc[w] = c; ++w;
                    if (c == r)
                        continue;
                    uint32_t a = r < c ? r : c, b = r < c ? c : r;
                    uint64_t key = ((uint64_t)a << 32) | b;
                    if (bsearch(&key, keys, odd, sizeof(uint64_t), orc_cmp_u64)) {
                        cr[w] = c; cc[w] = r; ++w;
                    }
                }
            uint32_t *nci = (uint32_t *)malloc(sizeof(uint32_t) * nn);
            if (!nci) {
                free(keys); free(cr); free(cc);
                return ORC_ERR_NOMEM;
            }
            int rc = orc_coo_to_csr(n, nn, cr, cc, m->rp, nci);
            free(cr); free(cc);
            if (rc) {
                free(keys); free(nci);
                return rc;
            }
            free(m->ci);
            m->ci = nci;
            m->nnz = nn;
            m->added_entries = (uint32_t)extra;
        }
        free(keys);
    }

    /* connectivity repair */
    uint32_t minn = n;
    for (uint32_t r = 0; r < n; ++r)
        if (m->rp[r + 1] != m->rp[r]) {
            minn = r;
            break;
        }
    if (minn == n)
        return n ? ORC_ERR_ARG : ORC_OK;
    uint8_t *vis = (uint8_t *)calloc(n, 1);
    uint32_t *q = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)n + 1));
    uint32_t *links = (uint32_t *)malloc(sizeof(uint32_t) * 2 * (size_t)n);
    if (!vis || !q || !links) {
        free(vis); free(q); free(links);
        return ORC_ERR_NOMEM;
    }
    size_t qh = 0, qt = 0, nl = 0, numv = 0;
    q[qt++] = minn;
    vis[minn] = 1;
    ++numv;
    size_t scan_from = 0;
    uint32_t pending = 0xFFFFFFFFu;
    while (numv != n) {
        while (qh < qt) {
            uint32_t v = q[qh++];
            for (uint32_t k = m->rp[v]; k < m->rp[v + 1]; ++k) {
                uint32_t c = m->ci[k];
                if (!vis[c]) {
                    vis[c] = 1;
                    q[qt++] = c;
                    ++numv;
                }
            }
        }
        if (pending != 0xFFFFFFFFu && !vis[pending]) {
            /* the BFS from the linked node did not come back to it (no entry
             * leads to it): see the header comment */
            vis[pending] = 1;
            ++numv;
        }
        pending = 0xFFFFFFFFu;
        if (numv != n) {
            /* all nodes below scan_from are visited, so this finds the same
             * first unvisited node as the reference's rescan from 0 */
            uint32_t i = (uint32_t)scan_from;
            while (vis[i])
                ++i;
            scan_from = i;
            int connected = 0;
            for (uint32_t j = i; j > 0; --j)
                if (vis[j - 1]) {
                    links[2 * nl] = j - 1;
                    links[2 * nl + 1] = i;
                    ++nl;
                    connected = 1;
                    break;
                }
            if (!connected)
                for (uint32_t j = i + 1; j < n; ++j)
                    if (vis[j]) {
                        links[2 * nl] = i;
                        links[2 * nl + 1] = j;
                        ++nl;
                        break;
                    }
            qh = qt = 0;
            q[qt++] = i;
            pending = i;
        }
    }
    free(vis);
    free(q);
    if (nl) {
        uint64_t nn = m->nnz + 2 * nl;
        uint32_t *cr = (uint32_t *)malloc(sizeof(uint32_t) * nn);
        uint32_t *cc = (uint32_t *)malloc(sizeof(uint32_t) * nn);
        uint32_t *nci = (uint32_t *)malloc(sizeof(uint32_t) * nn);
        if (!cr || !cc || !nci) {
            free(cr); free(cc); free(nci); free(links);
            return ORC_ERR_NOMEM;
        }
        uint64_t w = 0;
        for (uint32_t r = 0; r < n; ++r)
            for (uint32_t k = m->rp[r]; k < m->rp[r + 1]; ++k) {
                cr[w] = r; cc[w] = m->ci[k]; ++w;
            }
        for (size_t l = 0; l < nl; ++l) {
            /* (Graph.h:249-258): entry (second, first) then (first, second) */
            cr[w] = links[2 * l + 1]; cc[w] = links[2 * l]; ++w;
            cr[w] = links[2 * l]; cc[w] = links[2 * l + 1]; ++w;
        }
        int rc = orc_coo_to_csr(n, nn, cr, cc, m->rp, nci);
        free(cr); free(cc);
        if (rc) {
            free(nci); free(links);
            return rc;
        }
        free(m->ci);
        m->ci = nci;
        m->nnz = nn;
        m->added_links = (uint32_t)nl;
    }
    free(links);
    return ORC_OK;
}

/*
 * MatrixMarket reader (COO.cpp:89-199, loadMTX) followed by COO -> CSR and
 * prepareRCM(!symmetric) (Graph.h:293-312).  The reference also writes
 * .hicsr cache files next to the input; the oracle writes nothing.
 * Accepts `coordinate` with real|integer|pattern|complex and
 * general|symmetric|Hermitian; symmetric and Hermitian entries off the
 * diagonal are mirrored as they are read.  Indices are 1-based; an index of 0
 * or beyond the header's size is an error, as are more entries than declared.
 */
int orc_load_mtx(const char *path, orc_csr *out)
{
    memset(out, 0, sizeof(*out));
    FILE *f = fopen(path, "r");
    if (!f)
        return ORC_ERR_IO;
    size_t cap = 1 << 16;
    char *line = (char *)malloc(cap);
    if (!line) {
        fclose(f);
        return ORC_ERR_NOMEM;
    }
    int rc = ORC_OK;
    uint32_t *cr = NULL, *cc = NULL;
    if (!fgets(line, (int)cap, f) || strncmp(line, "%%MatrixMarket matrix coordinate", 32) != 0) {
        rc = ORC_ERR_FORMAT;
        goto done;
    }
    char t0[64], t1[64], t2[64], dtype[64], sym[64];
    if (sscanf(line, "%63s %63s %63s %63s %63s", t0, t1, t2, dtype, sym) != 5) {
        rc = ORC_ERR_FORMAT;
        goto done;
    }
    int pattern = strcmp(dtype, "pattern") == 0;
    if (!pattern && strcmp(dtype, "complex") != 0 && strcmp(dtype, "real") != 0 &&
        strcmp(dtype, "integer") != 0) {
        rc = ORC_ERR_FORMAT;
        goto done;
    }
    int symmetric = 0, hermitian = 0;
    if (strcmp(sym, "symmetric") == 0)
        symmetric = 1;
    else if (strcmp(sym, "Hermitian") == 0)
        hermitian = 1;
    else if (strcmp(sym, "general") != 0) {
        rc = ORC_ERR_FORMAT;
        goto done;
    }
    unsigned long long nr = 0, nc = 0, nz = 0;
    for (;;) {
        if (!fgets(line, (int)cap, f)) {
            rc = ORC_ERR_FORMAT;
            goto done;
        }
        if (line[0] == '%')
            continue;
        if (sscanf(line, "%llu %llu %llu", &nr, &nc, &nz) != 3) {
            rc = ORC_ERR_FORMAT;
            goto done;
        }
        break;
    }
    if (nr != nc || nr == 0 || nr >= 0xFFFFFFFFull) {
        rc = ORC_ERR_FORMAT;
        goto done;
    }
    size_t reserve = (size_t)nz * ((symmetric || hermitian) ? 2 : 1);
    cr = (uint32_t *)malloc(sizeof(uint32_t) * (reserve ? reserve : 1));
    cc = (uint32_t *)malloc(sizeof(uint32_t) * (reserve ? reserve : 1));
    if (!cr || !cc) {
        rc = ORC_ERR_NOMEM;
        goto done;
    }
    size_t read = 0, entries = 0;
    while (fgets(line, (int)cap, f)) {
        if (line[0] == '%')
            continue;
        char *p = line;
        while (*p && isspace((unsigned char)*p))
            ++p;
        if (!*p)
            continue;
        unsigned long long r, c;
        double d;
        int got = pattern ? sscanf(p, "%llu %llu", &r, &c) : sscanf(p, "%llu %llu %lf", &r, &c, &d);
        if (got != (pattern ? 2 : 3) || r == 0 || c == 0 || r > nr || c > nc || entries >= nz) {
            rc = ORC_ERR_FORMAT;
            goto done;
        }
        ++entries;
        cr[read] = (uint32_t)(r - 1);
        cc[read] = (uint32_t)(c - 1);
        ++read;
        if ((symmetric || hermitian) && r != c) {
            cr[read] = (uint32_t)(c - 1);
            cc[read] = (uint32_t)(r - 1);
            ++read;
        }
    }
    out->n = (uint32_t)nr;
    out->nnz = read;
    out->rp = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)nr + 1));
    out->ci = (uint32_t *)malloc(sizeof(uint32_t) * (read ? read : 1));
    if (!out->rp || !out->ci) {
        rc = ORC_ERR_NOMEM;
        goto done;
    }
    rc = orc_coo_to_csr(out->n, read, cr, cc, out->rp, out->ci);
    if (rc == ORC_OK)
        rc = orc_prepare_rcm(out, !symmetric);
done:
    free(cr);
    free(cc);
    free(line);
    fclose(f);
    if (rc != ORC_OK)
        orc_csr_free(out);
    return rc;
}

/* Accessors so that Python (ctypes) can read an orc_csr without mirroring
 * the struct layout. */
orc_csr *orc_csr_new(void) { return (orc_csr *)calloc(1, sizeof(orc_csr)); }
void orc_csr_delete(orc_csr *m)
{
    orc_csr_free(m);
    free(m);
}
uint32_t orc_csr_n(const orc_csr *m) { return m->n; }
uint64_t orc_csr_nnz(const orc_csr *m) { return m->nnz; }
const uint32_t *orc_csr_rp(const orc_csr *m) { return m->rp; }
const uint32_t *orc_csr_ci(const orc_csr *m) { return m->ci; }
uint32_t orc_csr_added_entries(const orc_csr *m) { return m->added_entries; }
uint32_t orc_csr_added_links(const orc_csr *m) { return m->added_links; }

/* prepareRCM on caller-provided CSR copies (for tests of raw CSR inputs). */
int orc_prepare_csr(orc_csr *m, uint32_t n, uint64_t nnz, const uint32_t *rp, const uint32_t *ci,
                    int check_sym)
{
    memset(m, 0, sizeof(*m));
    m->n = n;
    m->nnz = nnz;
    m->rp = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)n + 1));
    m->ci = (uint32_t *)malloc(sizeof(uint32_t) * (nnz ? nnz : 1));
    if (!m->rp || !m->ci) {
        orc_csr_free(m);
        return ORC_ERR_NOMEM;
    }
    memcpy(m->rp, rp, sizeof(uint32_t) * ((size_t)n + 1));
    memcpy(m->ci, ci, sizeof(uint32_t) * nnz);
    int rc = orc_prepare_rcm(m, check_sym);
    if (rc != ORC_OK)
        orc_csr_free(m);
    return rc;
}
