"""CPU model of the shared-memory engine's algorithm (csrc/resident.cu),
checked against the oracle: the chunk walk with chunk-local claim keys
(atomicMin of an order-preserving (parent, slot) key, placed nodes holding
0), the per-parent (valence, slot) rank, and the kernel's round control (a
search pass on group 0, the sorted pass from the same start on group 1 from
the second search on, stop when a search confirms the eccentricity).  Small
graphs only: plain Python loops."""
import numpy as np
import pytest

from conftest import golden_names, load_golden

UNVISITED = 0xFFFFFFFF
CLAIM = 0x80000000


def model_pass(rp, ci, start, sorted_, G, EW, short):
    """One pass: the queue, its level count and the first position of its
    last level, walked in chunks of at most G parents (and EW edges for the
    edge-parallel pass; one parent a thread when `short`)."""
    n = len(rp) - 1
    w = [UNVISITED] * n
    q = [start]
    w[start] = 0
    head, tail, lvl_end, L, lstart = 0, 1, 1, 0, 0
    while head < tail:
        if head == lvl_end:
            L, lstart, lvl_end = L + 1, head, tail
        # the chunk's parents
        parents, edges = [], 0
        while head + len(parents) < lvl_end and len(parents) < G:
            p = q[head + len(parents)]
            d = int(rp[p + 1] - rp[p])
            if not short and edges + d > EW:
                break
            parents.append(p)
            edges += d
        assert parents, "a row longer than a chunk"
        # bids: every edge bids its key; a placed node keeps 0
        bids = []
        e = 0
        for j, p in enumerate(parents):
            for k in range(int(rp[p]), int(rp[p + 1])):
                key = CLAIM | ((j << 5) | (k - int(rp[p])) if short else e)
                c = int(ci[k])
                w[c] = min(w[c], key)
                bids.append((j, c, key))
                e += 1
        # standing bids, in (parent, slot) order
        kids = [[] for _ in parents]
        for j, c, key in bids:
            if w[c] == key:
                kids[j].append(c)
        for j, c, key in bids:
            if w[c] == key:
                w[c] = 0
        for j, cs in enumerate(kids):
            if sorted_:
                cs = sorted(cs, key=lambda c: int(rp[c + 1] - rp[c]))  # stable: slot order on ties
            q.extend(cs)
        head += len(parents)
        tail = len(q)
    return q, L + 1, lstart


def model_reorder(rp, ci, G=128, EW=512, spec=True, outnodes=32):
    """The kernel's round control; returns (start, passes, ecc, CM order,
    levels) or None when a row is longer than a chunk (the host hands such a
    matrix to the team)."""
    n = len(rp) - 1
    maxdeg = int(np.diff(rp.astype(np.int64)).max())
    if maxdeg > EW:
        return None
    short = maxdeg <= 16
    searching = n > 1
    start = n // 2 if searching else 0
    passes = 1 if n == 1 else 0
    ecc = lastdist = 0
    sorted_from, sq, slev = None, None, None
    while True:
        if not searching and sorted_from == start:
            break
        run_sort = not searching or (spec and passes >= 1)
        if run_sort:
            sq, slev, _ = model_pass(rp, ci, start, True, G, EW, short)
            sorted_from = start
        if searching:
            q, lev, ls = model_pass(rp, ci, start, False, G, EW, short)
            passes += 1
            assert len(q) == n, "disconnected"
            dist = lev - 1
            if dist == lastdist:
                ecc, searching = dist, False
            else:
                lo = max(n - min(outnodes, n - 1), max(ls, 1))
                best, bestdeg = 0, UNVISITED
                for pos in range(lo, n):
                    d = int(rp[q[pos] + 1] - rp[q[pos]])
                    if d <= bestdeg:
                        best, bestdeg = q[pos], d
                start, lastdist = best, dist
    return start, passes, ecc, np.array(sq, dtype=np.uint32), slev


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("shape", [(128, 512, True), (32, 512, False), (8, 64, True)])
def test_model_matches_reference_goldens(name, shape):
    G, EW, spec = shape
    g = load_golden(name)
    n = g["row_ptr"].shape[0] - 1
    if n > 5000:
        pytest.skip("large for a pure-Python model")
    out = model_reorder(g["row_ptr"], g["col_idx"], G=G, EW=EW, spec=spec)
    if out is None:
        assert int(np.diff(g["row_ptr"].astype(np.int64)).max()) > EW
        return
    start, passes, ecc, perm, levels = out
    assert (start, passes, ecc) == (int(g["start"]), int(g["passes"]), int(g["ecc"]))
    assert np.array_equal(perm, g["perm"])
    assert levels == ecc + 1


def test_model_matches_oracle_on_generated(oracle_mod):
    from parallelbatchrcm_b200 import gen
    rng = np.random.default_rng(11)
    mats = [gen.grid2d(17, 13, seed=1), gen.grid3d(6, 5, 7, seed=2), gen.rgg(400, seed=3),
            gen.rgg(300, kmin=4, kmax=12, seed=4)]
    n = 200
    mats.append(gen.connect_components(gen.from_edges(n, rng.integers(0, n, 500), rng.integers(0, n, 500))))
    for m in mats:
        ref = oracle_mod.full_reorder(m.row_ptr, m.col_idx, reverse=False)
        for G, EW in ((128, 512), (16, 32)):
            start, passes, ecc, perm, _ = model_reorder(m.row_ptr, m.col_idx, G=G, EW=EW)
            assert (start, passes, ecc) == (ref["start"], ref["passes"], ref["ecc"])
            assert np.array_equal(perm, ref["perm"])
