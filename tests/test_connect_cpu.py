"""The rule the device connectivity repair (csrc/connect.cu) computes, pinned
on the CPU: the links prepareRCM adds (include/Graph.h:160-263, restated by
the oracle's orc_prepare_rcm) depend on the components alone -- (m - 1, m)
for every component whose smallest node m > 0 is not in the component of the
first non-empty row minn, and (0, minn) when row 0 is empty.  Checked here
with scipy's connected components against the oracle; the GPU tests check
the kernels against the oracle directly."""
import numpy as np
import pytest


def random_pattern(rng, n, m, diag_frac=0.7, dup_frac=0.0, empty_head=0):
    """Symmetric pattern with sorted rows: m random undirected pairs, the
    diagonal on a fraction of rows, some duplicated entries and optionally
    the first `empty_head` rows left empty."""
    u = rng.integers(empty_head, n, m)
    v = rng.integers(empty_head, n, m)
    d = np.nonzero(rng.random(n) < diag_frac)[0]
    d = d[d >= empty_head]
    rows = np.concatenate([u, v, d]).astype(np.uint64)
    cols = np.concatenate([v, u, d]).astype(np.uint64)
    key = np.unique((rows << np.uint64(32)) | cols)
    if dup_frac:
        key = np.sort(np.concatenate([key, key[rng.random(key.size) < dup_frac]]))
    r = (key >> np.uint64(32)).astype(np.int64)
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(r, minlength=n), out=rp[1:])
    return rp.astype(np.uint32), (key & np.uint64(0xFFFFFFFF)).astype(np.uint32)


def links_by_components(rp, ci):
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import connected_components

    n = rp.shape[0] - 1
    a = csr_matrix((np.ones(ci.shape[0], np.int8), ci, rp), shape=(n, n))
    _, lab = connected_components(a, directed=False)
    smallest = np.full(lab.max() + 1, n, np.int64)
    np.minimum.at(smallest, lab, np.arange(n))
    minn = int(np.nonzero(np.diff(rp))[0][0])
    mins = np.sort(smallest[smallest != smallest[lab[minn]]])
    return [(int(m) - 1, int(m)) if m > 0 else (0, minn) for m in mins]


def joined(rp, ci, links):
    n = rp.shape[0] - 1
    rows = np.repeat(np.arange(n, dtype=np.uint64), np.diff(rp).astype(np.int64))
    key = [(rows << np.uint64(32)) | ci.astype(np.uint64)]
    for a, b in links:
        key.append(np.array([(a << 32) | b, (b << 32) | a], np.uint64))
    key = np.sort(np.concatenate(key))
    r = (key >> np.uint64(32)).astype(np.int64)
    orp = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(r, minlength=n), out=orp[1:])
    return orp.astype(np.uint32), (key & np.uint64(0xFFFFFFFF)).astype(np.uint32)


@pytest.mark.parametrize("seed", range(40))
def test_links_follow_from_components(oracle_mod, seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(2, 400))
    head = int(rng.integers(0, 4)) if seed % 3 == 0 else 0
    rp, ci = random_pattern(rng, n, int(rng.integers(1, 2 * n)), diag_frac=rng.random(),
                            dup_frac=0.1 if seed % 2 else 0.0, empty_head=min(head, n - 1))
    if ci.shape[0] == 0:
        pytest.skip("no entries")
    erp, eci, _ = oracle_mod.prepare_csr(rp, ci, check_sym=False)
    arp, aci = joined(rp, ci, links_by_components(rp, ci))
    assert np.array_equal(arp, erp) and np.array_equal(aci, eci)


def unjoined_from_mtx(path):
    """The symmetric pattern of a 'pattern symmetric' MatrixMarket file
    before any link is added, rows sorted."""
    with open(path) as f:
        lines = [ln for ln in f if not ln.startswith("%")]
    n = int(lines[0].split()[0])
    e = np.array([[int(t) - 1 for t in ln.split()[:2]] for ln in lines[1:]], np.uint64)
    r, c = e[:, 0], e[:, 1]
    off = r != c
    key = np.sort(np.concatenate([(r << np.uint64(32)) | c, (c[off] << np.uint64(32)) | r[off]]))
    rows = (key >> np.uint64(32)).astype(np.int64)
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(rows, minlength=n), out=rp[1:])
    return rp.astype(np.uint32), (key & np.uint64(0xFFFFFFFF)).astype(np.uint32)


def test_components_fixture_links():
    """The golden file with three components, joined by the reference's own
    loader (tests/golden/mtx_components.npz): the rule gives the same CSR."""
    import os
    from conftest import GOLDEN, load_golden
    rp, ci = unjoined_from_mtx(os.path.join(GOLDEN, "mtx_components.mtx"))
    links = links_by_components(rp, ci)
    assert links == [(2, 3), (5, 6)]
    g = load_golden("mtx_components")
    arp, aci = joined(rp, ci, links)
    assert np.array_equal(arp, g["row_ptr"]) and np.array_equal(aci, g["col_idx"])
