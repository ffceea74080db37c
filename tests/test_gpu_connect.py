"""The device connectivity repair (pbrcm_connect_device, csrc/connect.cu)
against the oracle's restatement of prepareRCM (include/Graph.h:160-263):
the joined CSR must be identical entry for entry (integer work: exact)."""
import numpy as np
import pytest

from test_connect_cpu import random_pattern

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint32)


def _run(pbrcm, ctx, rp, ci, **kw):
    orp, oci, links = pbrcm.connect_device(_dev(rp), _dev(ci), ctx=ctx, **kw)
    return _host(orp), _host(oci), links


def _check(pbrcm, ctx, oracle_mod, rp, ci, **kw):
    arp, aci, links = _run(pbrcm, ctx, rp, ci, **kw)
    erp, eci, _ = oracle_mod.prepare_csr(rp, ci, check_sym=False)
    assert np.array_equal(arp, erp) and np.array_equal(aci, eci)
    assert links == (eci.shape[0] - ci.shape[0]) // 2
    return links


@pytest.mark.parametrize("seed", range(24))
def test_random_patterns_match_oracle(pbrcm, gpu_ctx, oracle_mod, seed):
    """Many small components, rows without the diagonal, empty rows (the
    first rows too, so that row 0 takes the (0, minn) link), duplicates."""
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(2, 5000))
    rp, ci = random_pattern(rng, n, int(rng.integers(1, 2 * n)), diag_frac=rng.random(),
                            dup_frac=0.1 if seed % 2 else 0.0, empty_head=int(rng.integers(0, 4)) if seed % 3 == 0 else 0)
    if ci.shape[0] == 0:
        pytest.skip("no entries")
    _check(pbrcm, gpu_ctx, oracle_mod, rp, ci)


def test_connected_matrix_unchanged(pbrcm, gpu_ctx):
    from parallelbatchrcm_b200 import gen
    m = gen.grid3d(24, 20, 16, seed=5)
    arp, aci, links = _run(pbrcm, gpu_ctx, m.row_ptr, m.col_idx)
    assert links == 0 and np.array_equal(arp, m.row_ptr) and np.array_equal(aci, m.col_idx)


def test_sparse_rgg_1m_matches_oracle(pbrcm, gpu_ctx, oracle_mod):
    """A 1M-node random geometric graph of 1-3 nearest neighbours per point
    before the loader joins it (about 40k components), the generator's own
    join, and a reorder of the joined matrix against the oracle."""
    from parallelbatchrcm_b200 import gen
    m = gen.rgg(1_000_000, kmin=1, kmax=3, long_frac=0.0, connect=False)
    links = _check(pbrcm, gpu_ctx, oracle_mod, m.row_ptr, m.col_idx)
    assert links > 10_000
    j = gen.connect_components(m)
    arp, aci, _ = _run(pbrcm, gpu_ctx, m.row_ptr, m.col_idx)
    assert np.array_equal(arp, j.row_ptr) and np.array_equal(aci, j.col_idx)
    perm, res = pbrcm.reorder(arp, aci, reverse=True, ctx=gpu_ctx)
    eperm = oracle_mod.full_reorder(arp, aci)["perm"]
    assert np.array_equal(perm, eperm)


def test_forest_of_small_trees(pbrcm, gpu_ctx, oracle_mod):
    """2M nodes in ~1M components (a random forest with half the edges a
    tree needs): long union chains and a million links."""
    rng = np.random.default_rng(9)
    n = 2_000_000
    child = rng.permutation(n)[: n // 2]
    par = (child * rng.random(child.size)).astype(np.int64)  # an earlier node: a forest
    rp, ci = random_pattern(rng, n, 0, diag_frac=1.0)
    rows = np.concatenate([np.repeat(np.arange(n), np.diff(rp).astype(np.int64)), child, par]).astype(np.uint64)
    cols = np.concatenate([ci.astype(np.int64), par, child]).astype(np.uint64)
    key = np.unique((rows << np.uint64(32)) | cols)
    r = (key >> np.uint64(32)).astype(np.int64)
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(r, minlength=n), out=rp[1:])
    rp, ci = rp.astype(np.uint32), (key & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    assert _check(pbrcm, gpu_ctx, oracle_mod, rp, ci) > n // 4


def test_output_room_grows(pbrcm, gpu_ctx, oracle_mod):
    """With room for only the input's entries the wrapper sees the size the
    call reports and calls again."""
    rng = np.random.default_rng(4)
    rp, ci = random_pattern(rng, 3000, 1500, diag_frac=0.5)
    _check(pbrcm, gpu_ctx, oracle_mod, rp, ci, cap=ci.shape[0])


def test_rejects_bad_patterns(pbrcm, gpu_ctx):
    from parallelbatchrcm_b200 import PbrcmError
    # not symmetric: 0 -> 1 without 1 -> 0
    rp, ci = np.array([0, 2, 3], np.uint32), np.array([0, 1, 1], np.uint32)
    with pytest.raises(PbrcmError) as e:
        _run(pbrcm, gpu_ctx, rp, ci)
    assert e.value.status == 1
    # a row not sorted by column
    rp, ci = np.array([0, 2, 4], np.uint32), np.array([1, 0, 0, 1], np.uint32)
    with pytest.raises(PbrcmError) as e:
        _run(pbrcm, gpu_ctx, rp, ci)
    assert e.value.status == 1
    # a column past the matrix
    rp, ci = np.array([0, 1, 2], np.uint32), np.array([0, 7], np.uint32)
    with pytest.raises(PbrcmError) as e:
        _run(pbrcm, gpu_ctx, rp, ci)
    assert e.value.status == 1
    # no entry at all
    rp, ci = np.zeros(4, np.uint32), np.zeros(1, np.uint32)[:0]
    import torch
    with pytest.raises(PbrcmError) as e:
        pbrcm.connect_device(_dev(rp), torch.zeros(1, dtype=torch.int32, device="cuda")[:0], ctx=gpu_ctx)
    assert e.value.status == 7
