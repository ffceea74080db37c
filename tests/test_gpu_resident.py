"""The shared-memory engine (csrc/resident.cu): a small matrix reordered by
one CTA that holds its CSR in shared memory, against the reference goldens
and the oracle, at every group shape; matrices it cannot take (a row longer
than its 512-edge chunks, too big for shared memory) go on to the team
engine with the same result."""
import os

import numpy as np
import pytest

from conftest import golden_names, load_golden

pytestmark = pytest.mark.gpu

GROUPS = [64, 128, 256]


@pytest.fixture(scope="module", params=GROUPS)
def res_ctx(request, pbrcm):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    old = os.environ.get("PBRCM_RESIDENT_GROUP")
    os.environ["PBRCM_RESIDENT_GROUP"] = str(request.param)
    try:
        ctx = pbrcm.Context(0)
    finally:
        if old is None:
            del os.environ["PBRCM_RESIDENT_GROUP"]
        else:
            os.environ["PBRCM_RESIDENT_GROUP"] = old
    yield ctx
    ctx.close()


def _small(rp):
    """Certainly within the engine: rows of at most 512 entries and a CSR
    plus two workspaces well inside 200 KB of shared memory."""
    n = rp.shape[0] - 1
    return int(np.diff(rp.astype(np.int64)).max()) <= 512 and 4 * (n + 1 + int(rp[-1])) + 16 * n <= 150_000


def _too_big(rp):
    """Certainly beyond it: the CSR and one workspace alone exceed the 227 KB
    a CTA can have, or a row is longer than a chunk."""
    n = rp.shape[0] - 1
    return int(np.diff(rp.astype(np.int64)).max()) > 512 or 4 * (n + 1 + int(rp[-1])) + 8 * n > 232_448


@pytest.mark.parametrize("name", golden_names())
def test_golden(pbrcm, res_ctx, oracle_mod, name):
    g = load_golden(name)
    rp, ci = g["row_ptr"], g["col_idx"]
    for reverse in (False, True):
        perm, res = pbrcm.reorder(rp, ci, reverse=reverse, ctx=res_ctx)
        assert res["status"] == 0
        if _small(rp):
            assert res["engine"] == 2
        if _too_big(rp):
            assert res["engine"] == 0  # handed on to the team
        assert (res["start_node"], res["peripheral_passes"], res["eccentricity"]) == (
            int(g["start"]), int(g["passes"]), int(g["ecc"]))
        assert np.array_equal(perm, g["perm"][::-1] if reverse else g["perm"])
        assert res["bandwidth"] == int(g["bandwidth"])
        assert res["initial_bandwidth"] == int(g["initial_bandwidth"])
        assert res["profile"] == oracle_mod.profile(rp, ci, perm)


def _graphs():
    from parallelbatchrcm_b200 import gen
    rng = np.random.default_rng(3)
    out = {
        "grid2d_70x50": gen.grid2d(70, 50, seed=41),
        "grid3d_14x13x12": gen.grid3d(14, 13, 12, seed=42),
        "rgg_2500": gen.rgg(2500, kmin=4, kmax=12, seed=43),
        "rgg_4000": gen.rgg(4000, kmin=4, kmax=12, seed=43),  # beyond shared memory
        "rgg_300": gen.rgg(300, seed=44),
    }
    # a shuffled path (one node a level: thousands of levels)
    n = 2500
    p = rng.permutation(n)
    out["path_2500"] = gen.from_edges(n, p[:-1], p[1:])
    # stars whose centre row has 512 (the engine's longest) and 513 entries
    for d in (511, 512):
        hub = np.zeros(d, dtype=np.int64)
        leaves = np.arange(1, d + 1)
        ring = gen.from_edges(d + 1, np.concatenate([hub, leaves[:-1]]), np.concatenate([leaves, leaves[1:]]))
        out[f"star_{d}"] = ring
    # circulant graphs (shuffled labels) whose rows have exactly 8, 16 and 17
    # entries: the edges of the row classes of the one-parent-a-thread pass
    for name, offs in (("circ_row8", [1, 2, 3, 1000]), ("circ_row16", [1, 2, 3, 4, 5, 6, 7, 1000]),
                       ("circ_row17", [1, 2, 3, 4, 5, 6, 7, 8])):
        n = 2000
        lab = rng.permutation(n)
        src = np.concatenate([np.arange(n)] * len(offs))
        dst = np.concatenate([(np.arange(n) + o) % n for o in offs])
        out[name] = gen.from_edges(n, lab[src], lab[dst])
    # random sparse graph, made connected
    m = 3000
    out["er_1500"] = gen.connect_components(gen.from_edges(1500, rng.integers(0, 1500, m), rng.integers(0, 1500, m)))
    return out


@pytest.mark.parametrize("case", list(_graphs()))
def test_generated_match_oracle(pbrcm, res_ctx, oracle_mod, case):
    m = _graphs()[case]
    perm, res = pbrcm.reorder(m.row_ptr, m.col_idx, reverse=True, ctx=res_ctx)
    ref = oracle_mod.full_reorder(m.row_ptr, m.col_idx, reverse=True)
    if _small(m.row_ptr):
        assert res["engine"] == 2
    if _too_big(m.row_ptr):
        assert res["engine"] == 0
    assert (res["start_node"], res["peripheral_passes"], res["eccentricity"]) == (
        ref["start"], ref["passes"], ref["ecc"])
    assert np.array_equal(perm, ref["perm"])
    assert res["bandwidth"] == ref["bandwidth"] and res["profile"] == ref["profile"]
    assert res["levels"] == ref["ecc"] + 1 or ref["passes"] == 0
    # start search alone, and explicit starts without the bandwidth
    assert pbrcm.find_peripheral(m.row_ptr, m.col_idx, ctx=res_ctx) == (ref["start"], ref["passes"], ref["ecc"])
    for s in (0, m.n - 1, m.n // 3):
        perm, res = pbrcm.reorder(m.row_ptr, m.col_idx, reverse=False, start=s, want_bandwidth=False, ctx=res_ctx)
        assert res["start_node"] == s and res["peripheral_passes"] == 0 and res["bandwidth"] == -1
        assert np.array_equal(perm, oracle_mod.cm_order(m.row_ptr, m.col_idx, s))


def test_device_entry_and_errors(pbrcm, res_ctx, oracle_mod):
    import torch
    from parallelbatchrcm_b200 import gen
    m = gen.grid2d(40, 30, seed=45)
    rp = torch.from_numpy(m.row_ptr.view(np.int32)).cuda()
    ci = torch.from_numpy(m.col_idx.view(np.int32)).cuda()
    perm, res = pbrcm.reorder_device(rp, ci, reverse=True, ctx=res_ctx)
    ref = oracle_mod.full_reorder(m.row_ptr, m.col_idx, reverse=True)
    assert res["engine"] == 2 and np.array_equal(perm.cpu().numpy().view(np.uint32), ref["perm"])
    assert res["device_ms"] > 0
    # two components: an error from the search and from an explicit start
    a, b = gen.grid2d(9, 8, seed=1), gen.grid2d(5, 3, seed=2)
    rp2 = np.concatenate([a.row_ptr, b.row_ptr[1:] + a.nnz]).astype(np.uint32)
    ci2 = np.concatenate([a.col_idx, b.col_idx + a.n]).astype(np.uint32)
    for start in (None, 2, a.n + 1):
        _, res = pbrcm.reorder(rp2, ci2, start=start, ctx=res_ctx, raise_on_error=False)
        assert res["status"] != 0 and res["engine"] == 2
        with pytest.raises(pbrcm.PbrcmError) as e:
            pbrcm.reorder(rp2, ci2, start=start, ctx=res_ctx)
        assert e.value.name == "PBRCM_ERR_DISCONNECTED"
    # one node, two nodes
    for rp3, ci3 in ((np.array([0, 1], np.uint32), np.array([0], np.uint32)),
                     (np.array([0, 2, 4], np.uint32), np.array([0, 1, 0, 1], np.uint32))):
        perm, res = pbrcm.reorder(rp3, ci3, reverse=False, ctx=res_ctx)
        ref = oracle_mod.full_reorder(rp3, ci3, reverse=False)
        assert res["engine"] == 2 and np.array_equal(perm, ref["perm"])
        assert (res["start_node"], res["peripheral_passes"], res["eccentricity"]) == (
            ref["start"], ref["passes"], ref["ecc"])


def test_too_big_for_shared_memory_goes_to_team(pbrcm, gpu_ctx, oracle_mod):
    from parallelbatchrcm_b200 import gen
    m = gen.grid2d(160, 150, seed=46)  # 24,000 nodes: CSR alone ~ 480 KB
    perm, res = pbrcm.reorder(m.row_ptr, m.col_idx, reverse=True, ctx=gpu_ctx)
    ref = oracle_mod.full_reorder(m.row_ptr, m.col_idx, reverse=True)
    assert res["engine"] == 0 and np.array_equal(perm, ref["perm"])
