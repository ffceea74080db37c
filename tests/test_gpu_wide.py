"""The level-synchronous engine for wide, shallow graphs (csrc/wide.cu)
against the golden fixtures and the oracle: run first on every matrix whose
rows fit its chunks (PBRCM_ENGINE=wide), and taken over automatically from
the team engine on random graphs whose BFS levels hold most of the nodes.
Integer work: every comparison is exact."""
import os

import numpy as np
import pytest

from conftest import golden_names, load_golden

pytestmark = pytest.mark.gpu


def _context(pbrcm, env):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        return pbrcm.Context(0)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


@pytest.fixture(scope="module")
def wide_ctx(pbrcm):
    ctx = _context(pbrcm, {"PBRCM_ENGINE": "wide"})
    yield ctx
    ctx.close()


def _fits(rp):
    return int(np.diff(rp).max()) <= 1024


@pytest.mark.parametrize("name", golden_names())
def test_golden_on_wide_engine(pbrcm, wide_ctx, oracle_mod, name):
    g = load_golden(name)
    rp, ci = g["row_ptr"], g["col_idx"]
    for reverse in (False, True):
        perm, res = pbrcm.reorder(rp, ci, reverse=reverse, ctx=wide_ctx)
        assert res["status"] == 0
        n = rp.shape[0] - 1
        if not _fits(rp) or n == 1:
            assert res["engine"] == 0
        elif (int(g["passes"]) + 1) * (int(g["ecc"]) + 1) <= 1016:  # level steps, at most
            assert res["engine"] == 1
        assert (res["start_node"], res["peripheral_passes"], res["eccentricity"]) == (
            int(g["start"]), int(g["passes"]), int(g["ecc"]))
        assert np.array_equal(perm, g["perm"][::-1] if reverse else g["perm"])
        assert res["bandwidth"] == int(g["bandwidth"])
        assert res["initial_bandwidth"] == int(g["initial_bandwidth"])
        assert res["profile"] == oracle_mod.profile(rp, ci, perm)


@pytest.mark.parametrize("name", ["grid2d_64x64_s1", "rgg_3000_s11", "caterpillar_40x60", "path_300"])
def test_explicit_starts_on_wide_engine(pbrcm, wide_ctx, oracle_mod, name):
    g = load_golden(name)
    n = g["row_ptr"].shape[0] - 1
    for s in (0, n - 1, n // 3):
        perm, res = pbrcm.reorder(g["row_ptr"], g["col_idx"], reverse=False, start=s, ctx=wide_ctx)
        assert res["engine"] == 1 and res["start_node"] == s and res["peripheral_passes"] == 0
        assert np.array_equal(perm, oracle_mod.cm_order(g["row_ptr"], g["col_idx"], s))


def _er(n, deg, seed):
    from parallelbatchrcm_b200 import gen
    rng = np.random.default_rng(seed)
    m = n * deg // 2
    return gen.connect_components(gen.from_edges(n, rng.integers(0, n, m), rng.integers(0, n, m)))


@pytest.mark.parametrize("case", ["er_300k_d8", "er_100k_d20", "grid3d_40"])
def test_generated_on_wide_engine(pbrcm, wide_ctx, oracle_mod, case):
    from parallelbatchrcm_b200 import gen
    m = {"er_300k_d8": lambda: _er(300_000, 8, 1), "er_100k_d20": lambda: _er(100_000, 20, 2),
         "grid3d_40": lambda: gen.grid3d(40, 40, 40, seed=21)}[case]()
    perm, res = pbrcm.reorder(m.row_ptr, m.col_idx, reverse=True, ctx=wide_ctx)
    ref = oracle_mod.full_reorder(m.row_ptr, m.col_idx, reverse=True)
    assert res["engine"] == 1
    assert (res["start_node"], res["peripheral_passes"], res["eccentricity"]) == (
        ref["start"], ref["passes"], ref["ecc"])
    assert np.array_equal(perm, ref["perm"])
    assert res["bandwidth"] == ref["bandwidth"] and res["profile"] == ref["profile"]


def test_team_hands_wide_graph_over(pbrcm, gpu_ctx, oracle_mod):
    """Default context: a 1M-node random graph (widest level ~58 % of the
    nodes) goes to the level-synchronous engine, a 3-D grid does not."""
    from parallelbatchrcm_b200 import gen
    m = _er(1_000_000, 8, 3)
    perm, res = pbrcm.reorder(m.row_ptr, m.col_idx, reverse=True, ctx=gpu_ctx)
    ref = oracle_mod.full_reorder(m.row_ptr, m.col_idx, reverse=True)
    assert res["engine"] == 1
    assert (res["start_node"], res["peripheral_passes"], res["eccentricity"]) == (
        ref["start"], ref["passes"], ref["ecc"])
    assert np.array_equal(perm, ref["perm"])
    assert res["bandwidth"] == ref["bandwidth"] and res["profile"] == ref["profile"]
    g = gen.grid3d(64, 64, 64, seed=5)
    _, res = pbrcm.reorder(g.row_ptr, g.col_idx, reverse=True, ctx=gpu_ctx)
    assert res["engine"] == 0


def test_wide_engine_device_entry_and_start_search(pbrcm, wide_ctx, oracle_mod):
    import torch
    m = _er(50_000, 6, 4)
    rp = torch.from_numpy(m.row_ptr.view(np.int32)).cuda()
    ci = torch.from_numpy(m.col_idx.view(np.int32)).cuda()
    perm, res = pbrcm.reorder_device(rp, ci, reverse=True, ctx=wide_ctx)
    ref = oracle_mod.full_reorder(m.row_ptr, m.col_idx, reverse=True)
    assert res["engine"] == 1 and np.array_equal(perm.cpu().numpy().view(np.uint32), ref["perm"])
    s, p, e = pbrcm.find_peripheral(m.row_ptr, m.col_idx, ctx=wide_ctx)
    assert (s, p, e) == (ref["start"], ref["passes"], ref["ecc"])


def test_deep_graph_handed_back(pbrcm, wide_ctx, oracle_mod):
    """A shuffled path of 3,000 nodes: its first pass alone has 1,500 levels,
    more level steps than the engine runs before it hands the matrix back to
    the team engine, which returns the same order."""
    from parallelbatchrcm_b200 import gen
    n = 3000
    p = np.random.default_rng(5).permutation(n)
    m = gen.from_edges(n, p[:-1], p[1:])
    perm, res = pbrcm.reorder(m.row_ptr, m.col_idx, reverse=True, ctx=wide_ctx)
    ref = oracle_mod.full_reorder(m.row_ptr, m.col_idx, reverse=True)
    assert res["engine"] == 0 and res["start_node"] == ref["start"]
    assert np.array_equal(perm, ref["perm"])


def test_wide_engine_reports_disconnected(pbrcm, wide_ctx):
    from parallelbatchrcm_b200 import gen
    a = gen.grid2d(30, 30, seed=None)
    n = a.n
    rp = np.concatenate([a.row_ptr, a.row_ptr[1:] + a.row_ptr[-1]]).astype(np.uint32)
    ci = np.concatenate([a.col_idx, a.col_idx + n]).astype(np.uint32)
    perm, res = pbrcm.reorder(rp, ci, reverse=True, ctx=wide_ctx, raise_on_error=False)
    assert res["status"] == 2 and res["engine"] == 1
