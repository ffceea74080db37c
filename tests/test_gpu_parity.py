"""GPU engine vs the reference (golden fixtures) and the oracle, through the
C ABI (libpbrcm.so).  Integer work: every comparison is exact."""
import numpy as np
import pytest

from conftest import golden_names, load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["default", "team"])
def any_ctx(request, gpu_ctx, gpu_ctx_team):
    """The default context (small matrices on the shared-memory engine) and
    one that keeps every matrix on the team engine."""
    return gpu_ctx if request.param == "default" else gpu_ctx_team


@pytest.mark.parametrize("name", golden_names())
def test_golden_auto_start(pbrcm, any_ctx, name):
    g = load_golden(name)
    perm, res = pbrcm.reorder(g["row_ptr"], g["col_idx"], reverse=False, ctx=any_ctx)
    assert res["status"] == 0
    assert (res["start_node"], res["peripheral_passes"], res["eccentricity"]) == (
        int(g["start"]), int(g["passes"]), int(g["ecc"]))
    assert np.array_equal(perm, g["perm"])
    assert res["bandwidth"] == int(g["bandwidth"])
    assert res["initial_bandwidth"] == int(g["initial_bandwidth"])


@pytest.mark.parametrize("name", golden_names())
def test_golden_reverse_and_profile(pbrcm, any_ctx, oracle_mod, name):
    g = load_golden(name)
    perm, res = pbrcm.reorder(g["row_ptr"], g["col_idx"], reverse=True, ctx=any_ctx)
    assert np.array_equal(perm, g["perm"][::-1])
    assert res["bandwidth"] == int(g["bandwidth"])
    assert res["profile"] == oracle_mod.profile(g["row_ptr"], g["col_idx"], perm)


@pytest.mark.parametrize("name", ["grid2d_64x64_s1", "rgg_3000_s11", "star_1500_ring7", "caterpillar_40x60",
                                  "mtx_general_dups", "path_300"])
def test_explicit_starts_match_oracle(pbrcm, any_ctx, oracle_mod, name):
    g = load_golden(name)
    n = g["row_ptr"].shape[0] - 1
    rng = np.random.default_rng(7)
    for s in sorted(set([0, n - 1] + list(rng.integers(0, n, 4)))):
        perm, res = pbrcm.reorder(g["row_ptr"], g["col_idx"], reverse=False, start=int(s), ctx=any_ctx)
        assert res["start_node"] == s and res["peripheral_passes"] == 0
        assert np.array_equal(perm, oracle_mod.cm_order(g["row_ptr"], g["col_idx"], int(s)))


def _cases():
    from parallelbatchrcm_b200 import gen
    return {
        "grid3d_40": lambda: gen.grid3d(40, 40, 40, seed=21),
        "grid3d_64x32x16": lambda: gen.grid3d(64, 32, 16, seed=22),
        "grid2d_300x200": lambda: gen.grid2d(300, 200, seed=23),
        "rgg_200k": lambda: gen.rgg(200_000, seed=24),
        "rgg_50k_k4": lambda: gen.rgg(50_000, kmin=4, kmax=12, seed=25),
    }


@pytest.mark.parametrize("case", list(_cases()))
def test_generated_match_oracle(pbrcm, gpu_ctx, oracle_mod, case):
    m = _cases()[case]()
    perm, res = pbrcm.reorder(m.row_ptr, m.col_idx, reverse=True, ctx=gpu_ctx)
    ref = oracle_mod.full_reorder(m.row_ptr, m.col_idx, reverse=True)
    assert (res["start_node"], res["peripheral_passes"], res["eccentricity"]) == (
        ref["start"], ref["passes"], ref["ecc"])
    assert np.array_equal(perm, ref["perm"])
    assert res["bandwidth"] == ref["bandwidth"] and res["profile"] == ref["profile"]


def test_find_peripheral_and_bandwidth_entry_points(pbrcm, gpu_ctx, oracle_mod):
    g = load_golden("rgg_20000_k4-12_s13")
    s, p, e = pbrcm.find_peripheral(g["row_ptr"], g["col_idx"], ctx=gpu_ctx)
    assert (s, p, e) == (int(g["start"]), int(g["passes"]), int(g["ecc"]))
    bw, bw0, prof = pbrcm.bandwidth(g["row_ptr"], g["col_idx"], g["perm"], ctx=gpu_ctx)
    assert bw == int(g["bandwidth"]) and bw0 == int(g["initial_bandwidth"])
    assert prof == oracle_mod.profile(g["row_ptr"], g["col_idx"], g["perm"])
    with pytest.raises(pbrcm.PbrcmError):
        bad = g["perm"].copy()
        bad[0] = bad[1]
        pbrcm.bandwidth(g["row_ptr"], g["col_idx"], bad, ctx=gpu_ctx)


def test_reference_shaped_surface(pbrcm, gpu_ctx):
    g = load_golden("grid3d_10x11x12_s5")
    graph = pbrcm.Graph.from_csr(g["row_ptr"], g["col_idx"])
    start = pbrcm.SimplePeripheral.findPeripheral(graph, None, False, ctx=gpu_ctx)
    assert start == int(g["start"])
    perm = []

    class Csv:
        text = ""

        def write(self, s):
            self.text += s

    csv = Csv()
    pbrcm.GPU_BATCH.rcm(graph, csv, perm, start, ctx=gpu_ctx)
    assert perm == [int(x) for x in g["perm"]]
    assert float(csv.text) > 0
    assert pbrcm.check_permutation(perm) == 0
    assert pbrcm.compute_bandwidth(graph, perm) == int(g["bandwidth"])
    assert pbrcm.check_bandwidth(graph) == int(g["initial_bandwidth"])
    assert pbrcm.max_valency(graph) == int(g["max_valency"])


def test_batch_equals_single(pbrcm, gpu_ctx):
    from parallelbatchrcm_b200 import gen
    mats = [(load_golden(n)["row_ptr"], load_golden(n)["col_idx"]) for n in golden_names()]
    for i in range(40):
        mats.append(((gen.grid2d(5 + i, 3 + i % 7, seed=i)).row_ptr, gen.grid2d(5 + i, 3 + i % 7, seed=i).col_idx))
    perms, results = pbrcm.reorder_batch(mats, reverse=True, ctx=gpu_ctx)
    for (rp, ci), p, r in zip(mats, perms, results):
        q, s = pbrcm.reorder(rp, ci, reverse=True, ctx=gpu_ctx)
        assert r["status"] == 0
        assert np.array_equal(p, q)
        assert (r["start_node"], r["bandwidth"], r["profile"]) == (s["start_node"], s["bandwidth"], s["profile"])


@pytest.mark.parametrize("csize", [2, 8, 16])
def test_batch_cluster_teams(pbrcm, oracle_mod, csize, monkeypatch):
    """Every matrix of a batch on thread-block-cluster teams (hardware cluster
    barriers, all-gather and gate hand-over through distributed shared
    memory), with small solo bounds so that most levels are split across the
    cluster's CTAs; a disconnected matrix in the batch reports its error and
    leaves the others intact."""
    from parallelbatchrcm_b200 import gen
    monkeypatch.setenv("PBRCM_BATCH_CLUSTER", str(csize))
    monkeypatch.setenv("PBRCM_BATCH_CLUSTER_NNZ", "1")
    monkeypatch.setenv("PBRCM_CLUSTER_SOLO_PARENTS", "8")
    monkeypatch.setenv("PBRCM_CLUSTER_SOLO_EDGES", "32")
    ctx = pbrcm.Context(0)
    try:
        names = golden_names()
        mats = [(load_golden(n)["row_ptr"], load_golden(n)["col_idx"]) for n in names]
        extra = [gen.grid3d(20, 18, 16, seed=31), gen.rgg(20_000, seed=32), gen.grid2d(150, 90, seed=33)]
        mats += [(m.row_ptr, m.col_idx) for m in extra]
        a, b = gen.grid2d(12, 9, seed=34), gen.grid2d(5, 4, seed=35)
        mats.append((np.concatenate([a.row_ptr, b.row_ptr[1:] + a.nnz]).astype(np.uint32),
                     np.concatenate([a.col_idx, b.col_idx + a.n]).astype(np.uint32)))
        perms, results = pbrcm.reorder_batch(mats, reverse=False, ctx=ctx, raise_on_error=False)
        for name, p, r in zip(names, perms, results):
            g = load_golden(name)
            assert r["status"] == 0, (name, r)
            assert np.array_equal(p, g["perm"]), name
            assert (r["start_node"], r["peripheral_passes"], r["bandwidth"]) == (
                int(g["start"]), int(g["passes"]), int(g["bandwidth"])), name
        for m, p, r in zip(extra, perms[len(names):], results[len(names):]):
            ref = oracle_mod.full_reorder(m.row_ptr, m.col_idx, reverse=False)
            assert r["status"] == 0 and np.array_equal(p, ref["perm"])
        assert results[-1]["status"] == 2  # PBRCM_ERR_DISCONNECTED
    finally:
        ctx.close()


def test_device_entry_point(pbrcm, gpu_ctx):
    import torch
    g = load_golden("rgg_3000_s11")
    rp = torch.from_numpy(g["row_ptr"].astype(np.int32)).cuda()
    ci = torch.from_numpy(g["col_idx"].astype(np.int32)).cuda()
    perm_t, res = pbrcm.reorder_device(rp, ci, reverse=False, ctx=gpu_ctx)
    assert np.array_equal(perm_t.cpu().numpy().astype(np.uint32), g["perm"])
    po = torch.empty_like(rp[:-1])
    out = pbrcm.reorder_batch_device([(rp, ci, po)], reverse=False, ctx=gpu_ctx)
    assert out[0]["status"] == 0
    assert np.array_equal(po.cpu().numpy().astype(np.uint32), g["perm"])


@pytest.mark.parametrize("cmax", [2, 8])
def test_session_cluster_teams(pbrcm, gpu_ctx, cmax, monkeypatch):
    """Requests above the session's one-CTA size run as thread-block-cluster
    teams (one cluster launch each, next to the other requests' kernels) and
    give the single-matrix result."""
    from parallelbatchrcm_b200 import gen
    monkeypatch.setenv("PBRCM_SESSION_CLUSTER_MAX", str(cmax))
    mats = [gen.grid3d(68, 68, 68, seed=41), gen.rgg(300_000, seed=42), gen.grid2d(560, 560, seed=43),
            gen.grid2d(40, 30, seed=44)]
    with pbrcm.Session(gpu_ctx, streams=8) as sess:
        tickets = [sess.submit(m.row_ptr, m.col_idx) for m in mats]
        sess.drain()
        for m, t in zip(mats, tickets):
            perm, res = sess.poll(t)
            q, r = pbrcm.reorder(m.row_ptr, m.col_idx, ctx=gpu_ctx)
            assert res["status"] == 0 and np.array_equal(perm, q) and res["bandwidth"] == r["bandwidth"]


def test_session_results_equal_single(pbrcm, gpu_ctx):
    from parallelbatchrcm_b200 import gen
    mats = [gen.grid2d(30 + 3 * i, 20 + i, seed=100 + i) for i in range(12)]
    mats += [gen.grid3d(12, 10, 9 + i, seed=200 + i) for i in range(6)]
    mats += [gen.rgg(4000 + 500 * i, seed=300 + i) for i in range(6)]
    g = load_golden("star_3000")
    mats.append(gen.Csr(g["row_ptr"], g["col_idx"]))
    with pbrcm.Session(gpu_ctx, streams=8) as sess:
        tickets = [sess.submit(m.row_ptr, m.col_idx) for m in mats]
        sess.drain()
        for m, t in zip(mats, tickets):
            out = sess.poll(t)
            assert out is not None
            perm, res = out
            q, s = pbrcm.reorder(m.row_ptr, m.col_idx, ctx=gpu_ctx)
            assert res["status"] == 0 and np.array_equal(perm, q) and res["bandwidth"] == s["bandwidth"]
        st = sess.stats()
        assert st["completed"] == len(mats) and st["p99_ms"] >= st["p50_ms"] > 0


@pytest.mark.parametrize("case", ["grid3d_128", "rgg_1M"])
def test_full_size_configs_match_oracle(pbrcm, gpu_ctx, oracle_mod, case):
    """The benchmark configurations at full size (128^3 grid, 2.1M nodes;
    1M-node RGG): start, passes, permutation, bandwidth and profile exact."""
    from parallelbatchrcm_b200 import gen
    m = gen.grid3d(128, 128, 128, seed=12345) if case == "grid3d_128" else gen.rgg(1_000_000, seed=7)
    perm, res = pbrcm.reorder(m.row_ptr, m.col_idx, reverse=True, ctx=gpu_ctx)
    ref = oracle_mod.full_reorder(m.row_ptr, m.col_idx, reverse=True)
    assert (res["start_node"], res["peripheral_passes"], res["eccentricity"]) == (
        ref["start"], ref["passes"], ref["ecc"])
    assert np.array_equal(perm, ref["perm"])
    assert res["bandwidth"] == ref["bandwidth"] and res["profile"] == ref["profile"]
