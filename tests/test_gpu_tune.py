"""The autotuner of the batch and serving shapes (pbrcm_autotune): every
setting it tries gives bit-identical permutations, the chosen settings are
the context's afterwards, and its cache file is applied only on a matching
device shape and library version."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _calibration():
    from parallelbatchrcm_b200 import gen
    specs = gen.mixed_batch_specs(count=48, nmax=40_000, seed=5)
    return [(m.row_ptr, m.col_idx) for m in (gen.make_from_spec(s) for s in specs)]


def test_autotune_keeps_permutations(pbrcm, tmp_path):
    mats = _calibration()
    ctx = pbrcm.Context(0)
    try:
        before, _ = pbrcm.reorder_batch(mats, reverse=True, ctx=ctx)
        path = str(tmp_path / "tuning.txt")
        t = pbrcm.autotune(mats, ctx=ctx, cache_path=path)
        assert t["source"] == 2 and t["trials"] >= 8 and t["sms"] > 0
        assert t["best_ms"] > 0 and t["best_ms"] <= t["default_ms"] * 1.05
        assert pbrcm.tuning_get(ctx)["batch_pool"] == t["batch_pool"]
        after, res = pbrcm.reorder_batch(mats, reverse=True, ctx=ctx)
        assert all(r["status"] == 0 for r in res)
        assert all(np.array_equal(a, b) for a, b in zip(before, after))
        # the session under the tuned cutoff gives the same results too
        with pbrcm.Session(ctx) as s:
            tk = [s.submit(rp, ci, reverse=True) for rp, ci in mats[:12]]
            s.drain()
            got = [s.poll(k)[0] for k in tk]
        assert all(np.array_equal(a, b) for a, b in zip(before[:12], got))
        # the cache file: applied to a fresh context, refused once edited to
        # another device shape
        ctx2 = pbrcm.Context(0)
        try:
            pbrcm.tuning_load(ctx2, path)
            t2 = pbrcm.tuning_get(ctx2)
            for k in ("batch_pool", "batch_kernel", "cluster_size", "cluster_max", "cluster_nnz", "session_cutoff_n",
                      "session_pool", "session_team_nnz", "session_cluster_max"):
                assert t2[k] == t[k], k
            assert t2["source"] == 1
            text = open(path).read().replace(f"sms={t['sms']}", f"sms={t['sms'] + 1}")
            bad = str(tmp_path / "other_device.txt")
            with open(bad, "w") as f:
                f.write(text)
            with pytest.raises(pbrcm.PbrcmError) as e:
                pbrcm.tuning_load(ctx2, bad)
            assert e.value.status == 10  # PBRCM_ERR_NOT_FOUND
        finally:
            ctx2.close()
    finally:
        ctx.close()


def test_tuning_file_read_at_context_creation(pbrcm, tmp_path, monkeypatch):
    ctx = pbrcm.Context(0)
    try:
        pbrcm.tuning_set(ctx, batch_pool=2, cluster_size=4, cluster_max=8, cluster_nnz=1 << 17,
                         session_cutoff_n=1 << 17)
        t = pbrcm.tuning_get(ctx)
        assert (t["batch_pool"], t["cluster_size"], t["cluster_max"]) == (2, 4, 8)
        with pytest.raises(pbrcm.PbrcmError):
            pbrcm.tuning_set(ctx, batch_pool=4)  # the session's one-request shape
        with pytest.raises(pbrcm.PbrcmError):
            pbrcm.tuning_set(ctx, batch_pool=8)
        with pytest.raises(pbrcm.PbrcmError):
            pbrcm.tuning_set(ctx, batch_kernel=2)
        sms = t["sms"]
    finally:
        ctx.close()
    path = tmp_path / "t.txt"
    version = pbrcm._lib.lib().pbrcm_version().decode()
    path.write_text(f"pbrcm-tuning 1\nversion={version}\nsms={sms}\nbatch_pool=3\ncluster_size=2\n"
                    f"cluster_max=32\ncluster_nnz=131072\nsession_cutoff_n=65536\n")
    monkeypatch.setenv("PBRCM_TUNING", str(path))
    monkeypatch.setenv("PBRCM_BATCH_CLUSTERS", "5")  # a knob still overrides one setting
    ctx = pbrcm.Context(0)
    try:
        t = pbrcm.tuning_get(ctx)
        assert t["source"] == 1
        assert (t["batch_pool"], t["cluster_size"], t["cluster_max"], t["cluster_nnz"],
                t["session_cutoff_n"]) == (3, 2, 5, 131072, 65536)
        mats = _calibration()[:16]
        got, res = pbrcm.reorder_batch(mats, reverse=True, ctx=ctx)
        ref, _ = pbrcm.reorder_batch(mats, reverse=True, ctx=pbrcm.Context(0))
        assert all(np.array_equal(a, b) for a, b in zip(got, ref))
    finally:
        ctx.close()
    assert os.path.exists(path)
