"""The output boundary on CPU: pbrcm_store_mtx against the reference's own
convert + storeMTX (byte for byte), and the oracle's P A P^T against its
definition B[i, j] = A[perm[i], perm[j]]."""
import os

import numpy as np
import pytest


def _random_csr(rng, n, per_row):
    rows = []
    for i in range(n):
        k = int(rng.integers(0, per_row + 1))
        rows.append(np.sort(rng.integers(0, n, k)).astype(np.uint32))
    rp = np.zeros(n + 1, np.uint32)
    np.cumsum([len(r) for r in rows], out=rp[1:])
    return rp, (np.concatenate(rows) if rows else np.zeros(0, np.uint32)).astype(np.uint32)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_store_mtx_matches_reference(pbrcm, oracle_mod, tmp_path, dtype):
    if not oracle_mod.ref_available():
        pytest.skip("reference CPU build not present")
    rng = np.random.default_rng(5)
    rp, ci = _random_csr(rng, 300, 9)
    vals = (rng.standard_normal(ci.shape[0]) * 10.0 ** rng.integers(-3, 6, ci.shape[0])).astype(dtype)
    ours, ref = str(tmp_path / "ours.mtx"), str(tmp_path / "ref.mtx")
    pbrcm.store_mtx(ours, rp, ci, vals)
    oracle_mod.ref_store_mtx(rp, ci, vals, ref)
    assert open(ours, "rb").read() == open(ref, "rb").read()


def test_store_mtx_pattern(pbrcm, tmp_path):
    rp = np.array([0, 2, 3], np.uint32)
    ci = np.array([0, 1, 1], np.uint32)
    path = str(tmp_path / "p.mtx")
    pbrcm.store_mtx(path, rp, ci)
    assert open(path).read() == "%%MatrixMarket matrix coordinate pattern general\n2 2 3\n1 1\n1 2\n2 2\n"


@pytest.mark.parametrize("seed", range(4))
def test_oracle_permute_is_p_a_pt(oracle_mod, seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 60))
    rp, ci = _random_csr(rng, n, 6)
    perm = rng.permutation(n).astype(np.uint32)
    vals = rng.standard_normal(ci.shape[0])
    orp, oci, ov, m = oracle_mod.permute_csr(rp, ci, perm, vals)
    # B[i, j] = A[perm[i], perm[j]], multiplicities and values included
    A = {}
    for r in range(n):
        for k in range(rp[r], rp[r + 1]):
            A.setdefault((r, int(ci[k])), []).append(vals[k])
    B = {}
    for i in range(n):
        cols = oci[orp[i]:orp[i + 1]]
        assert np.all(np.diff(cols.astype(np.int64)) >= 0)
        for k in range(orp[i], orp[i + 1]):
            B.setdefault((int(perm[i]), int(perm[oci[k]])), []).append(ov[k])
            assert ov[k] == vals[m[k]]
    assert A == B


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_hicsr_written_here_reads_in_the_reference(pbrcm, oracle_mod, tmp_path, dtype):
    if not oracle_mod.ref_available():
        pytest.skip("reference CPU build not present")
    rng = np.random.default_rng(9)
    rp, ci = _random_csr(rng, 200, 8)
    vals = rng.standard_normal(ci.shape[0]).astype(dtype)
    path = str(tmp_path / "m.hicsr")
    pbrcm.store_hicsr(path, rp, ci, vals)
    r_rp, r_ci, r_v = oracle_mod.ref_read_hicsr(path, dtype)
    assert np.array_equal(r_rp, rp) and np.array_equal(r_ci, ci) and np.array_equal(r_v, vals)
    o_rp, o_ci, o_v = pbrcm.load_hicsr(path)
    assert np.array_equal(o_rp, rp) and np.array_equal(o_ci, ci) and np.array_equal(o_v, vals)


def test_hicsr_caches_of_the_reference_read_here(pbrcm, oracle_mod, tmp_path):
    """The caches Graph<float>::load writes next to a MatrixMarket input: the
    raw CSR (.hicsr) equals this loader's parse before prepareRCM, the prepared
    one (.rcm.hicsr) the golden CSR."""
    if not oracle_mod.ref_available():
        pytest.skip("reference CPU build not present")
    from conftest import load_golden
    from test_oracle_golden import MTX_NAMES, golden_mtx_path
    for name in MTX_NAMES:
        d = tmp_path / name
        d.mkdir()
        raw, prepared = oracle_mod.ref_load_caches(golden_mtx_path(name, tmp_path), str(d))
        g = load_golden(name)
        p_rp, p_ci, p_v = pbrcm.load_hicsr(prepared)
        assert np.array_equal(p_rp, g["row_ptr"]) and np.array_equal(p_ci, g["col_idx"]), name
        assert p_v.dtype == np.float32
        r_rp, r_ci, _ = pbrcm.load_hicsr(raw)
        q_rp, q_ci = pbrcm.prepare_csr(r_rp, r_ci, True)
        assert np.array_equal(q_rp, g["row_ptr"]) and np.array_equal(q_ci, g["col_idx"]), name


def test_hicsr_rejects_other_files(pbrcm, tmp_path):
    path = tmp_path / "x.hicsr"
    path.write_bytes(b"not a csr cache" * 10)
    with pytest.raises(pbrcm.PbrcmError) as e:
        pbrcm.load_hicsr(str(path))
    assert e.value.name == "PBRCM_ERR_FORMAT"
