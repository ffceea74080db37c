"""The product loader (pbrcm_load_mtx / pbrcm_prepare_csr in libpbrcm, host
code) against the reference loader's output (golden) and the oracle."""
import numpy as np
import pytest

from conftest import load_golden
from test_oracle_golden import MTX_NAMES, golden_mtx_path


@pytest.mark.parametrize("name", MTX_NAMES)
def test_load_mtx_matches_reference(pbrcm, name, tmp_path):
    g = load_golden(name)
    rp, ci = pbrcm.load_mtx(golden_mtx_path(name, tmp_path))
    assert np.array_equal(rp, g["row_ptr"]) and np.array_equal(ci, g["col_idx"])


def _random_pattern(rng, n, m):
    r = rng.integers(0, n, m).astype(np.uint64)
    c = rng.integers(0, n, m).astype(np.uint64)
    key = np.sort((r << np.uint64(32)) | c)
    rows = (key >> np.uint64(32)).astype(np.int64)
    rp = np.zeros(n + 1, np.uint32)
    np.cumsum(np.bincount(rows, minlength=n), out=rp[1:])
    return rp, (key & np.uint64(0xFFFFFFFF)).astype(np.uint32)


@pytest.mark.parametrize("seed", range(6))
def test_prepare_csr_matches_oracle(pbrcm, oracle_mod, seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(5, 400))
    rp, ci = _random_pattern(rng, n, int(rng.integers(n, 4 * n)))
    # add the diagonal so that no row is empty (the loaders differ from the
    # reference only on rows with no entry at all)
    rp2, ci2 = [], []
    rows = np.repeat(np.arange(n), np.diff(rp))
    key = np.concatenate([(rows.astype(np.uint64) << np.uint64(32)) | ci.astype(np.uint64),
                          (np.arange(n, dtype=np.uint64) << np.uint64(32)) | np.arange(n, dtype=np.uint64)])
    key = np.sort(key)
    r = (key >> np.uint64(32)).astype(np.int64)
    rp = np.zeros(n + 1, np.uint32)
    np.cumsum(np.bincount(r, minlength=n), out=rp[1:])
    ci = (key & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    for check_sym in (True, False):
        a_rp, a_ci = pbrcm.prepare_csr(rp, ci, check_sym)
        b_rp, b_ci, _ = oracle_mod.prepare_csr(rp, ci, check_sym)
        assert np.array_equal(a_rp, b_rp) and np.array_equal(a_ci, b_ci)


@pytest.mark.parametrize("text", [
    "%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n",          # not coordinate
    "%%MatrixMarket matrix coordinate real skew-symmetric\n2 2 1\n1 2 1\n",  # unsupported symmetry
    "%%MatrixMarket matrix coordinate real general\n2 2 1\n0 1 1.0\n",       # index 0
    "%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1.0\n",       # index past the size
    "%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1 1.0\n2 2 1.0\n",  # more entries than declared
    "%%MatrixMarket matrix coordinate real general\n2 3 1\n1 1 1.0\n",       # not square
    "%%MatrixMarket matrix coordinate real general\n2 2 1\n1 x 1.0\n",       # garbage
])
def test_load_mtx_rejects_bad_input(pbrcm, tmp_path, text):
    p = tmp_path / "bad.mtx"
    p.write_text(text)
    with pytest.raises(pbrcm.PbrcmError) as e:
        pbrcm.load_mtx(str(p))
    assert e.value.name == "PBRCM_ERR_FORMAT"


def test_load_mtx_missing_file(pbrcm, tmp_path):
    with pytest.raises(pbrcm.PbrcmError) as e:
        pbrcm.load_mtx(str(tmp_path / "nope.mtx"))
    assert e.value.name == "PBRCM_ERR_IO"
    g = pbrcm.Graph()
    assert g.load(str(tmp_path / "nope.mtx")) == -1


def test_generators_are_loader_fixed_points(pbrcm, tmp_path):
    """A generated pattern written as .mtx and read back by the loader is
    unchanged: the generators emit exactly what the reference loader builds."""
    from parallelbatchrcm_b200 import gen
    for m in (gen.grid2d(9, 7, seed=2), gen.grid3d(4, 5, 3, seed=4), gen.rgg(800, seed=5)):
        p = str(tmp_path / "g.mtx")
        gen.write_mtx(m, p)
        rp, ci = pbrcm.load_mtx(p)
        assert np.array_equal(rp, m.row_ptr) and np.array_equal(ci, m.col_idx)
