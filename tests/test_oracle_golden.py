"""The C oracle (oracle/pbrcm_oracle.c) against the golden fixtures, which
were produced by the reference's own code (tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_names, load_golden


@pytest.mark.parametrize("name", golden_names())
def test_cm_order_matches_reference(oracle_mod, name):
    g = load_golden(name)
    perm = oracle_mod.cm_order(g["row_ptr"], g["col_idx"], int(g["start"]), True)
    assert np.array_equal(perm, g["perm"])


@pytest.mark.parametrize("name", golden_names())
def test_peripheral_matches_reference(oracle_mod, name):
    g = load_golden(name)
    s, passes, ecc = oracle_mod.peripheral(g["row_ptr"], g["col_idx"])
    assert (s, passes, ecc) == (int(g["start"]), int(g["passes"]), int(g["ecc"]))


@pytest.mark.parametrize("name", golden_names())
def test_bandwidths_match_reference(oracle_mod, name):
    g = load_golden(name)
    assert oracle_mod.bandwidth(g["row_ptr"], g["col_idx"], g["perm"]) == int(g["bandwidth"])
    assert oracle_mod.initial_bandwidth(g["row_ptr"], g["col_idx"]) == int(g["initial_bandwidth"])
    assert oracle_mod.max_valency(g["row_ptr"]) == int(g["max_valency"])
    assert oracle_mod.check_permutation(g["perm"])


def golden_mtx_path(name, tmp_path):
    """The MatrixMarket input of a golden case (kept in tests/golden, or the
    64x64 grid regenerated by the seeded generator)."""
    path = os.path.join(GOLDEN, name + ".mtx")
    if os.path.exists(path):
        return path
    if name == "mtx_grid2d_64x64_s1":
        from parallelbatchrcm_b200 import gen
        path = str(tmp_path / "c1.mtx")
        gen.write_mtx(gen.grid2d(64, 64, seed=1), path)
        return path
    pytest.skip("no .mtx for this case")


MTX_NAMES = [n for n in golden_names() if n.startswith("mtx_")]


@pytest.mark.parametrize("name", MTX_NAMES)
def test_oracle_loader_matches_reference(oracle_mod, name, tmp_path):
    g = load_golden(name)
    rp, ci, _ = oracle_mod.load_mtx(golden_mtx_path(name, tmp_path))
    assert np.array_equal(rp, g["row_ptr"]) and np.array_equal(ci, g["col_idx"])


def test_profile_definition(oracle_mod):
    # path 0-1-2 in natural order: rows 1 and 2 reach one column back
    rp = np.array([0, 2, 5, 7], np.uint32)
    ci = np.array([0, 1, 0, 1, 2, 1, 2], np.uint32)
    assert oracle_mod.profile(rp, ci, np.array([0, 1, 2], np.uint32)) == 2
    assert oracle_mod.bandwidth(rp, ci, np.array([0, 2, 1], np.uint32)) == 2
