"""Regenerates the golden fixtures in tests/golden/ from the REFERENCE itself.

Every case is run through oracle/_ref/ref_rcm -- the reference's own CPU
sources (Graph::load, findPeripheral, rcm_seq<true>, computeBandwidth,
checkBandwidth), compiled unchanged by oracle/Makefile -- and its outputs are
stored next to the input pattern:

    <case>.npz: row_ptr, col_idx (the CSR the reference loader built),
                perm (Cuthill-McKee order, not reversed), start, passes, ecc,
                bandwidth, initial_bandwidth, max_valency

Cases given as MatrixMarket text go through the reference loader (parse,
sort, symmetry repair, connectivity repair); the others are raw CSRs.

Run in a container that has the reference sources:
    make -C oracle ref && python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from parallelbatchrcm_b200 import gen  # noqa: E402


def star(leaves: int, extra_every: int = 0, seed: int = 3) -> gen.Csr:
    """A hub joined to `leaves` leaves; every `extra_every`-th leaf also joins
    a ring of the leaves so that leaf valences differ (ties and non-ties)."""
    n = leaves + 1
    u = list(np.zeros(leaves, dtype=np.int64))
    v = list(np.arange(1, n, dtype=np.int64))
    if extra_every:
        for i in range(1, n - extra_every, extra_every):
            u.append(i)
            v.append(i + extra_every)
    u, v = np.array(u), np.array(v)
    p = np.random.default_rng(seed).permutation(n)
    return gen.from_edges(n, p[u], p[v])


def path(n: int, seed: int = 5) -> gen.Csr:
    p = np.random.default_rng(seed).permutation(n)
    a = np.arange(n - 1)
    return gen.from_edges(n, p[a], p[a + 1])


def caterpillar(spine: int, legs: int, seed: int = 9) -> gen.Csr:
    """A path whose nodes each carry `legs` pendant nodes: wide levels with
    many equal-valence children per parent."""
    n = spine * (legs + 1)
    u, v = [], []
    for i in range(spine - 1):
        u.append(i)
        v.append(i + 1)
    for i in range(spine):
        for k in range(legs):
            u.append(i)
            v.append(spine + i * legs + k)
    p = np.random.default_rng(seed).permutation(n)
    return gen.from_edges(n, p[np.array(u)], p[np.array(v)])


MTX_CASES = {
    # general pattern with duplicates and missing mirrors -> symmetry repair
    "mtx_general_dups": """%%MatrixMarket matrix coordinate real general
% single entries get mirrored; the (4,5) pair stored twice counts as matched
% (the loader's toggle map), so its mirror is never added; a blank data line
6 6 10
1 2 1.0
2 1 1.0

2 3 2.0
3 4 1.0
4 3 1.0
4 5 1.0
4 5 1.0
5 6 1.0
6 1 3.0
3 3 1.0
""",
    # three components -> connectivity repair
    "mtx_components": """%%MatrixMarket matrix coordinate pattern symmetric
9 9 8
1 1
2 1
3 2
5 4
6 5
6 6
8 7
9 8
""",
    # integer field, symmetric with diagonal
    "mtx_integer_sym": """%%MatrixMarket matrix coordinate integer symmetric
5 5 7
1 1 4
2 1 -1
3 2 -1
4 3 -1
5 4 -1
5 1 -1
3 3 4
""",
}


def csr_cases():
    return {
        "grid2d_64x64_s1": gen.grid2d(64, 64, seed=1),  # the single-matrix CPU config
        "grid2d_8x8_s3": gen.grid2d(8, 8, seed=3),
        "grid2d_17x5_natural": gen.grid2d(17, 5, seed=None),
        "grid3d_10x11x12_s5": gen.grid3d(10, 11, 12, seed=5),
        "rgg_3000_s11": gen.rgg(3000, seed=11),
        "rgg_20000_k4-12_s13": gen.rgg(20000, kmin=4, kmax=12, seed=13),
        "star_3000": star(3000),                      # hub row > 2048 edges
        "star_1500_ring7": star(1500, extra_every=7),  # big segment, mixed valences
        "path_300": path(300),
        "caterpillar_40x60": caterpillar(40, 60),
        "single_node": gen.Csr(np.array([0, 1], np.uint32), np.array([0], np.uint32)),
        "two_nodes": gen.from_edges(2, np.array([0]), np.array([1])),
    }


def save(name: str, rp, ci, info: dict, perm) -> None:
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"), row_ptr=np.asarray(rp, np.uint32), col_idx=np.asarray(ci, np.uint32),
        perm=np.asarray(perm, np.uint32), start=info["start"], passes=info["peripheral_passes"], ecc=info["ecc"],
        bandwidth=info["bandwidth"], initial_bandwidth=info["initial_bandwidth"],
        max_valency=info["max_valency"])
    print(f"{name:28s} n={info['n']:6d} nnz={info['nnz']:7d} start={info['start']} passes="
          f"{info['peripheral_passes']} ecc={info['ecc']} bw={info['initial_bandwidth']}->{info['bandwidth']}")


def main() -> None:
    if not O.ref_available():
        sys.exit("oracle/_ref/ref_rcm not built: run `make -C oracle ref` where the reference sources exist")
    for name, m in csr_cases().items():
        info, perm = O.ref_reorder_csr(m.row_ptr, m.col_idx)
        assert info["check_permutation"] == 0 and info["placed"] == m.n
        save(name, m.row_ptr, m.col_idx, info, perm)
    with tempfile.TemporaryDirectory() as td:
        for name, text in MTX_CASES.items():
            p = os.path.join(td, name + ".mtx")
            with open(p, "w") as f:
                f.write(text)
            with open(os.path.join(HERE, name + ".mtx"), "w") as f:
                f.write(text)
            info, rp, ci, perm = O.ref_load_and_reorder(p)
            save(name, rp, ci, info, perm)
        # the 64x64 grid also as the .mtx file the loader reads
        g = gen.grid2d(64, 64, seed=1)
        p = os.path.join(td, "c1.mtx")
        gen.write_mtx(g, p)
        info, rp, ci, perm = O.ref_load_and_reorder(p)
        assert np.array_equal(rp, g.row_ptr) and np.array_equal(ci, g.col_idx)
        save("mtx_grid2d_64x64_s1", rp, ci, info, perm)


if __name__ == "__main__":
    main()
