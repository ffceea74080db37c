"""Seeded synthetic sparse-matrix patterns for the RCM workloads.

The reference reorders SuiteSparse matrices that it downloads at run time
(mats/get_sample_matrices.py); none ship with it and this project has no
network, so its workloads are seeded synthetic patterns of the same kinds:

* ``grid2d``  -- 5-point Laplacian pattern of an nx x ny grid,
* ``grid3d``  -- 7-point Laplacian pattern of an nx x ny x nz grid,
* ``rgg``     -- random geometric graph: points uniform in the unit square,
  each joined to its k nearest neighbours (k drawn per point), symmetrised,
  plus a fraction of random long-range edges,

each with the diagonal stored and node labels shuffled by a seeded random
permutation.  Every generator returns the CSR that the reference loader
(Graph::load, Graph.h:266-332) builds from the matching MatrixMarket file:
rows sorted by column, symmetric, no duplicate entries, and connected by the
loader's rule (Graph.h:160-263: each further component, in order of its
smallest node m, gets the link (m-1, m)).  ``write_mtx`` writes that file.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

__all__ = [
    "Csr", "grid2d", "grid3d", "rgg", "erdos_renyi", "from_edges", "connect_components",
    "write_mtx", "mixed_batch_specs", "make_from_spec", "poisson_stream_specs",
]


@dataclass
class Csr:
    """A square sparse pattern: row_ptr (n+1, uint32), col_idx (nnz, uint32)."""
    row_ptr: np.ndarray
    col_idx: np.ndarray
    name: str = ""

    @property
    def n(self) -> int:
        return int(self.row_ptr.shape[0] - 1)

    @property
    def nnz(self) -> int:
        return int(self.col_idx.shape[0])


def _sorted_unique(key: np.ndarray) -> np.ndarray:
    """Sorted distinct values (np.unique is far slower than a sort here)."""
    key = np.sort(key)
    if key.shape[0] == 0:
        return key
    keep = np.empty(key.shape[0], dtype=bool)
    keep[0] = True
    np.not_equal(key[1:], key[:-1], out=keep[1:])
    return key[keep]


def from_edges(n: int, u: np.ndarray, v: np.ndarray, diag: bool = True) -> Csr:
    """CSR of the undirected pattern {u_i, v_i} (+ diagonal), deduplicated,
    rows sorted by column."""
    u = np.asarray(u, dtype=np.uint64)
    v = np.asarray(v, dtype=np.uint64)
    keep = u != v
    u, v = u[keep], v[keep]
    parts_r = [u, v]
    parts_c = [v, u]
    if diag:
        d = np.arange(n, dtype=np.uint64)
        parts_r.append(d)
        parts_c.append(d)
    key = (np.concatenate(parts_r) << np.uint64(32)) | np.concatenate(parts_c)
    key = _sorted_unique(key)
    rows = (key >> np.uint64(32)).astype(np.int64)
    cols = (key & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    rp = np.zeros(n + 1, dtype=np.uint64)
    np.cumsum(np.bincount(rows, minlength=n), out=rp[1:])
    if rp[-1] >= 2**32 - 1:
        raise ValueError("pattern too large for 32-bit offsets")
    return Csr(rp.astype(np.uint32), cols)


def connect_components(m: Csr) -> Csr:
    """Adds the links the reference loader adds to join components
    (Graph.h:160-263).  For a pattern whose rows are all non-empty the
    loader's BFS visits components in order of their smallest node m and links
    each later component by the edge (m-1, m)."""
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import connected_components

    n = m.n
    if n <= 1:
        return m
    if np.any(np.diff(m.row_ptr) == 0):
        raise ValueError("connect_components expects non-empty rows")
    a = csr_matrix((np.ones(m.nnz, dtype=np.int8), m.col_idx, m.row_ptr), shape=(n, n))
    ncomp, labels = connected_components(a, directed=False)
    if ncomp == 1:
        return m
    first = np.full(ncomp, n, dtype=np.int64)
    np.minimum.at(first, labels, np.arange(n))
    starts = np.sort(first)[1:]
    rows = np.repeat(np.arange(n, dtype=np.uint64), np.diff(m.row_ptr).astype(np.int64))
    key = np.concatenate([
        (rows << np.uint64(32)) | m.col_idx.astype(np.uint64),
        (starts.astype(np.uint64) - 1) << np.uint64(32) | starts.astype(np.uint64),
        starts.astype(np.uint64) << np.uint64(32) | (starts.astype(np.uint64) - 1),
    ])
    key = np.sort(key)  # the loader keeps duplicates (CSR.cpp:170-200)
    r = (key >> np.uint64(32)).astype(np.int64)
    rp = np.zeros(n + 1, dtype=np.uint64)
    np.cumsum(np.bincount(r, minlength=n), out=rp[1:])
    return Csr(rp.astype(np.uint32), (key & np.uint64(0xFFFFFFFF)).astype(np.uint32), m.name)


def _relabel(n: int, u: np.ndarray, v: np.ndarray, seed: int | None):
    if seed is None:
        return u, v
    p = np.random.default_rng(seed).permutation(n).astype(np.int64)
    return p[u], p[v]


def grid2d(nx: int, ny: int, seed: int | None = 1) -> Csr:
    """5-point Laplacian pattern on an nx x ny grid, labels shuffled with
    numpy default_rng(seed).permutation (seed None = natural order)."""
    idx = np.arange(nx * ny, dtype=np.int64).reshape(ny, nx)
    u = np.concatenate([idx[:, :-1].ravel(), idx[:-1, :].ravel()])
    v = np.concatenate([idx[:, 1:].ravel(), idx[1:, :].ravel()])
    u, v = _relabel(nx * ny, u, v, seed)
    m = from_edges(nx * ny, u, v)
    m.name = f"grid2d_{nx}x{ny}_s{seed}"
    return m


def grid3d(nx: int, ny: int, nz: int, seed: int | None = 12345) -> Csr:
    """7-point Laplacian pattern on an nx x ny x nz grid, labels shuffled."""
    idx = np.arange(nx * ny * nz, dtype=np.int64).reshape(nz, ny, nx)
    u = np.concatenate([idx[:, :, :-1].ravel(), idx[:, :-1, :].ravel(), idx[:-1, :, :].ravel()])
    v = np.concatenate([idx[:, :, 1:].ravel(), idx[:, 1:, :].ravel(), idx[1:, :, :].ravel()])
    u, v = _relabel(nx * ny * nz, u, v, seed)
    m = from_edges(nx * ny * nz, u, v)
    m.name = f"grid3d_{nx}x{ny}x{nz}_s{seed}"
    return m


def rgg(n: int, kmin: int = 6, kmax: int = 14, long_frac: float = 0.001, seed: int = 7,
        connect: bool = True) -> Csr:
    """Random geometric graph: n points uniform in [0,1]^2, point i joined to
    its k_i ~ U{kmin..kmax} nearest neighbours, symmetrised, plus
    round(long_frac * |E|) uniformly random long-range edges; labels shuffled;
    components joined by the loader's rule (connect=False: left apart)."""
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    pts = rng.random((n, 2))
    k = rng.integers(kmin, kmax + 1, size=n)
    kq = min(kmax + 1, n)
    _, nb = cKDTree(pts).query(pts, k=kq)
    nb = np.asarray(nb, dtype=np.int64).reshape(n, kq)
    take = np.arange(kq)[None, :] <= k[:, None]
    take[:, 0] = False  # column 0 is the point itself
    u = np.repeat(np.arange(n, dtype=np.int64), take.sum(axis=1))
    v = nb[take]
    lo, hi = np.minimum(u, v), np.maximum(u, v)
    e = _sorted_unique(lo * n + hi)
    nlong = int(round(long_frac * e.shape[0]))
    a = rng.integers(0, n, size=nlong)
    b = rng.integers(0, n, size=nlong)
    u = np.concatenate([e // n, a])
    v = np.concatenate([e % n, b])
    u, v = _relabel(n, u, v, seed + 1)
    m = from_edges(n, u, v)
    if connect:
        m = connect_components(m)
    m.name = f"rgg_{n}_k{kmin}-{kmax}_s{seed}" + ("" if connect else "_raw")
    return m


def erdos_renyi(n: int, deg: int, seed: int = 2) -> Csr:
    """Random graph: n * deg / 2 uniformly random node pairs (self pairs and
    repeats merge), symmetrised, joined by the loader's rule.  Its BFS levels
    are few and wide (2M nodes, degree 14: 10 levels, the widest 1.46M)."""
    rng = np.random.default_rng(seed)
    m = n * deg // 2
    g = connect_components(from_edges(n, rng.integers(0, n, m), rng.integers(0, n, m)))
    g.name = f"er_{n}_d{deg}_s{seed}"
    return g


def write_mtx(m: Csr, path: str, symmetric: bool = True, field: str = "real") -> None:
    """Writes the pattern as MatrixMarket coordinate (values 1).  symmetric:
    lower triangle incl. diagonal, as the loader expects for `symmetric`."""
    n = m.n
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(m.row_ptr).astype(np.int64))
    cols = m.col_idx.astype(np.int64)
    if symmetric:
        keep = rows >= cols
        rows, cols = rows[keep], cols[keep]
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate {field} {'symmetric' if symmetric else 'general'}\n")
        f.write(f"{n} {n} {rows.shape[0]}\n")
        if field == "pattern":
            data = np.stack([rows + 1, cols + 1], axis=1)
            np.savetxt(f, data, fmt="%d %d")
        else:
            data = np.stack([rows + 1, cols + 1], axis=1)
            np.savetxt(f, data, fmt="%d %d 1.0")


# ---------------------------------------------------------------------------
# Workload streams (many-matrix batch and serving arrivals)
# ---------------------------------------------------------------------------

def _near_square(n: int):
    a = max(2, int(round(math.sqrt(n))))
    return a, max(2, int(round(n / a)))


def _near_cubic(n: int):
    a = max(2, int(round(n ** (1 / 3))))
    b = max(2, int(round(math.sqrt(n / a))))
    return a, b, max(2, int(round(n / (a * b))))


def mixed_batch_specs(count: int = 4096, nmin: int = 500, nmax: int = 200_000, seed: int = 42,
                      kmin: int = 4, kmax: int = 12):
    """Specs of the many-matrix batch: n log-uniform in [nmin, nmax]; 40% 2-D
    grids (near-square), 30% 3-D grids (near-cubic), 30% RGGs with k ~
    U{kmin..kmax}; each with its own seed."""
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(math.log(nmin), math.log(nmax), size=count)).astype(np.int64)
    kind = rng.choice(3, size=count, p=[0.4, 0.3, 0.3])
    seeds = rng.integers(1, 2**31 - 1, size=count)
    specs = []
    for i in range(count):
        if kind[i] == 0:
            specs.append(("grid2d", _near_square(int(n[i])), int(seeds[i])))
        elif kind[i] == 1:
            specs.append(("grid3d", _near_cubic(int(n[i])), int(seeds[i])))
        else:
            specs.append(("rgg", (int(n[i]), kmin, kmax), int(seeds[i])))
    return specs


def spec_nnz_estimate(spec) -> int:
    """Approximate nnz of a spec's matrix without building it (for sharding)."""
    kind, dims, _ = spec
    if kind == "grid2d":
        a, b = dims[0], dims[1]
        return 5 * a * b - 2 * (a + b)
    if kind == "grid3d":
        a, b, c = dims[0], dims[1], dims[2]
        return 7 * a * b * c - 2 * (a * b + b * c + a * c)
    n, kmin, kmax = dims
    return int(n * (1 + 1.5 * (kmin + kmax) / 2))


def make_from_spec(spec) -> Csr:
    kind, dims, seed = spec
    if kind == "grid2d":
        return grid2d(dims[0], dims[1], seed=seed)
    if kind == "grid3d":
        return grid3d(dims[0], dims[1], dims[2], seed=seed)
    if kind == "rgg":
        return rgg(dims[0], kmin=dims[1], kmax=dims[2], seed=seed)
    raise ValueError(kind)


def poisson_stream_specs(count: int, rate_per_s: float, nmin: int = 1000, nmax: int = 2_000_000,
                         seed: int = 99):
    """Serving stream: (arrival_time_s, spec) with Poisson arrivals at
    rate_per_s and n log-uniform in [nmin, nmax] over the three kinds (equal
    shares); RGGs use k ~ U{6..14}."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_per_s, size=count)
    t = np.cumsum(gaps) - gaps[0]
    n = np.exp(rng.uniform(math.log(nmin), math.log(nmax), size=count)).astype(np.int64)
    kind = rng.integers(0, 3, size=count)
    seeds = rng.integers(1, 2**31 - 1, size=count)
    out = []
    for i in range(count):
        if kind[i] == 0:
            spec = ("grid2d", _near_square(int(n[i])), int(seeds[i]))
        elif kind[i] == 1:
            spec = ("grid3d", _near_cubic(int(n[i])), int(seeds[i]))
        else:
            spec = ("rgg", (int(n[i]), 6, 14), int(seeds[i]))
        out.append((float(t[i]), spec))
    return out
