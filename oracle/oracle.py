"""ctypes wrapper of the parity oracle -- TEST INFRASTRUCTURE ONLY.

Loads oracle/libpbrcm_oracle.so (the C restatement in pbrcm_oracle.c) and,
when built, drives oracle/_ref/ref_rcm (the reference's own CPU sources).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the product never does.
"""
from __future__ import annotations

import ctypes
import json
import os
import shutil
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpbrcm_oracle.so")
REF_BIN = os.path.join(HERE, "_ref", "ref_rcm")
REF_GPU_BIN = os.path.join(HERE, "_ref", "ref_gpu_simple")

_u32p = ctypes.POINTER(ctypes.c_uint32)
_lib = None


def build(ref_dir: str | None = None) -> None:
    """Builds the oracle library (and, given the reference's source tree, the
    reference driver) with oracle/Makefile."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if ref_dir:
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF_DIR={ref_dir}"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_cm_order.restype = ctypes.c_int64
        L.orc_cm_order.argtypes = [ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint32, ctypes.c_int, _u32p]
        L.orc_peripheral.restype = ctypes.c_int64
        L.orc_peripheral.argtypes = [ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint32, _u32p, _u32p]
        L.orc_bandwidth.restype = ctypes.c_int64
        L.orc_bandwidth.argtypes = [ctypes.c_uint32, _u32p, _u32p, _u32p]
        L.orc_initial_bandwidth.restype = ctypes.c_int64
        L.orc_initial_bandwidth.argtypes = [ctypes.c_uint32, _u32p, _u32p]
        L.orc_max_valency.restype = ctypes.c_int64
        L.orc_max_valency.argtypes = [ctypes.c_uint32, _u32p]
        L.orc_profile.restype = ctypes.c_uint64
        L.orc_profile.argtypes = [ctypes.c_uint32, _u32p, _u32p, _u32p]
        L.orc_check_permutation.restype = ctypes.c_int
        L.orc_check_permutation.argtypes = [ctypes.c_uint32, _u32p]
        L.orc_csr_new.restype = ctypes.c_void_p
        L.orc_csr_delete.argtypes = [ctypes.c_void_p]
        L.orc_csr_n.restype = ctypes.c_uint32
        L.orc_csr_n.argtypes = [ctypes.c_void_p]
        L.orc_csr_nnz.restype = ctypes.c_uint64
        L.orc_csr_nnz.argtypes = [ctypes.c_void_p]
        L.orc_csr_rp.restype = _u32p
        L.orc_csr_rp.argtypes = [ctypes.c_void_p]
        L.orc_csr_ci.restype = _u32p
        L.orc_csr_ci.argtypes = [ctypes.c_void_p]
        L.orc_csr_added_links.restype = ctypes.c_uint32
        L.orc_csr_added_links.argtypes = [ctypes.c_void_p]
        L.orc_csr_added_entries.restype = ctypes.c_uint32
        L.orc_csr_added_entries.argtypes = [ctypes.c_void_p]
        L.orc_load_mtx.restype = ctypes.c_int
        L.orc_load_mtx.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
        L.orc_prepare_csr.restype = ctypes.c_int
        L.orc_prepare_csr.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, _u32p, _u32p,
                                      ctypes.c_int]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(_u32p)


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint32)


def cm_order(rp, ci, start: int, sort_by_degree: bool = True) -> np.ndarray:
    """Cuthill-McKee order (not reversed) from `start`; rcm_cpu.cpp:57-104."""
    rp, ci = _u32(rp), _u32(ci)
    n = rp.shape[0] - 1
    perm = np.zeros(max(n, 1), dtype=np.uint32)
    got = lib().orc_cm_order(n, _p(rp), _p(ci), start, int(sort_by_degree), _p(perm))
    if got < 0:
        raise ValueError(f"orc_cm_order failed: {got}")
    return perm[:got]


def peripheral(rp, ci, outputnodes: int = 32):
    """(start, passes, ecc); simple_peripheral.cpp:92-141."""
    rp, ci = _u32(rp), _u32(ci)
    n = rp.shape[0] - 1
    it = ctypes.c_uint32(0)
    ecc = ctypes.c_uint32(0)
    s = lib().orc_peripheral(n, _p(rp), _p(ci), outputnodes, ctypes.byref(it), ctypes.byref(ecc))
    if s < 0:
        raise ValueError(f"orc_peripheral failed: {s}")
    return int(s), int(it.value), int(ecc.value)


def bandwidth(rp, ci, perm) -> int:
    rp, ci, perm = _u32(rp), _u32(ci), _u32(perm)
    return int(lib().orc_bandwidth(rp.shape[0] - 1, _p(rp), _p(ci), _p(perm)))


def initial_bandwidth(rp, ci) -> int:
    rp, ci = _u32(rp), _u32(ci)
    return int(lib().orc_initial_bandwidth(rp.shape[0] - 1, _p(rp), _p(ci)))


def max_valency(rp) -> int:
    rp = _u32(rp)
    return int(lib().orc_max_valency(rp.shape[0] - 1, _p(rp)))


def profile(rp, ci, perm) -> int:
    rp, ci, perm = _u32(rp), _u32(ci), _u32(perm)
    return int(lib().orc_profile(rp.shape[0] - 1, _p(rp), _p(ci), _p(perm)))


def check_permutation(perm) -> bool:
    perm = _u32(perm)
    return lib().orc_check_permutation(perm.shape[0], _p(perm)) == 0


def _take_csr(h):
    L = lib()
    n = L.orc_csr_n(h)
    nnz = L.orc_csr_nnz(h)
    rp = np.ctypeslib.as_array(L.orc_csr_rp(h), shape=(n + 1,)).copy()
    ci = np.ctypeslib.as_array(L.orc_csr_ci(h), shape=(max(nnz, 1),))[:nnz].copy()
    info = {"added_links": int(L.orc_csr_added_links(h)), "added_entries": int(L.orc_csr_added_entries(h))}
    L.orc_csr_delete(h)
    return rp, ci, info


def load_mtx(path: str):
    """(row_ptr, col_idx, info) as Graph::load builds them (no cache files)."""
    L = lib()
    h = L.orc_csr_new()
    rc = L.orc_load_mtx(path.encode(), h)
    if rc != 0:
        L.orc_csr_delete(h)
        raise ValueError(f"orc_load_mtx failed: {rc}")
    return _take_csr(h)


def prepare_csr(rp, ci, check_sym: bool = True):
    """prepareRCM (Graph.h:74-264) on a raw CSR."""
    rp, ci = _u32(rp), _u32(ci)
    L = lib()
    h = L.orc_csr_new()
    rc = L.orc_prepare_csr(h, rp.shape[0] - 1, ci.shape[0], _p(rp), _p(ci), int(check_sym))
    if rc != 0:
        L.orc_csr_delete(h)
        raise ValueError(f"orc_prepare_csr failed: {rc}")
    return _take_csr(h)


def full_reorder(rp, ci, start: int | None = None, reverse: bool = True):
    """What the drop-in returns: {perm, start, bandwidth, profile, passes, ecc}
    with automatic start unless given, CM order reversed when `reverse`."""
    passes = ecc = 0
    if start is None:
        start, passes, ecc = peripheral(rp, ci)
    cm = cm_order(rp, ci, start, True)
    perm = cm[::-1].copy() if reverse else cm
    return {
        "perm": perm, "start": start, "bandwidth": bandwidth(rp, ci, perm),
        "profile": profile(rp, ci, perm), "passes": passes, "ecc": ecc,
    }


# --------------------------------------------------------------------------
# The reference itself (oracle/_ref/ref_rcm), where it has been built.
# --------------------------------------------------------------------------

def ref_available() -> bool:
    return os.path.exists(REF_BIN)


def _parse_json(out: str) -> dict:
    for line in out.splitlines()[::-1]:
        if line.startswith("JSON "):
            return json.loads(line[5:])
    raise RuntimeError(f"no JSON line in reference output: {out[-500:]}")


def ref_load_and_reorder(mtx_path: str, start: int | None = None):
    """Runs the reference's Graph::load + findPeripheral + rcm_seq<true> on a
    copy of `mtx_path` in a scratch dir (the loader writes cache files next to
    its input).  Returns (info dict, row_ptr, col_idx, perm)."""
    with tempfile.TemporaryDirectory() as td:
        src = os.path.join(td, "m.mtx")
        shutil.copyfile(mtx_path, src)
        out = os.path.join(td, "out")
        cmd = [REF_BIN, "load", src, out] + ([str(start)] if start is not None else [])
        r = subprocess.run(cmd, capture_output=True, text=True, check=True)
        info = _parse_json(r.stdout)
        rp = np.fromfile(out + ".rp", dtype=np.uint32)
        ci = np.fromfile(out + ".ci", dtype=np.uint32)
        perm = np.fromfile(out + ".perm", dtype=np.uint32)
    return info, rp, ci, perm


def ref_reorder_csr(rp, ci, start: int | None = None):
    """The reference's findPeripheral + rcm_seq<true> on a raw CSR.
    Returns (info dict, perm)."""
    with tempfile.TemporaryDirectory() as td:
        _u32(rp).tofile(os.path.join(td, "rp"))
        _u32(ci).tofile(os.path.join(td, "ci"))
        out = os.path.join(td, "out")
        cmd = [REF_BIN, "csr", os.path.join(td, "rp"), os.path.join(td, "ci"), out]
        if start is not None:
            cmd.append(str(start))
        r = subprocess.run(cmd, capture_output=True, text=True, check=True)
        info = _parse_json(r.stdout)
        perm = np.fromfile(out + ".perm", dtype=np.uint32)
    return info, perm


def ref_time(rp, ci, threads: int, steps: int, timeout: float | None = None):
    """Times `steps` full reorders (findPeripheral + RealCPU::rcm<true>) on
    the host with the reference's own code.  Returns a list of dicts."""
    with tempfile.TemporaryDirectory() as td:
        _u32(rp).tofile(os.path.join(td, "rp"))
        _u32(ci).tofile(os.path.join(td, "ci"))
        r = subprocess.run([REF_BIN, "time", os.path.join(td, "rp"), os.path.join(td, "ci"),
                            str(threads), str(steps)], capture_output=True, text=True, check=True,
                           timeout=timeout)
    return [json.loads(line[5:]) for line in r.stdout.splitlines() if line.startswith("JSON ")]


def ref_gpu_simple(rp, ci, start: int, timeout: float | None = 600):
    """The reference's own GPU_SIMPLE::rcm (src/device/rcm_gpu.cu) from
    `start` (oracle/_ref/ref_gpu_simple): (mean ms of its 20 timed runs, CM
    order).  None if that build is missing."""
    if not os.path.exists(REF_GPU_BIN):
        return None
    with tempfile.TemporaryDirectory() as td:
        _u32(rp).tofile(os.path.join(td, "rp"))
        _u32(ci).tofile(os.path.join(td, "ci"))
        out = os.path.join(td, "out")
        r = subprocess.run([REF_GPU_BIN, os.path.join(td, "rp"), os.path.join(td, "ci"), str(int(start)), out],
                           capture_output=True, text=True, check=True, timeout=timeout)
        info = _parse_json(r.stdout)
        perm = np.fromfile(out + ".perm", dtype=np.uint32)
    return info["ms"], perm


def write_pack(path: str, mats) -> None:
    """Writes CSRs [(row_ptr, col_idx), ...] as one pack file: u64 count, then
    per matrix u64 n, u64 nnz, row_ptr (n+1 u32), col_idx (nnz u32)."""
    with open(path, "wb") as f:
        f.write(np.uint64(len(mats)).tobytes())
        for rp, ci in mats:
            rp, ci = _u32(rp), _u32(ci)
            f.write(np.array([rp.shape[0] - 1, ci.shape[0]], dtype=np.uint64).tobytes())
            f.write(rp.tobytes())
            f.write(ci.tobytes())


def ref_time_batch(mats, threads: int, reps: int = 1, timeout: float | None = None, want_perms: bool = False):
    """The reference's findPeripheral + rcm_seq<true> over a stream of
    matrices on `threads` host threads (oracle/_ref/ref_rcm timebatch), `reps`
    times over the loaded graphs.  Returns (one info dict per rep with
    wall_ms, start nodes, FNV-1a hashes of the CM orders) and, with
    want_perms, a fourth item: the CM orders (one uint32 array per matrix)."""
    with tempfile.TemporaryDirectory() as td:
        pack = os.path.join(td, "pack")
        write_pack(pack, mats)
        out = os.path.join(td, "out")
        r = subprocess.run([REF_BIN, "timebatch", pack, str(threads), out, str(reps)], capture_output=True,
                           text=True, check=True, timeout=timeout)
        info = [json.loads(line[5:]) for line in r.stdout.splitlines() if line.startswith("JSON ")]
        raw = np.fromfile(out + ".hash", dtype=np.uint32).reshape(-1, 4)
        allp = np.fromfile(out + ".perm", dtype=np.uint32) if want_perms else None
    starts = raw[:, 0].copy()
    hashes = raw[:, 2].astype(np.uint64) | (raw[:, 3].astype(np.uint64) << np.uint64(32))
    if not want_perms:
        return info, starts, hashes
    ns = np.array([np.asarray(rp).shape[0] - 1 for rp, _ in mats], dtype=np.int64)
    offs = np.concatenate([[0], np.cumsum(ns)])
    perms = [allp[offs[i]:offs[i + 1]] for i in range(len(mats))]
    return info, starts, hashes, perms


def fnv1a_u32(a) -> int:
    """FNV-1a over the u32 words of `a`, as ref_rcm timebatch hashes a
    permutation."""
    h = 1469598103934665603
    for v in _u32(a).tolist():
        h = ((h ^ v) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def permute_csr(rp, ci, perm, vals=None):
    """B = P A P^T as the reference's -o path computes it
    (include/device/rcm_cusolver.cuh:154-185: cusolverSpXcsrpermHost with
    p = q = perm, then apply_permutation_in_place of the values through its
    map): row i of B is row perm[i] of A, columns renamed through the inverse
    permutation and sorted, equal columns in their original order.  Returns
    (row_ptr, col_idx, vals or None, map)."""
    rp, ci, perm = _u32(rp).astype(np.int64), _u32(ci).astype(np.int64), _u32(perm).astype(np.int64)
    n = rp.shape[0] - 1
    inv = np.empty(n, np.int64)
    inv[perm] = np.arange(n)
    lens = (rp[1:] - rp[:-1])[perm]
    out_rp = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=out_rp[1:])
    row = np.repeat(np.arange(n), lens)
    idx = rp[perm][row] + (np.arange(out_rp[-1]) - out_rp[row])
    newc = inv[ci[idx]] if idx.size else np.zeros(0, np.int64)
    order = np.lexsort((newc, row))  # stable: by row, then new column
    m = idx[order]
    return (out_rp.astype(np.uint32), newc[order].astype(np.uint32),
            (np.asarray(vals)[m] if vals is not None else None), m.astype(np.uint32))


def ref_store_mtx(rp, ci, vals, path: str) -> None:
    """The reference's convert(COO, CSR) + storeMTX (src/CSR.cpp:210-231,
    src/COO.cpp:213-251) on a CSR with float64 (or float32) values."""
    with tempfile.TemporaryDirectory() as td:
        _u32(rp).tofile(os.path.join(td, "rp"))
        _u32(ci).tofile(os.path.join(td, "ci"))
        v = np.asarray(vals)
        v.tofile(os.path.join(td, "v"))
        mode = "store64" if v.dtype == np.float64 else "store32"
        subprocess.run([REF_BIN, mode, os.path.join(td, "rp"), os.path.join(td, "ci"), os.path.join(td, "v"), path],
                       capture_output=True, text=True, check=True)


def ref_read_hicsr(path: str, dtype):
    """The reference's loadCSR<float|double> on a .hicsr file: (rp, ci, vals)."""
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "o")
        mode = "hicsr64" if np.dtype(dtype) == np.float64 else "hicsr32"
        subprocess.run([REF_BIN, mode, path, out], capture_output=True, text=True, check=True)
        return (np.fromfile(out + ".rp", dtype=np.uint32), np.fromfile(out + ".ci", dtype=np.uint32),
                np.fromfile(out + ".v", dtype=dtype))


def ref_load_caches(mtx_path: str, workdir: str):
    """Runs the reference's Graph<float>::load on a copy of `mtx_path` in
    `workdir`; returns the paths of the .hicsr and .rcm.hicsr caches it wrote
    (include/Graph.h:266-332)."""
    src = os.path.join(workdir, "m.mtx")
    shutil.copyfile(mtx_path, src)
    subprocess.run([REF_BIN, "load", src, os.path.join(workdir, "out")], capture_output=True, text=True, check=True)
    return src + ".hicsr", src + ".rcm.hicsr"
