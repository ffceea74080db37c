"""Python host API over libpbrcm (the C ABI in include/pbrcm.h).

Two layers:

* array API -- ``reorder``, ``reorder_device``, ``find_peripheral``,
  ``bandwidth``, ``reorder_batch``, ``Session``, ``load_mtx``,
  ``prepare_csr``: numpy host arrays (or torch CUDA tensors for the device
  forms) in, numpy / tensors out.
* reference-shaped API -- ``Graph``, ``GPU_BATCH.rcm``,
  ``SimplePeripheral.find_peripheral``, ``compute_bandwidth``,
  ``check_bandwidth``, ``max_valency``, ``check_permutation``: the names,
  argument meaning and error behaviour of the reference's GPU_BATCH surface
  (include/rcm_gpu_batch.h:40-41, include/simple_peripheral.h:46,
  src/main.cpp:94-226), so that code written against the reference reads the
  same.

Every call runs on the GPU through libpbrcm; a failing status raises
``PbrcmError`` (the reference throws std::runtime_error on a device error,
src/device/rcm_gpu_batch.cu:84-87).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Iterable, Sequence

import numpy as np

from . import _lib
from ._lib import AUTO_START, DEBUG_PHANTOM_CTA, Matrix, Options, Result, SessionConfig, SessionStats, Tuning

__all__ = [
    "PbrcmError", "Context", "default_options", "reorder", "reorder_device", "reorder_device_noalloc",
    "find_peripheral",
    "bandwidth", "reorder_batch", "reorder_batch_device", "Session", "load_mtx", "prepare_csr", "connect_device",
    "permute",
    "permute_device", "store_mtx", "load_hicsr", "store_hicsr", "autotune", "tuning_get", "tuning_set",
    "tuning_load",
    "Graph", "GPU_BATCH", "SimplePeripheral", "compute_bandwidth", "check_bandwidth", "max_valency",
    "check_permutation", "AUTO_START", "DEBUG_PHANTOM_CTA",
]


class PbrcmError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = int(status)
        self.name = _lib.STATUS.get(self.status, str(status))
        super().__init__(f"{what}: {self.name}" if what else self.name)


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise PbrcmError(rc, what)


def _u32(a) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return a


def _ptr(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


def default_options(reverse: bool = True, start: int | None = None, want_bandwidth: bool = True,
                    peripheral_nodes: int = 32, wait_limit_ms: int = 2000, debug_flags: int = 0,
                    stable: bool = True) -> Options:
    o = Options()
    _lib.lib().pbrcm_default_options(ctypes.byref(o))
    o.reverse = 1 if reverse else 0
    o.start_node = AUTO_START if start is None else int(start)
    o.want_bandwidth = 1 if want_bandwidth else 0
    o.peripheral_nodes = int(peripheral_nodes)
    o.wait_limit_ms = int(wait_limit_ms)
    o.debug_flags = int(debug_flags)
    o.stable = 1 if stable else 0
    return o


class Context:
    """A device context (stream + reusable device workspace)."""

    def __init__(self, device: int = -1):
        h = ctypes.c_void_p()
        _check(_lib.lib().pbrcm_context_create(int(device), ctypes.byref(h)), "pbrcm_context_create")
        self.handle = h

    def close(self) -> None:
        if self.handle:
            _lib.lib().pbrcm_context_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _h(ctx):
    return ctx.handle if ctx is not None else None


def reorder(row_ptr, col_idx, *, reverse: bool = True, start: int | None = None, want_bandwidth: bool = True,
            ctx: Context | None = None, perm_out: np.ndarray | None = None, raise_on_error: bool = True,
            **opt_kw):
    """Full reorder of one matrix from host arrays.  Returns (perm, result
    dict); perm[k] = original node at position k (reversed CM when
    `reverse`)."""
    rp, ci = _u32(row_ptr), _u32(col_idx)
    n = rp.shape[0] - 1
    perm = perm_out if perm_out is not None else np.empty(max(n, 1), dtype=np.uint32)
    res = Result()
    o = default_options(reverse=reverse, start=start, want_bandwidth=want_bandwidth, **opt_kw)
    rc = _lib.lib().pbrcm_reorder(_h(ctx), _ptr(rp), _ptr(ci), n, ci.shape[0], ctypes.byref(o), _ptr(perm),
                                  ctypes.byref(res))
    if raise_on_error:
        _check(rc, "pbrcm_reorder")
    d = res.as_dict()
    d["rc"] = rc
    return perm[:n], d


def reorder_device(row_ptr_t, col_idx_t, perm_t=None, *, reverse: bool = True, start: int | None = None,
                   want_bandwidth: bool = True, ctx: Context | None = None, stream=None, raise_on_error=True,
                   **opt_kw):
    """Full reorder of one matrix whose CSR is already on the GPU (torch
    int32/uint32 CUDA tensors).  Returns (perm tensor, result dict)."""
    import torch

    n = row_ptr_t.numel() - 1
    if perm_t is None:
        perm_t = torch.empty(n, dtype=torch.int32, device=row_ptr_t.device)
    res = Result()
    o = default_options(reverse=reverse, start=start, want_bandwidth=want_bandwidth, **opt_kw)
    st = ctypes.c_void_p(stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream)
    rc = _lib.lib().pbrcm_reorder_device(_h(ctx), ctypes.c_void_p(row_ptr_t.data_ptr()),
                                         ctypes.c_void_p(col_idx_t.data_ptr()), n, col_idx_t.numel(),
                                         ctypes.byref(o), ctypes.c_void_p(perm_t.data_ptr()), ctypes.byref(res), st)
    if raise_on_error:
        _check(rc, "pbrcm_reorder_device")
    d = res.as_dict()
    d["rc"] = rc
    return perm_t, d


def reorder_device_noalloc(row_ptr_t, col_idx_t, perm_t, *, reverse: bool = True, start: int | None = None,
                           want_bandwidth: bool = True, stream=None, raise_on_error: bool = True, **opt_kw):
    """Full reorder of a device-resident CSR that allocates no device memory
    (pbrcm_reorder_device_noalloc): for callers that cannot allocate while
    they run.  perm_t (n int32/uint32 on the GPU) receives the permutation.
    At most 2^20 nodes and rows of at most 1024 entries; calls that overlap on
    the GPU race on the shared scratch, so serialise them.  Returns the
    result dict."""
    import torch

    n = row_ptr_t.numel() - 1
    res = Result()
    o = default_options(reverse=reverse, start=start, want_bandwidth=want_bandwidth, **opt_kw)
    st = ctypes.c_void_p(stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream)
    rc = _lib.lib().pbrcm_reorder_device_noalloc(ctypes.c_void_p(row_ptr_t.data_ptr()),
                                                 ctypes.c_void_p(col_idx_t.data_ptr()), n, col_idx_t.numel(),
                                                 ctypes.byref(o), ctypes.c_void_p(perm_t.data_ptr()),
                                                 ctypes.byref(res), st)
    if raise_on_error:
        _check(rc, "pbrcm_reorder_device_noalloc")
    d = res.as_dict()
    d["rc"] = rc
    return d


def find_peripheral(row_ptr, col_idx, ctx: Context | None = None):
    """(start, passes, eccentricity) of the pseudo-peripheral search
    (src/simple_peripheral.cpp:92-141) on the GPU."""
    rp, ci = _u32(row_ptr), _u32(col_idx)
    s, p, e = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
    _check(_lib.lib().pbrcm_find_peripheral(_h(ctx), _ptr(rp), _ptr(ci), rp.shape[0] - 1, ci.shape[0],
                                            ctypes.byref(s), ctypes.byref(p), ctypes.byref(e)),
           "pbrcm_find_peripheral")
    return s.value, p.value, e.value


def bandwidth(row_ptr, col_idx, perm, ctx: Context | None = None):
    """(bandwidth, initial_bandwidth, profile) of `perm` on the GPU."""
    rp, ci, pm = _u32(row_ptr), _u32(col_idx), _u32(perm)
    bw, bw0, prof = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_uint64()
    _check(_lib.lib().pbrcm_bandwidth(_h(ctx), _ptr(rp), _ptr(ci), rp.shape[0] - 1, ci.shape[0], _ptr(pm),
                                      ctypes.byref(bw), ctypes.byref(bw0), ctypes.byref(prof)), "pbrcm_bandwidth")
    return bw.value, bw0.value, prof.value


# the pbrcm_matrix array of a batch as a numpy record view, so that a batch
# of thousands of matrices is described by column assignments rather than
# one ctypes field write at a time
_MATRIX_DTYPE = np.dtype({
    "names": [n for n, _ in Matrix._fields_],
    "formats": [np.uint64, np.uint64, np.uint32, np.uint32, np.uint64, np.uint64],
    "offsets": [getattr(Matrix, n).offset for n, _ in Matrix._fields_],
    "itemsize": ctypes.sizeof(Matrix),
})


def _addr(a: np.ndarray) -> int:
    """Data address of a numpy array (cheaper than a.ctypes.data)."""
    return a.__array_interface__["data"][0]


def _matrix_array(row_ptr, col_idx, n, nnz, perm_out):
    """pbrcm_matrix[len(n)] from per-matrix address / size lists."""
    arr = (Matrix * len(n))()
    if len(n):
        v = np.frombuffer(arr, dtype=_MATRIX_DTYPE)
        v["row_ptr"] = row_ptr
        v["col_idx"] = col_idx
        v["n"] = n
        v["nnz"] = nnz
        v["perm_out"] = perm_out
    return arr


class BatchResults(Sequence):
    """The per-matrix results of a batch: a sequence of result dicts, each
    built when first read (a batch of thousands of matrices returns without
    building them all)."""

    def __init__(self, res):
        self._res = res
        self._d = [None] * len(res)

    def __len__(self) -> int:
        return len(self._d)

    def __getitem__(self, i):
        if isinstance(i, slice):
            return [self[k] for k in range(*i.indices(len(self)))]
        if i < 0:
            i += len(self)
        d = self._d[i]
        if d is None:
            d = self._d[i] = self._res[i].as_dict()
        return d


class PreparedBatch:
    """A batch's matrix descriptors built once, for a caller that reorders the
    same buffers again and again (a service that refills fixed pinned
    staging, or device buffers, per call: the library then replays its
    captured launch, and the binding skips rebuilding thousands of
    descriptors).  Holds references to the buffers.

    Host form: ``PreparedBatch(mats, perms_out=None)`` with (row_ptr, col_idx)
    numpy arrays; device form: ``PreparedBatch(dmats, device=True)`` with
    (row_ptr, col_idx, perm_out) torch tensors.  Pass it to reorder_batch /
    reorder_batch_device in place of the list."""

    def __init__(self, mats: Sequence, perms_out: Sequence | None = None, device: bool = False):
        self.device = device
        self.count = len(mats)
        if device:
            self.mats = list(mats)
            self.ns = [m[0].numel() - 1 for m in self.mats]
            self.arr = _matrix_array([m[0].data_ptr() for m in self.mats], [m[1].data_ptr() for m in self.mats],
                                     self.ns, [m[1].numel() for m in self.mats],
                                     [m[2].data_ptr() for m in self.mats])
            return
        keep, perms, ns = [], [], []
        for i, m in enumerate(mats):
            rp, ci = _u32(m[0]), _u32(m[1])
            n = rp.shape[0] - 1
            if perms_out is not None:
                p = perms_out[i]
                if p.dtype != np.uint32 or not p.flags.c_contiguous or p.shape[0] < n:
                    raise ValueError("perms_out[i] must be a contiguous uint32 array of n entries")
            else:
                p = np.empty(max(n, 1), dtype=np.uint32)
            keep.append((rp, ci))
            perms.append(p)
            ns.append(n)
        self.mats, self.perms, self.ns = keep, perms, ns
        self.arr = _matrix_array([_addr(rp) for rp, _ in keep], [_addr(ci) for _, ci in keep], ns,
                                 [ci.shape[0] for _, ci in keep], [_addr(p) for p in perms])


def reorder_batch(mats: Sequence, *, reverse: bool = True, start: int | None = None, want_bandwidth: bool = True,
                  ctx: Context | None = None, raise_on_error: bool = True, perms_out: Sequence | None = None,
                  **opt_kw):
    """Reorders many (row_ptr, col_idx) host matrices in one persistent
    launch.  perms_out: optional uint32 host arrays (n entries each, e.g.
    pinned) that receive the permutations.  Returns (list of perms, list of
    result dicts)."""
    pb = mats if isinstance(mats, PreparedBatch) else PreparedBatch(mats, perms_out)
    if pb.device:
        raise ValueError("a device PreparedBatch goes to reorder_batch_device")
    res = (Result * pb.count)()
    o = default_options(reverse=reverse, start=start, want_bandwidth=want_bandwidth, **opt_kw)
    rc = _lib.lib().pbrcm_reorder_batch(_h(ctx), pb.arr, pb.count, ctypes.byref(o), res)
    if raise_on_error:
        _check(rc, "pbrcm_reorder_batch")
    return [p[:n] for p, n in zip(pb.perms, pb.ns)], BatchResults(res)


def reorder_batch_device(mats: Sequence, *, reverse: bool = True, ctx: Context | None = None, stream=None,
                         raise_on_error: bool = True, **opt_kw):
    """Batched reorder of device-resident (row_ptr, col_idx, perm_out) torch
    tensors.  Returns the results (a sequence of result dicts)."""
    import torch

    pb = mats if isinstance(mats, PreparedBatch) else PreparedBatch(mats, device=True)
    if not pb.device:
        raise ValueError("a host PreparedBatch goes to reorder_batch")
    res = (Result * pb.count)()
    o = default_options(reverse=reverse, **opt_kw)
    st = ctypes.c_void_p(stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream)
    rc = _lib.lib().pbrcm_reorder_batch_device(_h(ctx), pb.arr, pb.count, ctypes.byref(o), res, st)
    if raise_on_error:
        _check(rc, "pbrcm_reorder_batch_device")
    return BatchResults(res)


def autotune(mats: Sequence, *, ctx: Context, cache_path: str | None = None, reverse: bool = True,
             **opt_kw) -> dict:
    """Measures the batch and serving shapes on a calibration batch of
    (row_ptr, col_idx) host matrices (pbrcm_autotune): the chosen settings
    become ctx's and, with cache_path, are written there.  Returns them."""
    keep = []
    arr = (Matrix * len(mats))()
    for i, m in enumerate(mats):
        rp, ci = _u32(m[0]), _u32(m[1])
        keep += [rp, ci]
        arr[i].row_ptr = rp.ctypes.data
        arr[i].col_idx = ci.ctypes.data
        arr[i].n = rp.shape[0] - 1
        arr[i].nnz = ci.shape[0]
        arr[i].perm_out = None
    o = default_options(reverse=reverse, **opt_kw)
    t = Tuning()
    path = cache_path.encode() if cache_path else None
    _check(_lib.lib().pbrcm_autotune(ctx.handle, arr, len(mats), ctypes.byref(o), path, ctypes.byref(t)),
           "pbrcm_autotune")
    return t.as_dict()


def tuning_get(ctx: Context) -> dict:
    t = Tuning()
    _check(_lib.lib().pbrcm_tuning_get(ctx.handle, ctypes.byref(t)), "pbrcm_tuning_get")
    return t.as_dict()


def tuning_set(ctx: Context, **kw) -> None:
    """Sets some of the context's batch / serving settings (the others stay)."""
    t = Tuning()
    _check(_lib.lib().pbrcm_tuning_get(ctx.handle, ctypes.byref(t)), "pbrcm_tuning_get")
    for k, v in kw.items():
        setattr(t, k, v)
    _check(_lib.lib().pbrcm_tuning_set(ctx.handle, ctypes.byref(t)), "pbrcm_tuning_set")


def tuning_load(ctx: Context, path: str) -> None:
    _check(_lib.lib().pbrcm_tuning_load(ctx.handle, path.encode()), "pbrcm_tuning_load")


class Session:
    """Serving session: submit requests at any time; they are admitted by
    device memory footprint and run concurrently (continuous batching)."""

    def __init__(self, ctx: Context, memory_cap_bytes: int = 0, max_inflight: int = 0, streams: int = 0):
        cfg = SessionConfig()
        cfg.memory_cap_bytes = memory_cap_bytes
        cfg.max_inflight = max_inflight
        cfg.streams = streams
        h = ctypes.c_void_p()
        _check(_lib.lib().pbrcm_session_create(ctx.handle, ctypes.byref(cfg), ctypes.byref(h)),
               "pbrcm_session_create")
        self.handle = h
        self.ctx = ctx
        self._n = {}

    def submit(self, row_ptr, col_idx, *, reverse: bool = True, start: int | None = None,
               want_bandwidth: bool = True, **opt_kw) -> int:
        rp, ci = _u32(row_ptr), _u32(col_idx)
        t = ctypes.c_uint64()
        o = default_options(reverse=reverse, start=start, want_bandwidth=want_bandwidth, **opt_kw)
        _check(_lib.lib().pbrcm_session_submit(self.handle, _ptr(rp), _ptr(ci), rp.shape[0] - 1, ci.shape[0],
                                               ctypes.byref(o), ctypes.byref(t)), "pbrcm_session_submit")
        self._n[t.value] = np.empty(max(rp.shape[0] - 1, 1), dtype=np.uint32)
        return t.value

    def poll(self, ticket: int):
        """None while running; (perm, result dict) once done."""
        perm = self._n[ticket]
        res = Result()
        done = ctypes.c_int32()
        rc = _lib.lib().pbrcm_session_poll(self.handle, ticket, _ptr(perm), ctypes.byref(res), ctypes.byref(done))
        if rc != 0 and done.value == 0:
            _check(rc, "pbrcm_session_poll")
        if not done.value:
            return None
        del self._n[ticket]
        d = res.as_dict()
        d["rc"] = rc
        return perm, d

    def drain(self) -> None:
        _check(_lib.lib().pbrcm_session_drain(self.handle), "pbrcm_session_drain")

    def stats(self) -> dict:
        st = SessionStats()
        _check(_lib.lib().pbrcm_session_stats_get(self.handle, ctypes.byref(st)), "pbrcm_session_stats_get")
        return {name: getattr(st, name) for name, _ in st._fields_}

    def close(self) -> None:
        if self.handle:
            _lib.lib().pbrcm_session_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _take_csr(n: int, nnz: int, rp_p, ci_p):
    L = _lib.lib()
    rp = np.ctypeslib.as_array(rp_p, shape=(n + 1,)).copy()
    ci = np.ctypeslib.as_array(ci_p, shape=(max(nnz, 1),))[:nnz].copy()
    L.pbrcm_free(ctypes.cast(rp_p, ctypes.c_void_p))
    L.pbrcm_free(ctypes.cast(ci_p, ctypes.c_void_p))
    return rp, ci


def load_mtx(path: str):
    """(row_ptr, col_idx) of a MatrixMarket file with the reference loader's
    semantics (include/Graph.h:266-332), without writing cache files."""
    n, nnz = ctypes.c_uint32(), ctypes.c_uint64()
    rp_p, ci_p = ctypes.POINTER(ctypes.c_uint32)(), ctypes.POINTER(ctypes.c_uint32)()
    _check(_lib.lib().pbrcm_load_mtx(path.encode(), ctypes.byref(n), ctypes.byref(nnz), ctypes.byref(rp_p),
                                     ctypes.byref(ci_p)), f"pbrcm_load_mtx({path})")
    return _take_csr(n.value, nnz.value, rp_p, ci_p)


def _vals(vals):
    if vals is None:
        return None, 0
    v = np.ascontiguousarray(vals)
    if v.dtype.itemsize not in (4, 8):
        raise ValueError("values must have 4 or 8 bytes per entry")
    return v, v.dtype.itemsize


def permute(row_ptr, col_idx, perm, vals=None, *, want_map: bool = False, ctx: Context | None = None):
    """B = P A P^T (the reference's `-o` reordering, CuSolverRCM::reorder,
    include/device/rcm_cusolver.cuh:154-185): row i of B is row perm[i] of A
    with columns renamed to their positions and sorted.  Returns (row_ptr,
    col_idx, vals or None, map or None); map[k] = entry of A behind entry k."""
    rp, ci, pm = _u32(row_ptr), _u32(col_idx), _u32(perm)
    v, vb = _vals(vals)
    n, nnz = rp.shape[0] - 1, ci.shape[0]
    orp = np.empty(n + 1, np.uint32)
    oci = np.empty(max(nnz, 1), np.uint32)
    ov = np.empty(max(nnz, 1), v.dtype) if v is not None else None
    om = np.empty(max(nnz, 1), np.uint32) if want_map else None
    _check(_lib.lib().pbrcm_permute(_h(ctx), _ptr(rp), _ptr(ci), _ptr(v) if v is not None else None, vb, n, nnz,
                                    _ptr(pm), _ptr(orp), _ptr(oci), _ptr(ov) if ov is not None else None,
                                    _ptr(om) if om is not None else None), "pbrcm_permute")
    return orp, oci[:nnz], (ov[:nnz] if ov is not None else None), (om[:nnz] if om is not None else None)


def permute_device(row_ptr_t, col_idx_t, perm_t, vals_t=None, *, want_map: bool = False,
                   ctx: Context | None = None, stream=None):
    """permute() on device-resident torch tensors.  Returns (row_ptr, col_idx,
    vals or None, map or None) as tensors on the same device."""
    import torch

    n, nnz = row_ptr_t.numel() - 1, col_idx_t.numel()
    dev = row_ptr_t.device
    orp = torch.empty(n + 1, dtype=torch.int32, device=dev)
    oci = torch.empty(max(nnz, 1), dtype=torch.int32, device=dev)
    ov = torch.empty(max(nnz, 1), dtype=vals_t.dtype, device=dev) if vals_t is not None else None
    om = torch.empty(max(nnz, 1), dtype=torch.int32, device=dev) if want_map else None
    vb = vals_t.element_size() if vals_t is not None else 0
    st = stream.cuda_stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
    _check(_lib.lib().pbrcm_permute_device(
        _h(ctx), row_ptr_t.data_ptr(), col_idx_t.data_ptr(), vals_t.data_ptr() if vals_t is not None else None,
        vb, n, nnz, perm_t.data_ptr(), orp.data_ptr(), oci.data_ptr(), ov.data_ptr() if ov is not None else None,
        om.data_ptr() if om is not None else None, st), "pbrcm_permute_device")
    return orp, oci[:nnz], (ov[:nnz] if ov is not None else None), (om[:nnz] if om is not None else None)


def connect_device(row_ptr_t, col_idx_t, *, cap: int | None = None, ctx: Context | None = None, stream=None):
    """The loader's connectivity repair (Graph<T>::prepareRCM,
    include/Graph.h:160-263) on device-resident torch tensors of a symmetric
    pattern with sorted rows.  Returns (row_ptr, col_idx, links): the joined
    CSR on the same device and the number of links added.  The output is
    first given room for `cap` entries (default: nnz plus a small slack) and
    reallocated to the exact size if the matrix needs more."""
    import torch

    n, nnz = row_ptr_t.numel() - 1, col_idx_t.numel()
    dev = row_ptr_t.device
    orp = torch.empty(n + 1, dtype=torch.int32, device=dev)
    room = cap if cap is not None else nnz + 2 * min(max(n - 1, 0), max(1024, n // 64))
    st = stream.cuda_stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
    L = _lib.lib()
    for _ in range(2):
        oci = torch.empty(max(room, 1), dtype=torch.int32, device=dev)
        got, links = ctypes.c_uint64(0), ctypes.c_uint32(0)
        rc = L.pbrcm_connect_device(_h(ctx), row_ptr_t.data_ptr(), col_idx_t.data_ptr(), n, nnz, orp.data_ptr(),
                                    oci.data_ptr(), room, ctypes.byref(got), ctypes.byref(links), st)
        if rc == 1 and got.value > room:  # PBRCM_ERR_ARG with the size needed: too little room
            room = got.value
            continue
        _check(rc, "pbrcm_connect_device")
        return orp, oci[:got.value], links.value
    raise PbrcmError(1, "pbrcm_connect_device: output size changed between calls")


def load_hicsr(path: str):
    """(row_ptr, col_idx, values) of a reference `.hicsr` CSR cache
    (src/CSR.cpp:57-168); values float32 or float64 as stored."""
    L = _lib.lib()
    n, nnz, vb = ctypes.c_uint32(), ctypes.c_uint64(), ctypes.c_uint32()
    rp_p, ci_p = ctypes.POINTER(ctypes.c_uint32)(), ctypes.POINTER(ctypes.c_uint32)()
    v_p = ctypes.c_void_p()
    _check(L.pbrcm_load_hicsr(path.encode(), ctypes.byref(n), ctypes.byref(nnz), ctypes.byref(rp_p),
                              ctypes.byref(ci_p), ctypes.byref(v_p), ctypes.byref(vb)), f"pbrcm_load_hicsr({path})")
    dt = np.float64 if vb.value == 8 else np.float32
    buf = (ctypes.c_char * (vb.value * max(nnz.value, 1))).from_address(v_p.value)
    vals = np.frombuffer(buf, dtype=dt)[:nnz.value].copy()
    L.pbrcm_free(v_p)
    rp, ci = _take_csr(n.value, nnz.value, rp_p, ci_p)
    return rp, ci, vals


def store_hicsr(path: str, row_ptr, col_idx, vals=None):
    """Writes a `.hicsr` CSR cache the reference's loadCSR reads."""
    rp, ci = _u32(row_ptr), _u32(col_idx)
    v, vb = _vals(vals)
    _check(_lib.lib().pbrcm_store_hicsr(path.encode(), rp.shape[0] - 1, ci.shape[0], _ptr(rp), _ptr(ci),
                                        _ptr(v) if v is not None else None, vb), f"pbrcm_store_hicsr({path})")


def store_mtx(path: str, row_ptr, col_idx, vals=None):
    """Writes a MatrixMarket file in the reference's storeMTX format
    (src/COO.cpp:213-251); without values a `pattern` file."""
    rp, ci = _u32(row_ptr), _u32(col_idx)
    v, vb = _vals(vals)
    _check(_lib.lib().pbrcm_store_mtx(path.encode(), rp.shape[0] - 1, ci.shape[0], _ptr(rp), _ptr(ci),
                                      _ptr(v) if v is not None else None, vb), f"pbrcm_store_mtx({path})")


def prepare_csr(row_ptr, col_idx, check_symmetry: bool = True):
    """prepareRCM (include/Graph.h:74-264): symmetry repair + connectivity
    repair of a raw CSR."""
    rp, ci = _u32(row_ptr), _u32(col_idx)
    nnz = ctypes.c_uint64()
    rp_p, ci_p = ctypes.POINTER(ctypes.c_uint32)(), ctypes.POINTER(ctypes.c_uint32)()
    _check(_lib.lib().pbrcm_prepare_csr(_ptr(rp), _ptr(ci), rp.shape[0] - 1, ci.shape[0], int(check_symmetry),
                                        ctypes.byref(nnz), ctypes.byref(rp_p), ctypes.byref(ci_p)),
           "pbrcm_prepare_csr")
    return _take_csr(rp.shape[0] - 1, nnz.value, rp_p, ci_p)


# ---------------------------------------------------------------------------
# Reference-shaped surface
# ---------------------------------------------------------------------------

@dataclass
class _CSR:
    """Mirror of CSR<T> (include/CSR.h:43-75): rows, cols, nnz, row_offsets,
    col_ids, data."""
    row_offsets: np.ndarray
    col_ids: np.ndarray
    data: np.ndarray | None = None

    @property
    def rows(self) -> int:
        return int(self.row_offsets.shape[0] - 1)

    @property
    def cols(self) -> int:
        return self.rows

    @property
    def nnz(self) -> int:
        return int(self.col_ids.shape[0])


@dataclass
class Graph:
    """Mirror of Graph<T> (include/Graph.h:42-333)."""
    csr: _CSR = field(default_factory=lambda: _CSR(np.zeros(1, np.uint32), np.zeros(0, np.uint32)))

    @classmethod
    def from_csr(cls, row_offsets, col_ids) -> "Graph":
        return cls(_CSR(_u32(row_offsets), _u32(col_ids)))

    def load(self, file: str) -> int:
        """Graph::load (include/Graph.h:266-332): 0 on success, -1 if the file
        cannot be read (the reference prints the error and returns -1)."""
        try:
            rp, ci = load_mtx(file)
        except PbrcmError:
            return -1
        self.csr = _CSR(rp, ci)
        return 0

    @property
    def size(self) -> int:
        return self.csr.rows

    def neighbour_count(self, node: int) -> int:
        return int(self.csr.row_offsets[node + 1] - self.csr.row_offsets[node])

    def prepareRCM(self, check_sym: bool = True) -> None:
        rp, ci = prepare_csr(self.csr.row_offsets, self.csr.col_ids, check_sym)
        self.csr = _CSR(rp, ci)


class GPU_BATCH:
    """Mirror of namespace GPU_BATCH (include/rcm_gpu_batch.h:37-45)."""

    @staticmethod
    def rcm(graph: Graph, csv_file, permutation: list, start_node: int, ctx: Context | None = None) -> None:
        """GPU_BATCH::rcm (src/device/rcm_gpu_batch.cu:42-112): fills
        `permutation` with the Cuthill-McKee order from `start_node` (the
        reference's output order: not reversed) and appends the device time in
        ms to `csv_file` (any object with write(), or None)."""
        perm, res = reorder(graph.csr.row_offsets, graph.csr.col_ids, reverse=False, start=start_node,
                            want_bandwidth=False, ctx=ctx)
        permutation.clear()
        permutation.extend(int(x) for x in perm)
        if csv_file is not None:
            csv_file.write(f"{res['device_ms']}")

    @staticmethod
    def findPeripheral(graph: Graph, csv_file=None, writeOutput: bool = False, ctx: Context | None = None) -> int:
        return SimplePeripheral.findPeripheral(graph, csv_file, writeOutput, ctx=ctx)


class SimplePeripheral:
    """Mirror of namespace SimplePeripheral (include/simple_peripheral.h:40-47),
    computed on the GPU."""

    @staticmethod
    def findPeripheral(graph: Graph, csv_file=None, writeOutput: bool = False, outputnodes: int = 32,
                       ctx: Context | None = None) -> int:
        if outputnodes != 32:
            raise ValueError("the GPU search keeps 32 nodes per pass, as the reference default")
        s, _, _ = find_peripheral(graph.csr.row_offsets, graph.csr.col_ids, ctx=ctx)
        return s


def compute_bandwidth(graph: Graph, permutation: Iterable[int]) -> int:
    """computeBandwidth (src/main.cpp:143-184); -1 for an empty permutation."""
    perm = _u32(list(permutation) if not isinstance(permutation, np.ndarray) else permutation)
    if perm.shape[0] == 0:
        return -1
    bw, _, _ = bandwidth(graph.csr.row_offsets, graph.csr.col_ids, perm)
    return int(bw)


def check_bandwidth(graph: Graph) -> int:
    """checkBandwidth (src/main.cpp:114-129): bandwidth of the input as
    stored."""
    n = graph.csr.rows
    _, bw0, _ = bandwidth(graph.csr.row_offsets, graph.csr.col_ids, np.arange(n, dtype=np.uint32))
    return int(bw0)


def max_valency(graph: Graph) -> int:
    """maxValency (src/main.cpp:131-140)."""
    return int(np.max(np.diff(graph.csr.row_offsets.astype(np.int64)))) if graph.csr.rows else 0


def check_permutation(permutation) -> int:
    """checkPermutation (src/main.cpp:186-226): 0 if a bijection, -1 if not."""
    p = np.asarray(permutation, dtype=np.int64)
    n = p.shape[0]
    if n == 0:
        return 0
    if p.min() < 0 or p.max() >= n:
        return -1
    return 0 if np.unique(p).shape[0] == n else -1
