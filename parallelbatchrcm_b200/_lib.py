"""ctypes binding of libpbrcm.so (include/pbrcm.h).

The library is built in-tree by ``parallelbatchrcm_b200.build`` (nvcc,
sm_100a).  There is no fallback: if the shared library is missing, importing
this module raises.  ``PBRCM_LIB`` selects another build (for example the
bounds-checked ``libpbrcm_checks.so``).
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_LIB = os.path.join(HERE, "libpbrcm.so")
CHECKS_LIB = os.path.join(HERE, "libpbrcm_checks.so")

AUTO_START = 0xFFFFFFFF
DEBUG_PHANTOM_CTA = 0x1

STATUS = {
    0: "PBRCM_OK", 1: "PBRCM_ERR_ARG", 2: "PBRCM_ERR_DISCONNECTED", 3: "PBRCM_ERR_TIMEOUT",
    4: "PBRCM_ERR_OOM", 5: "PBRCM_ERR_CUDA", 6: "PBRCM_ERR_IO", 7: "PBRCM_ERR_FORMAT",
    8: "PBRCM_ERR_CHECK", 9: "PBRCM_ERR_BUSY", 10: "PBRCM_ERR_NOT_FOUND",
}


class Options(ctypes.Structure):
    _fields_ = [
        ("reverse", ctypes.c_uint32), ("start_node", ctypes.c_uint32), ("stable", ctypes.c_uint32),
        ("want_bandwidth", ctypes.c_uint32), ("peripheral_nodes", ctypes.c_uint32),
        ("wait_limit_ms", ctypes.c_uint32), ("debug_flags", ctypes.c_uint32), ("reserved", ctypes.c_uint32),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int32), ("start_node", ctypes.c_uint32), ("peripheral_passes", ctypes.c_uint32),
        ("eccentricity", ctypes.c_uint32), ("levels", ctypes.c_uint32), ("placed", ctypes.c_uint32),
        ("bandwidth", ctypes.c_int64), ("initial_bandwidth", ctypes.c_int64), ("profile", ctypes.c_uint64),
        ("device_ms", ctypes.c_float), ("total_ms", ctypes.c_float), ("engine", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class Matrix(ctypes.Structure):
    _fields_ = [
        ("row_ptr", ctypes.c_void_p), ("col_idx", ctypes.c_void_p), ("n", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32), ("nnz", ctypes.c_uint64), ("perm_out", ctypes.c_void_p),
    ]


class SessionConfig(ctypes.Structure):
    _fields_ = [
        ("memory_cap_bytes", ctypes.c_uint64), ("max_inflight", ctypes.c_uint32), ("streams", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32 * 4),
    ]


class SessionStats(ctypes.Structure):
    _fields_ = [
        ("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("bytes_in_flight", ctypes.c_uint64),
        ("peak_bytes_in_flight", ctypes.c_uint64), ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
        ("max_ms", ctypes.c_double), ("busy_s", ctypes.c_double),
    ]


class Tuning(ctypes.Structure):
    _fields_ = [
        ("batch_pool", ctypes.c_uint32), ("batch_kernel", ctypes.c_uint32),
        ("cluster_size", ctypes.c_uint32), ("cluster_max", ctypes.c_uint32),
        ("cluster_nnz", ctypes.c_uint32), ("session_cutoff_n", ctypes.c_uint32), ("session_pool", ctypes.c_uint32),
        ("session_team_nnz", ctypes.c_uint32), ("session_cluster_max", ctypes.c_uint32),
        ("sms", ctypes.c_uint32),
        ("trials", ctypes.c_uint32), ("source", ctypes.c_uint32), ("default_ms", ctypes.c_float),
        ("best_ms", ctypes.c_float), ("session_default_ms", ctypes.c_float), ("session_best_ms", ctypes.c_float),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


# every symbol include/pbrcm.h declares, with (restype, argtypes)
_vp = ctypes.c_void_p
_u32 = ctypes.c_uint32
_u64 = ctypes.c_uint64
_i32 = ctypes.c_int32
_pu32 = ctypes.POINTER(ctypes.c_uint32)
SIGNATURES = {
    "pbrcm_default_options": (None, [ctypes.POINTER(Options)]),
    "pbrcm_version": (ctypes.c_char_p, []),
    "pbrcm_status_string": (ctypes.c_char_p, [_i32]),
    "pbrcm_context_create": (_i32, [_i32, ctypes.POINTER(_vp)]),
    "pbrcm_context_destroy": (None, [_vp]),
    "pbrcm_reorder": (_i32, [_vp, _vp, _vp, _u32, _u64, ctypes.POINTER(Options), _vp, ctypes.POINTER(Result)]),
    "pbrcm_reorder_device": (_i32, [_vp, _vp, _vp, _u32, _u64, ctypes.POINTER(Options), _vp,
                                    ctypes.POINTER(Result), _vp]),
    "pbrcm_reorder_device_noalloc": (_i32, [_vp, _vp, _u32, _u64, ctypes.POINTER(Options), _vp,
                                            ctypes.POINTER(Result), _vp]),
    "pbrcm_find_peripheral": (_i32, [_vp, _vp, _vp, _u32, _u64, _pu32, _pu32, _pu32]),
    "pbrcm_bandwidth": (_i32, [_vp, _vp, _vp, _u32, _u64, _vp, ctypes.POINTER(ctypes.c_int64),
                               ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_uint64)]),
    "pbrcm_reorder_batch": (_i32, [_vp, ctypes.POINTER(Matrix), _u32, ctypes.POINTER(Options),
                                   ctypes.POINTER(Result)]),
    "pbrcm_reorder_batch_device": (_i32, [_vp, ctypes.POINTER(Matrix), _u32, ctypes.POINTER(Options),
                                          ctypes.POINTER(Result), _vp]),
    "pbrcm_session_create": (_i32, [_vp, ctypes.POINTER(SessionConfig), ctypes.POINTER(_vp)]),
    "pbrcm_session_destroy": (None, [_vp]),
    "pbrcm_session_submit": (_i32, [_vp, _vp, _vp, _u32, _u64, ctypes.POINTER(Options),
                                    ctypes.POINTER(ctypes.c_uint64)]),
    "pbrcm_session_poll": (_i32, [_vp, _u64, _vp, ctypes.POINTER(Result), ctypes.POINTER(_i32)]),
    "pbrcm_session_drain": (_i32, [_vp]),
    "pbrcm_session_stats_get": (_i32, [_vp, ctypes.POINTER(SessionStats)]),
    "pbrcm_load_mtx": (_i32, [ctypes.c_char_p, _pu32, ctypes.POINTER(ctypes.c_uint64),
                              ctypes.POINTER(_pu32), ctypes.POINTER(_pu32)]),
    "pbrcm_prepare_csr": (_i32, [_vp, _vp, _u32, _u64, _i32, ctypes.POINTER(ctypes.c_uint64),
                                 ctypes.POINTER(_pu32), ctypes.POINTER(_pu32)]),
    "pbrcm_free": (None, [_vp]),
    "pbrcm_permute": (_i32, [_vp, _vp, _vp, _vp, _u32, _u32, _u64, _vp, _vp, _vp, _vp, _vp]),
    "pbrcm_permute_device": (_i32, [_vp, _vp, _vp, _vp, _u32, _u32, _u64, _vp, _vp, _vp, _vp, _vp, _vp]),
    "pbrcm_connect_device": (_i32, [_vp, _vp, _vp, _u32, _u64, _vp, _vp, _u64, ctypes.POINTER(ctypes.c_uint64),
                                    _pu32, _vp]),
    "pbrcm_store_mtx": (_i32, [ctypes.c_char_p, _u32, _u64, _vp, _vp, _vp, _u32]),
    "pbrcm_load_hicsr": (_i32, [ctypes.c_char_p, _pu32, ctypes.POINTER(ctypes.c_uint64),
                                ctypes.POINTER(ctypes.POINTER(ctypes.c_uint32)),
                                ctypes.POINTER(ctypes.POINTER(ctypes.c_uint32)), ctypes.POINTER(_vp), _pu32]),
    "pbrcm_store_hicsr": (_i32, [ctypes.c_char_p, _u32, _u64, _vp, _vp, _vp, _u32]),
    "pbrcm_autotune": (_i32, [_vp, ctypes.POINTER(Matrix), _u32, ctypes.POINTER(Options), ctypes.c_char_p,
                              ctypes.POINTER(Tuning)]),
    "pbrcm_tuning_get": (_i32, [_vp, ctypes.POINTER(Tuning)]),
    "pbrcm_tuning_set": (_i32, [_vp, ctypes.POINTER(Tuning)]),
    "pbrcm_tuning_load": (_i32, [_vp, ctypes.c_char_p]),
}

_lib = None


def lib_path() -> str:
    return os.environ.get("PBRCM_LIB", DEFAULT_LIB)


def lib():
    """The loaded libpbrcm.so.  Raises if it has not been built."""
    global _lib
    if _lib is None:
        path = lib_path()
        if not os.path.exists(path):
            raise ImportError(
                f"libpbrcm not built ({path} missing): run "
                "`python -c 'import parallelbatchrcm_b200.build as b; b.build()'` (needs nvcc)")
        L = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib
