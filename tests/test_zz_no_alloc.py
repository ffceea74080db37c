"""pbrcm_reorder_device_noalloc -- the entry point that allocates nothing.

It serves callers that cannot call cudaMalloc while they run (a host
application whose device memory belongs to its own pool or to a budget fixed
at start-up, or code that must not let an allocation synchronise the device
mid-flight): all of its scratch lives in a static device array reserved when
the library loads.  These tests call it through the C ABI (ctypes) and check
that its permutation and result equal those of pbrcm_reorder_device, the
allocating entry point, bit for bit, on consecutive calls that share the
array; and that inputs beyond its stated limits are refused.  This file is
collected last so that a failure here leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _noalloc(L, rp_t, ci_t, perm_t, reverse, stream_ptr):
    from parallelbatchrcm_b200._lib import Result
    import parallelbatchrcm_b200 as P
    o = P.default_options(reverse=reverse)
    res = Result()
    rc = L.pbrcm_reorder_device_noalloc(ctypes.c_void_p(rp_t.data_ptr()), ctypes.c_void_p(ci_t.data_ptr()),
                                        rp_t.numel() - 1, ci_t.numel(), ctypes.byref(o),
                                        ctypes.c_void_p(perm_t.data_ptr()), ctypes.byref(res),
                                        ctypes.c_void_p(stream_ptr))
    return rc, res.as_dict()


def _device(m):
    import torch
    rp = torch.from_numpy(np.ascontiguousarray(m[0]).astype(np.int32)).cuda()
    ci = torch.from_numpy(np.ascontiguousarray(m[1]).astype(np.int32)).cuda()
    return rp, ci


def test_noalloc_equals_allocating_entry_point(pbrcm, gpu_ctx):
    import torch
    from parallelbatchrcm_b200 import _lib, gen
    L = _lib.lib()
    g = load_golden("grid2d_64x64_s1")
    m3 = gen.grid3d(40, 40, 40, seed=21)
    mats = [(g["row_ptr"], g["col_idx"]), (m3.row_ptr, m3.col_idx), (g["row_ptr"], g["col_idx"])]
    stream = torch.cuda.current_stream().cuda_stream
    for rp_h, ci_h in mats:  # consecutive calls share the static scratch
        rp, ci = _device((rp_h, ci_h))
        n = rp.numel() - 1
        for reverse in (True, False):
            want, ref = pbrcm.reorder_device(rp, ci, reverse=reverse, ctx=gpu_ctx)
            got = torch.full((n,), -1, dtype=torch.int32, device="cuda")
            rc, res = _noalloc(L, rp, ci, got, reverse, stream)
            assert rc == 0 and res["status"] == 0
            assert torch.equal(got, want)
            # small matrices on the shared-memory engine (no scratch), the rest on the team
            assert res["engine"] == (2 if n <= 4096 else 0) == ref["engine"]
            for k in ("start_node", "peripheral_passes", "eccentricity", "levels", "placed", "bandwidth",
                      "initial_bandwidth", "profile"):
                assert res[k] == ref[k], k
    # and against the reference's own output (golden, CM order)
    rp, ci = _device((g["row_ptr"], g["col_idx"]))
    got = torch.empty(rp.numel() - 1, dtype=torch.int32, device="cuda")
    rc, res = _noalloc(L, rp, ci, got, False, stream)
    assert rc == 0 and np.array_equal(got.cpu().numpy().astype(np.uint32), g["perm"])


def test_noalloc_at_its_node_limit(pbrcm, gpu_ctx):
    """n = 2^20 exactly (a 1024 x 1024 grid): the node table and the queue
    records fill the static scratch; same permutation and result as the
    allocating entry point."""
    import torch
    from parallelbatchrcm_b200 import _lib, gen
    L = _lib.lib()
    m = gen.grid2d(1024, 1024, seed=29)
    assert m.n == 1 << 20
    rp, ci = _device((m.row_ptr, m.col_idx))
    stream = torch.cuda.current_stream().cuda_stream
    want, ref = pbrcm.reorder_device(rp, ci, reverse=True, ctx=gpu_ctx)
    got = torch.full((m.n,), -1, dtype=torch.int32, device="cuda")
    rc, res = _noalloc(L, rp, ci, got, True, stream)
    assert rc == 0 and res["status"] == 0
    assert torch.equal(got, want)
    for k in ("start_node", "peripheral_passes", "eccentricity", "levels", "placed", "bandwidth", "profile"):
        assert res[k] == ref[k], k
    assert res["device_ms"] > 0


def test_noalloc_refuses_inputs_beyond_its_limits(pbrcm, gpu_ctx):
    import torch
    from parallelbatchrcm_b200 import _lib
    L = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    # more nodes than the static scratch holds: refused before any device work
    rp = torch.zeros(4, dtype=torch.int32, device="cuda")
    ci = torch.zeros(4, dtype=torch.int32, device="cuda")
    perm = torch.zeros(4, dtype=torch.int32, device="cuda")
    from parallelbatchrcm_b200._lib import Result
    import parallelbatchrcm_b200 as P
    o = P.default_options()
    res = Result()
    rc = L.pbrcm_reorder_device_noalloc(ctypes.c_void_p(rp.data_ptr()), ctypes.c_void_p(ci.data_ptr()),
                                        (1 << 20) + 1, 4, ctypes.byref(o), ctypes.c_void_p(perm.data_ptr()),
                                        ctypes.byref(res), ctypes.c_void_p(stream))
    assert rc == 1  # PBRCM_ERR_ARG
    # a row longer than 1024 entries
    g = load_golden("star_3000")
    rp, ci = _device((g["row_ptr"], g["col_idx"]))
    perm = torch.empty(rp.numel() - 1, dtype=torch.int32, device="cuda")
    rc, res = _noalloc(L, rp, ci, perm, True, stream)
    assert rc == 1
    # the entry point still works afterwards
    g = load_golden("rgg_3000_s11")
    rp, ci = _device((g["row_ptr"], g["col_idx"]))
    perm = torch.empty(rp.numel() - 1, dtype=torch.int32, device="cuda")
    rc, res = _noalloc(L, rp, ci, perm, False, stream)
    assert rc == 0 and np.array_equal(perm.cpu().numpy().astype(np.uint32), g["perm"])
