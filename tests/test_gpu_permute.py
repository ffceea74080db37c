"""P A P^T on the GPU (pbrcm_permute / pbrcm_permute_device) against the
oracle, and the oracle against the reference's own call: cuSOLVER's
cusolverSpXcsrpermHost with p = q = perm, as CuSolverRCM::reorder makes it
(include/device/rcm_cusolver.cuh:154-185).  Integer work: exact."""
import ctypes
import ctypes.util
import glob
import os

import numpy as np
import pytest

from conftest import golden_names, load_golden

pytestmark = pytest.mark.gpu


def _cases():
    from parallelbatchrcm_b200 import gen
    out = [(n, load_golden(n)["row_ptr"], load_golden(n)["col_idx"], load_golden(n)["perm"]) for n in golden_names()]
    m = gen.grid3d(30, 20, 10, seed=3)
    out.append(("grid3d_30x20x10_random_perm", m.row_ptr, m.col_idx,
                np.random.default_rng(3).permutation(m.n).astype(np.uint32)))
    return out


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_permute_matches_oracle(pbrcm, gpu_ctx, oracle_mod, case):
    """Golden matrices with their RCM permutation (star_3000's center row has
    3,000 entries: the long-row path), values of both widths, the map."""
    _, rp, ci, perm = case
    rng = np.random.default_rng(1)
    for dtype in (np.float64, np.float32):
        vals = rng.standard_normal(ci.shape[0]).astype(dtype)
        orp, oci, ov, om = pbrcm.permute(rp, ci, perm, vals, want_map=True, ctx=gpu_ctx)
        erp, eci, ev, em = oracle_mod.permute_csr(rp, ci, perm, vals)
        assert np.array_equal(orp, erp) and np.array_equal(oci, eci)
        assert np.array_equal(om, em) and np.array_equal(ov, ev)
    orp, oci, ov, om = pbrcm.permute(rp, ci, perm, ctx=gpu_ctx)
    assert ov is None and om is None and np.array_equal(oci, eci)


def test_permute_device_large(pbrcm, gpu_ctx, oracle_mod):
    """The 128^3 grid with its RCM order, through the device entry point."""
    import torch
    from parallelbatchrcm_b200 import gen
    m = gen.grid3d(128, 128, 128, seed=12345)
    rp = torch.from_numpy(m.row_ptr.view(np.int32)).cuda()
    ci = torch.from_numpy(m.col_idx.view(np.int32)).cuda()
    perm_t, res = pbrcm.reorder_device(rp, ci, reverse=True, ctx=gpu_ctx)
    vals = torch.arange(m.nnz, dtype=torch.float64, device="cuda")
    orp, oci, ov, om = pbrcm.permute_device(rp, ci, perm_t, vals, want_map=True, ctx=gpu_ctx)
    perm = perm_t.cpu().numpy().view(np.uint32)
    erp, eci, _, em = oracle_mod.permute_csr(m.row_ptr, m.col_idx, perm)
    assert np.array_equal(orp.cpu().numpy().view(np.uint32), erp)
    assert np.array_equal(oci.cpu().numpy().view(np.uint32), eci)
    assert np.array_equal(om.cpu().numpy().view(np.uint32), em)
    assert np.array_equal(ov.cpu().numpy(), em.astype(np.float64))
    # the reordered matrix has the bandwidth the reorder reported
    b = np.repeat(np.arange(m.n), np.diff(erp.astype(np.int64)))
    assert int(np.abs(b - eci.astype(np.int64)).max()) == res["bandwidth"]


def test_permute_rejects_a_non_permutation(pbrcm, gpu_ctx):
    g = load_golden("grid2d_8x8_s3")
    bad = g["perm"].copy()
    bad[3] = bad[4]
    with pytest.raises(pbrcm.PbrcmError) as e:
        pbrcm.permute(g["row_ptr"], g["col_idx"], bad, ctx=gpu_ctx)
    assert e.value.name == "PBRCM_ERR_ARG"
    # and the context stays usable
    orp, oci, _, _ = pbrcm.permute(g["row_ptr"], g["col_idx"], g["perm"], ctx=gpu_ctx)
    assert orp[-1] == g["col_idx"].shape[0]


def _cusolver():
    names = [ctypes.util.find_library("cusolver"), ctypes.util.find_library("cusparse")]
    paths = []
    for base, pat in (("cusolver", "libcusolver.so*"), ("cusparse", "libcusparse.so*")):
        hits = sorted(glob.glob(os.path.join("/usr/local/cuda/lib64", pat)))
        paths.append(hits[0] if hits else None)
    try:
        sol = ctypes.CDLL(names[0] or paths[0])
        sp = ctypes.CDLL(names[1] or paths[1])
    except (OSError, TypeError):
        return None
    return sol, sp


def test_oracle_matches_cusolver_csrperm(oracle_mod):
    """Pins the oracle's P A P^T (sorted columns, map) on the reference's own
    library call, run here as the reference runs it."""
    libs = _cusolver()
    if libs is None:
        pytest.skip("cuSOLVER not found")
    sol, sp = libs
    handle, descr = ctypes.c_void_p(), ctypes.c_void_p()
    assert sol.cusolverSpCreate(ctypes.byref(handle)) == 0
    assert sp.cusparseCreateMatDescr(ctypes.byref(descr)) == 0
    try:
        assert sp.cusparseSetMatType(descr, 0) == 0        # CUSPARSE_MATRIX_TYPE_GENERAL
        assert sp.cusparseSetMatIndexBase(descr, 0) == 0   # CUSPARSE_INDEX_BASE_ZERO
        for name in ["grid2d_17x5_natural", "rgg_3000_s11", "caterpillar_40x60", "mtx_integer_sym"]:
            g = load_golden(name)
            rp, ci, perm = g["row_ptr"], g["col_idx"], g["perm"]
            n, nnz = rp.shape[0] - 1, ci.shape[0]
            A_rp = rp.astype(np.int32).copy()
            A_ci = ci.astype(np.int32).copy()
            p = perm.astype(np.int32).copy()
            mp = np.arange(nnz, dtype=np.int32)
            size = ctypes.c_size_t()
            i32p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
            assert sol.cusolverSpXcsrperm_bufferSizeHost(handle, n, n, nnz, descr, i32p(A_rp), i32p(A_ci), i32p(p),
                                                         i32p(p), ctypes.byref(size)) == 0
            buf = ctypes.create_string_buffer(max(size.value, 1))
            assert sol.cusolverSpXcsrpermHost(handle, n, n, nnz, descr, i32p(A_rp), i32p(A_ci), i32p(p), i32p(p),
                                              i32p(mp), buf) == 0
            erp, eci, _, em = oracle_mod.permute_csr(rp, ci, perm)
            assert np.array_equal(A_rp.astype(np.uint32), erp), name
            assert np.array_equal(A_ci.astype(np.uint32), eci), name
            assert np.array_equal(mp.astype(np.uint32), em), name
    finally:
        sp.cusparseDestroyMatDescr(descr)
        sol.cusolverSpDestroy(handle)


def test_permute_long_row_on_a_fresh_context(pbrcm, oracle_mod):
    """A row of 3,000 entries on a context that has no scratch yet: the
    long-row pass runs after the scratch is allocated."""
    g = load_golden("star_3000")
    ctx = pbrcm.Context(0)
    try:
        vals = np.arange(g["col_idx"].shape[0], dtype=np.float32)
        for _ in range(2):
            orp, oci, ov, om = pbrcm.permute(g["row_ptr"], g["col_idx"], g["perm"], vals, want_map=True, ctx=ctx)
            erp, eci, ev, em = oracle_mod.permute_csr(g["row_ptr"], g["col_idx"], g["perm"], vals)
            assert np.array_equal(orp, erp) and np.array_equal(oci, eci) and np.array_equal(om, em)
            assert np.array_equal(ov, ev)
    finally:
        ctx.close()
