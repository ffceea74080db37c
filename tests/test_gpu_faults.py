"""Failure paths on the GPU without faulting it: every device wait is bounded
and reports a status; bad inputs are rejected before the engine runs."""
import os
import subprocess
import sys
import time

import numpy as np
import pytest

from conftest import ROOT, load_golden

pytestmark = pytest.mark.gpu


def test_phantom_cta_times_out_and_context_survives(pbrcm, gpu_ctx):
    """A grid barrier that waits for one CTA more than were launched (nothing
    ever arrives) must give up after the wait limit with PBRCM_ERR_TIMEOUT;
    the next call on the same context must work."""
    g = load_golden("grid2d_64x64_s1")
    t0 = time.time()
    perm, res = pbrcm.reorder(g["row_ptr"], g["col_idx"], ctx=gpu_ctx, wait_limit_ms=200,
                              debug_flags=pbrcm.DEBUG_PHANTOM_CTA, raise_on_error=False)
    assert res["rc"] == 3 and res["status"] == 3
    assert time.time() - t0 < 20
    perm, res = pbrcm.reorder(g["row_ptr"], g["col_idx"], reverse=False, ctx=gpu_ctx)
    assert np.array_equal(perm, g["perm"])


def test_disconnected_graph_is_an_error(pbrcm, gpu_ctx):
    from parallelbatchrcm_b200 import gen
    a = gen.grid2d(10, 10, seed=1)
    b = gen.grid2d(7, 3, seed=2)
    n = a.n + b.n
    rp = np.concatenate([a.row_ptr, b.row_ptr[1:] + a.nnz]).astype(np.uint32)
    ci = np.concatenate([a.col_idx, b.col_idx + a.n]).astype(np.uint32)
    assert rp.shape[0] == n + 1
    for start in (None, 3, a.n + 2):
        with pytest.raises(pbrcm.PbrcmError) as e:
            pbrcm.reorder(rp, ci, start=start, ctx=gpu_ctx)
        assert e.value.name == "PBRCM_ERR_DISCONNECTED"
    # the loader's connectivity repair makes it valid
    rp2, ci2 = pbrcm.prepare_csr(rp, ci, False)
    perm, res = pbrcm.reorder(rp2, ci2, ctx=gpu_ctx)
    assert res["status"] == 0 and pbrcm.check_permutation(perm) == 0


@pytest.mark.parametrize("kind", ["col_out_of_range", "row_ptr_decreasing", "row_ptr_end", "start_out_of_range"])
def test_invalid_csr_rejected(pbrcm, gpu_ctx, kind):
    g = load_golden("grid2d_8x8_s3")
    rp, ci = g["row_ptr"].copy(), g["col_idx"].copy()
    start = None
    if kind == "col_out_of_range":
        ci[5] = 64
    elif kind == "row_ptr_decreasing":
        rp[10], rp[11] = rp[11], rp[10]
    elif kind == "row_ptr_end":
        rp[-1] += 1  # claims one entry more than col_idx holds
    elif kind == "start_out_of_range":
        start = 64
    with pytest.raises(pbrcm.PbrcmError) as e:
        pbrcm.reorder(rp, ci, start=start, ctx=gpu_ctx)
    assert e.value.name == "PBRCM_ERR_ARG"
    # context still fine
    perm, res = pbrcm.reorder(g["row_ptr"], g["col_idx"], reverse=False, ctx=gpu_ctx)
    assert np.array_equal(perm, g["perm"])


def test_bounds_checked_build_agrees(pbrcm):
    """Runs the golden cases on libpbrcm_checks.so (every device index
    range-checked; a failed check reports PBRCM_ERR_CHECK instead of touching
    memory) in a fresh process and expects identical results."""
    from parallelbatchrcm_b200 import _lib
    if not os.path.exists(_lib.CHECKS_LIB):
        pytest.skip("checks build not present")
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r); sys.path.insert(0, %r)\n"
        "from conftest import golden_names, load_golden\n"
        "import parallelbatchrcm_b200 as P\n"
        "ctx = P.Context(0)\n"
        "for name in golden_names():\n"
        "    g = load_golden(name)\n"
        "    perm, res = P.reorder(g['row_ptr'], g['col_idx'], reverse=False, ctx=ctx)\n"
        "    assert res['status'] == 0, (name, res)\n"
        "    assert np.array_equal(perm, g['perm']), name\n"
        "    assert res['bandwidth'] == int(g['bandwidth']), name\n"
        "mats = [(load_golden(n)['row_ptr'], load_golden(n)['col_idx']) for n in golden_names()]\n"
        "perms, rs = P.reorder_batch(mats, reverse=False, ctx=ctx)\n"
        "for n, p, r in zip(golden_names(), perms, rs):\n"
        "    assert r['status'] == 0 and np.array_equal(p, load_golden(n)['perm']), n\n"
        "import os\n"
        "os.environ.update(PBRCM_BATCH_CLUSTER='4', PBRCM_BATCH_CLUSTER_NNZ='1',\n"
        "                  PBRCM_CLUSTER_SOLO_PARENTS='8', PBRCM_CLUSTER_SOLO_EDGES='32')\n"
        "ctx2 = P.Context(0)\n"
        "perms, rs = P.reorder_batch(mats, reverse=False, ctx=ctx2)\n"
        "for n, p, r in zip(golden_names(), perms, rs):\n"
        "    assert r['status'] == 0 and np.array_equal(p, load_golden(n)['perm']), ('cluster', n)\n"
        "print('CHECKS_OK')\n"
    ) % (ROOT, os.path.join(ROOT, "tests"))
    env = dict(os.environ, PBRCM_LIB=_lib.CHECKS_LIB)
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert "CHECKS_OK" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]
