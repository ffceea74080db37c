"""Parity at the stated configurations, through the C ABI, against the oracle.

* the many-matrix batch: a seeded subset of the 4,096-matrix mixed stream
  (n log-uniform in [500, 200,000], seed 42) that spans the whole n range --
  every 16th matrix by size plus the 16 largest, which the batch gives to
  thread-block-cluster teams -- on device buffers and from host buffers
  (the copy-overlapped path); every permutation, start node and bandwidth
  is checked against the oracle;
* the serving stream: requests of the Poisson generator (n log-uniform in
  [1,000, 2,000,000], seed 99), including one of 1-2M nodes, submitted on
  their arrival times to a session; every result against the oracle;
* admission: a request larger than the memory cap is refused with
  PBRCM_ERR_BUSY, and a cap below two requests keeps the device bytes in
  flight under it while both complete.
Integer work: every comparison is exact."""
import multiprocessing as mp
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PBRCM_ERR_BUSY = 9


def _make(spec):
    from parallelbatchrcm_b200 import gen
    m = gen.make_from_spec(spec)
    return m.row_ptr, m.col_idx


def _oracle_reorder(args):
    import oracle as O
    rp, ci = args
    r = O.full_reorder(rp, ci, reverse=True)
    return r["perm"], r["start"], r["bandwidth"]


def _pool_map(fn, items):
    ctx = mp.get_context("spawn")
    with ctx.Pool(min(16, max(1, len(items)))) as pool:
        return pool.map(fn, items, chunksize=1)


@pytest.fixture(scope="module")
def c4_subset():
    from parallelbatchrcm_b200 import gen
    specs = gen.mixed_batch_specs(count=4096, seed=42)
    by_size = sorted(range(len(specs)), key=lambda i: gen.spec_nnz_estimate(specs[i]))
    pick = sorted(set(by_size[::16]) | set(by_size[-16:]))
    mats = _pool_map(_make, [specs[i] for i in pick])
    refs = _pool_map(_oracle_reorder, mats)
    return mats, refs


def _check(mats, refs, perms, results):
    for k, ((rp, ci), (rperm, rstart, rbw), p, r) in enumerate(zip(mats, refs, perms, results)):
        assert r["status"] == 0, (k, r)
        assert r["start_node"] == rstart, k
        assert np.array_equal(np.asarray(p).view(np.uint32), rperm), k
        assert r["bandwidth"] == rbw, k


def test_mixed_batch_subset_device(pbrcm, gpu_ctx, c4_subset):
    import torch
    mats, refs = c4_subset
    assert len(mats) >= 256 and max(rp.shape[0] - 1 for rp, _ in mats) > 150_000
    dev = torch.device("cuda", 0)
    dm = [(torch.from_numpy(rp.view(np.int32)).to(dev), torch.from_numpy(ci.view(np.int32)).to(dev),
           torch.empty(rp.shape[0] - 1, dtype=torch.int32, device=dev)) for rp, ci in mats]
    results = pbrcm.reorder_batch_device(dm, reverse=True, ctx=gpu_ctx)
    _check(mats, refs, [p.cpu().numpy() for _, _, p in dm], results)
    # per-matrix latency inside the batch: positive, at most the launch
    assert all(0 < r["device_ms"] < 60_000 for r in results)


def test_mixed_batch_subset_host_overlapped(pbrcm, gpu_ctx, c4_subset):
    """Host buffers: the CSRs are copied in waves while the kernel runs."""
    import torch
    mats, refs = c4_subset
    pinned = [(torch.from_numpy(rp.view(np.int32)).pin_memory().numpy().view(np.uint32),
               torch.from_numpy(ci.view(np.int32)).pin_memory().numpy().view(np.uint32)) for rp, ci in mats]
    for src in (pinned, mats):  # pinned and pageable host memory
        perms, results = pbrcm.reorder_batch(src, reverse=True, ctx=gpu_ctx)
        _check(mats, refs, perms, results)


def test_mixed_batch_pool_shapes_identical(pbrcm, c4_subset, monkeypatch):
    """Every pool shape (groups per CTA), with the general batch kernel and
    with the solo batch kernel, gives the oracle's permutations."""
    mats, refs = c4_subset
    small = mats[::4]
    shapes = [(p, k) for p in (0, 1, 2, 3, 5, 6, 7) for k in ("0", "1")]
    for pool, solo_kernel in shapes:
        monkeypatch.setenv("PBRCM_BATCH_POOL", str(pool))
        monkeypatch.setenv("PBRCM_BATCH_SOLO_KERNEL", solo_kernel)
        ctx = pbrcm.Context(0)
        try:
            perms, results = pbrcm.reorder_batch(small, reverse=True, ctx=ctx)
            _check(small, refs[::4], perms, results)
        finally:
            ctx.close()


def test_batch_graph_replay_between_other_batches(pbrcm, c4_subset):
    """A captured batch (device buffers; pinned host buffers) replayed after
    other batches of the same context have rewritten its staging: every
    replay gives the oracle's permutations."""
    import torch
    mats, refs = c4_subset
    a, ra = mats[:48], refs[:48]
    b = mats[48:96]
    dev = torch.device("cuda", 0)
    ctx = pbrcm.Context(0)
    try:
        dm = [(torch.from_numpy(rp.view(np.int32)).to(dev), torch.from_numpy(ci.view(np.int32)).to(dev),
               torch.empty(rp.shape[0] - 1, dtype=torch.int32, device=dev)) for rp, ci in a]
        pinned = [(torch.from_numpy(rp.view(np.int32)).pin_memory().numpy().view(np.uint32),
                   torch.from_numpy(ci.view(np.int32)).pin_memory().numpy().view(np.uint32)) for rp, ci in a]
        outs = [torch.empty(rp.shape[0] - 1, dtype=torch.int32).pin_memory().numpy().view(np.uint32) for rp, _ in a]
        dprep = pbrcm.PreparedBatch(dm, device=True)
        hprep = pbrcm.PreparedBatch(pinned, perms_out=outs)
        for rep in range(3):
            for _, _, p in dm:
                p.fill_(-1)
            # captured, then replayed (the list, then its prepared descriptors)
            res = pbrcm.reorder_batch_device(dm if rep == 0 else dprep, reverse=True, ctx=ctx)
            _check(a, ra, [p.cpu().numpy() for _, _, p in dm], res)
            pbrcm.reorder_batch(b, reverse=True, ctx=ctx)  # pageable: plain launches over the staging
            for o in outs:
                o.fill(0xFFFFFFFF)
            if rep == 0:
                perms, res = pbrcm.reorder_batch(pinned, reverse=True, ctx=ctx, perms_out=outs)
            else:
                perms, res = pbrcm.reorder_batch(hprep, reverse=True, ctx=ctx)
            _check(a, ra, perms, res)
            pbrcm.reorder_batch(b[: 8 + 8 * rep], reverse=True, ctx=ctx)
    finally:
        ctx.close()


def test_batch_pinned_slab_in_place(pbrcm, c4_subset):
    """Host matrices laid out in one pinned slab (row_ptr, col_idx and the
    permutation of each matrix side by side): one copy brings a matrix's CSR
    in, the kernel writes each permutation into the slab itself; captured on
    the first call, replayed on the second."""
    import torch
    mats, refs = c4_subset
    mats, refs = mats[::3], refs[::3]
    words = sum(rp.shape[0] + ci.shape[0] + rp.shape[0] - 1 for rp, ci in mats)
    slab = torch.empty(words, dtype=torch.int32).pin_memory()
    flat = slab.numpy().view(np.uint32)
    hm, hp, o = [], [], 0
    for rp, ci in mats:
        a = flat[o:o + rp.shape[0]]
        a[:] = rp
        o += rp.shape[0]
        b = flat[o:o + ci.shape[0]]
        b[:] = ci
        o += ci.shape[0]
        p = flat[o:o + rp.shape[0] - 1]
        o += rp.shape[0] - 1
        hm.append((a, b))
        hp.append(p)
    ctx = pbrcm.Context(0)
    try:
        prep = pbrcm.PreparedBatch(hm, perms_out=hp)
        for _ in range(2):
            for p in hp:
                p.fill(0xFFFFFFFF)
            perms, res = pbrcm.reorder_batch(prep, reverse=True, ctx=ctx)
            _check(mats, refs, perms, res)
            _check(mats, refs, hp, res)
    finally:
        ctx.close()


def test_batch_large_matrices_global_visited(pbrcm, gpu_ctx, oracle_mod):
    """Matrices over 2^18 nodes in a batch: the one-group engine keeps their
    visited bitmap in global memory (the others in shared memory)."""
    from parallelbatchrcm_b200 import gen
    ms = [gen.grid2d(600, 500, seed=41), gen.grid3d(70, 66, 64, seed=42), gen.rgg(400_000, kmin=4, kmax=12, seed=43),
          gen.grid2d(40, 30, seed=44), gen.grid3d(20, 20, 20, seed=45)]
    assert sum(m.n > (1 << 18) for m in ms) == 3
    perms, results = pbrcm.reorder_batch([(m.row_ptr, m.col_idx) for m in ms], reverse=True, ctx=gpu_ctx)
    for m, p, r in zip(ms, perms, results):
        ref = oracle_mod.full_reorder(m.row_ptr, m.col_idx, reverse=True)
        assert r["status"] == 0 and r["start_node"] == ref["start"]
        assert np.array_equal(p, ref["perm"]) and r["bandwidth"] == ref["bandwidth"]


@pytest.fixture(scope="module")
def c5_stream():
    from parallelbatchrcm_b200 import gen
    stream = gen.poisson_stream_specs(24, rate_per_s=200.0, seed=99)
    # one request of 1-2M nodes in the stream (the generator's top decade)
    big = ("grid3d", (110, 110, 110), 4242)
    stream.insert(5, (stream[5][0], big))
    mats = _pool_map(_make, [s for _, s in stream])
    refs = _pool_map(_oracle_reorder, mats)
    return [t for t, _ in stream], mats, refs


def test_serving_stream_matches_oracle(pbrcm, gpu_ctx, c5_stream):
    arrivals, mats, refs = c5_stream
    assert max(rp.shape[0] - 1 for rp, _ in mats) >= 1_000_000
    sess = pbrcm.Session(gpu_ctx)
    tickets = [None] * len(mats)
    t0 = time.perf_counter()

    def submit():
        for i, (rp, ci) in enumerate(mats):
            d = t0 + arrivals[i] - time.perf_counter()
            if d > 0:
                time.sleep(d)
            tickets[i] = sess.submit(rp, ci, reverse=True)

    th = threading.Thread(target=submit)
    th.start()
    out = [None] * len(mats)
    deadline = time.time() + 300
    while any(o is None for o in out) and time.time() < deadline:
        for i in range(len(mats)):
            if out[i] is None and tickets[i] is not None:
                out[i] = sess.poll(tickets[i])
        time.sleep(0.001)
    th.join()
    st = sess.stats()
    sess.close()
    assert all(o is not None for o in out)
    _check(mats, refs, [o[0] for o in out], [o[1] for o in out])
    assert st["completed"] == len(mats) and st["p99_ms"] >= st["p50_ms"] > 0


def test_admission_refuses_oversize_request(pbrcm, gpu_ctx):
    from parallelbatchrcm_b200 import gen
    m = gen.grid2d(300, 300, seed=5)
    sess = pbrcm.Session(gpu_ctx, memory_cap_bytes=1 << 20)  # 1 MiB: below this request's footprint
    try:
        with pytest.raises(pbrcm.PbrcmError) as e:
            sess.submit(m.row_ptr, m.col_idx)
        assert e.value.status == PBRCM_ERR_BUSY
    finally:
        sess.close()


def test_admission_cap_bounds_bytes_in_flight(pbrcm, gpu_ctx, oracle_mod):
    """A cap that holds one request but not two: the second waits until the
    first has finished; both complete, exactly."""
    from parallelbatchrcm_b200 import gen
    a, b = gen.grid3d(60, 60, 60, seed=6), gen.grid3d(60, 60, 58, seed=7)
    # the device footprint of the larger one, as the session counts it
    with pbrcm.Session(gpu_ctx) as probe:
        t = probe.submit(a.row_ptr, a.col_idx)
        probe.drain()
        probe.poll(t)
        one = probe.stats()["peak_bytes_in_flight"]
    assert one > 4 * a.nnz
    sess = pbrcm.Session(gpu_ctx, memory_cap_bytes=one + (one // 4))  # one fits, two do not
    try:
        ta = sess.submit(a.row_ptr, a.col_idx)
        tb = sess.submit(b.row_ptr, b.col_idx)
        sess.drain()
        pa, ra = sess.poll(ta)
        pb, rb = sess.poll(tb)
        st = sess.stats()
    finally:
        sess.close()
    assert ra["status"] == 0 and rb["status"] == 0
    assert np.array_equal(pa, oracle_mod.full_reorder(a.row_ptr, a.col_idx)["perm"])
    assert np.array_equal(pb, oracle_mod.full_reorder(b.row_ptr, b.col_idx)["perm"])
    assert 0 < st["peak_bytes_in_flight"] <= one
