"""Workloads of bench.py (one JSON line on rank 0 each).

mixed (default)  The metric's own configuration: 4,096 independent matrices,
       n log-uniform in [500, 200,000], 40% 2-D 5-point grids, 30% 3-D
       7-point grids (near-cubic), 30% random geometric graphs with k ~
       U{4..12}, labels shuffled (seed 42).  `value` = batched reorders/s of
       one persistent launch (pbrcm_reorder_batch_device, CSRs resident in
       HBM); beside it plain one-matrix-at-a-time GPU RCM on the same stream
       (pbrcm_reorder_device per matrix), per-matrix p50/p99 latency, e2e
       through pbrcm_reorder_batch from pinned host buffers, the roofline of
       the batch launch, the serving session on a Poisson stream of requests
       (n in [1e3, 2e6], seed 99) against a plain FIFO worker, and the
       single-matrix 128^3 grid and the 64^2 grid (shared-memory engine, the
       reference's serial code timed beside it) as extra keys.  cpu_baseline: the
       reference's own findPeripheral + rcm_seq<true> (oracle/_ref) over the
       same 4,096 matrices on every host thread; its permutations are also
       compared with the batched ones.
single the 128^3 7-point grid alone (one cooperative launch per reorder).
batch  the many-matrix batch alone (any count: PBRCM_BENCH_COUNT).
serve  the serving sweep alone (PBRCM_SERVE_COUNT requests, PBRCM_SERVE_RATES).
permute / connect / wide   P A P^T, the loader's connectivity repair, and a
       wide random graph (level-synchronous engine).
small  small matrices (the 64^2 grid first) on the shared-memory engine
       beside the team engine and the reference's serial CPU code.

Under torchrun each rank takes its own share: the batch stream has
4,096 matrices per GPU (weak scaling, no exchange between GPUs); one matrix
does not shard, so the single-matrix workloads run replicas.
"""
from __future__ import annotations

import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

from parallelbatchrcm_b200 import gen

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "reorders/s & Gnnz/s batched vs plain GPU RCM; p50/p99 latency; bit-exact perms"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------------------
# ranks, clocks, peaks
# ---------------------------------------------------------------------------
def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        # NCCL between GPUs; gloo where there is none (the multi-rank logic is
        # tested that way on CPU)
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws, x: float) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    """(HBM GB/s, "measured"|"fallback"): the pool's measured copy bandwidth."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_value(name: str, key: str):
    """An integer `key: value` line of a committed ncu summary under
    profiles/ (e.g. the DRAM traffic of one launch), or None."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            if line.startswith(key + ":"):
                return int(line.split(":")[1])
    return None


# ---------------------------------------------------------------------------
# algorithmic bytes of one full reorder (u32 indices)
# ---------------------------------------------------------------------------
def reorder_bytes(n: int, nnz: int, passes: int) -> int:
    """Bytes a full reorder must move at least: each start-search BFS pass
    reads row_ptr 4(n+1) and col_idx 4 nnz and writes a visited word 4n; the
    Cuthill-McKee pass moves the same plus the permutation 4n; the bandwidth
    reads row_ptr, col_idx, the permutation and writes the inverse (4n + 4n)
    and gathers the inverse once per entry (4 nnz)."""
    bfs = 4 * (n + 1) + 4 * nnz + 4 * n
    rcm = bfs + 4 * n
    bw = 4 * (n + 1) + 8 * nnz + 8 * n
    return passes * bfs + rcm + bw


# ---------------------------------------------------------------------------
# inputs
# ---------------------------------------------------------------------------
def _make(spec):
    m = gen.make_from_spec(spec)
    return m.row_ptr, m.col_idx


def generate(specs, procs: int | None = None):
    """Generates the matrices of `specs` with a spawn-started process pool
    (safe before or after CUDA is initialised)."""
    procs = procs or max(1, min(len(specs), (os.cpu_count() or 2) - 1, 64))
    if procs == 1 or len(specs) < 8:
        return [_make(s) for s in specs]
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        return pool.map(_make, specs, chunksize=max(1, len(specs) // (procs * 8)))


def mixed_specs(count: int, ws: int, rank: int):
    """This rank's share of the mixed stream: count matrices per GPU drawn
    from one seeded stream of count * ws (rank r takes every ws-th); at one
    GPU exactly the 4,096-matrix configuration."""
    return gen.mixed_batch_specs(count=count * ws, seed=42)[rank::ws]


def quantiles(v):
    v = sorted(v)
    if not v:
        return None, None
    q = lambda f: v[min(len(v) - 1, int(round(f * (len(v) - 1))))]  # noqa: E731
    return q(0.5), q(0.99)


def shard_by_nnz(nnz, parts: int):
    """Greedy longest-first assignment of matrices to `parts` GPUs by nnz (a
    batch of independent matrices needs no exchange between GPUs).  Returns
    one sorted index list per part."""
    load = [0] * parts
    out = [[] for _ in range(parts)]
    for i in sorted(range(len(nnz)), key=lambda k: (-int(nnz[k]), k)):
        p = min(range(parts), key=lambda q: (load[q], q))
        out[p].append(i)
        load[p] += int(nnz[i])
    return [sorted(x) for x in out]


def _oracle():
    """The oracle package (test infrastructure); bench code calls it only in
    its cpu_baseline legs."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    return O


# ---------------------------------------------------------------------------
# reference CPU timings (cpu_baseline legs)
# ---------------------------------------------------------------------------
def reference_stream(mats, reps: int, threads: int | None = None, want_perms: bool = False):
    """The reference's findPeripheral + rcm_seq<true> over the stream on every
    host thread (oracle/_ref/ref_rcm timebatch) `reps` times.  Returns
    (wall seconds per rep, threads, kind, perms or None).  Without the
    reference build: the oracle port, serially, once over the stream."""
    O = _oracle()
    threads = threads or os.cpu_count() or 1
    if O.ref_available():
        out = O.ref_time_batch(mats, threads, reps=reps, want_perms=want_perms)
        info = out[0]
        if any(i["failed"] for i in info):
            raise RuntimeError(f"reference run failed on {max(i['failed'] for i in info)} matrices")
        return [i["wall_ms"] / 1e3 for i in info], threads, "reference", (out[3] if want_perms else None)
    t0 = time.perf_counter()
    perms = [O.full_reorder(rp, ci, reverse=False)["perm"] for rp, ci in mats]
    return [time.perf_counter() - t0], 1, "port", (perms if want_perms else None)


def reference_single(rp, ci, steps: int, threads: int, timeout: float = 600.0):
    """The reference's own CPU code on one matrix (oracle/_ref/ref_rcm time:
    findPeripheral + RealCPU::rcm<true>, serial rcm_seq at 1 thread, else
    CPU_BATCH with batch 512 as src/main.cpp:456-483 runs it), else the port.
    Returns (reorder ms list, kind, threads)."""
    O = _oracle()
    if O.ref_available():
        rows = O.ref_time(rp, ci, threads, steps, timeout=timeout)
        return [r["reorder_ms"] for r in rows], "reference", threads
    ms = []
    for _ in range(steps):
        t0 = time.perf_counter()
        O.full_reorder(rp, ci)
        ms.append((time.perf_counter() - t0) * 1e3)
    return ms, "port", 1


# ---------------------------------------------------------------------------
# the default workload: the 4,096-matrix batch, plain, serving, 128^3 grid
# ---------------------------------------------------------------------------
def _upload(mats, dev):
    import torch
    return [(torch.from_numpy(rp.view(np.int32)).to(dev), torch.from_numpy(ci.view(np.int32)).to(dev),
             torch.empty(rp.shape[0] - 1, dtype=torch.int32, device=dev)) for rp, ci in mats]


def pinned_views(mats):
    """Copies the CSRs into one pinned host slab; returns (row_ptr / col_idx
    views, permutation views, the slab)."""
    import torch
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
        hm.append((a, b))
        hp.append(flat[o:o + rp.shape[0] - 1])
        o += rp.shape[0] - 1
    return hm, hp, slab


def _batched_step(P, ctx, db, stream):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    res = P.reorder_batch_device(db, reverse=True, ctx=ctx, stream=stream)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1), res


def _plain_pass(P, ctx, dmats, stream):
    """Plain one-matrix-at-a-time GPU RCM: pbrcm_reorder_device per matrix
    (one cooperative team launch each), event-timed per matrix."""
    import torch
    lat = []
    for rp_d, ci_d, po in dmats:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        P.reorder_device(rp_d, ci_d, po, reverse=True, ctx=ctx, stream=stream)
        e1.record(stream)
        e1.synchronize()
        lat.append(e0.elapsed_time(e1))
    return lat


def _serve_session(P, ctx, mats, arrivals, streams=96):
    """Submits each request at its arrival time from a thread; once all are
    in, drains the session and reads every result.  Latency = the arrival's
    delay to submission + the session's own submit -> completion time, so
    that no polling loop competes with the session's worker."""
    sess = P.Session(ctx, streams=streams)
    n = len(mats)
    tick = [None] * n
    t_sub = [0.0] * n
    t0 = time.perf_counter() + 0.05

    def submitter():
        for i in range(n):
            while True:
                d = t0 + arrivals[i] - time.perf_counter()
                if d <= 0:
                    break
                time.sleep(min(d, 0.001))
            t_sub[i] = time.perf_counter()
            tick[i] = sess.submit(mats[i][0], mats[i][1])

    th = threading.Thread(target=submitter)
    th.start()
    th.join()
    sess.drain()
    lat, perms = [], []
    for i in range(n):
        out = sess.poll(tick[i])
        assert out is not None and out[1]["status"] == 0, out
        perms.append(out[0])
        lat.append((t_sub[i] - (t0 + arrivals[i])) * 1e3 + out[1]["total_ms"])
    makespan = max(arrivals[i] + lat[i] / 1e3 for i in range(n))
    sess.close()
    return lat, makespan, perms


def _serve_plain(P, ctx, mats, arrivals):
    n = len(mats)
    done_at = [0.0] * n
    perms = [None] * n
    t0 = time.perf_counter() + 0.05
    for i in range(n):
        d = t0 + arrivals[i] - time.perf_counter()
        if d > 0:
            time.sleep(d)
        perms[i], _ = P.reorder(mats[i][0], mats[i][1], ctx=ctx)
        done_at[i] = time.perf_counter()
    lat = [(done_at[i] - (t0 + arrivals[i])) * 1e3 for i in range(n)]
    return lat, max(done_at) - t0, perms


def measure_serve(P, ctx, mats, gaps, rates):
    """Session (continuous batching) against the plain FIFO worker at each
    arrival rate; both from host buffers, latency = arrival -> result.  One
    untimed pass of the session first: it fills the context's pinned
    staging pool, as a running service would have it."""
    _serve_session(P, ctx, mats, [0.0] * len(mats))
    rows = []
    for rate in rates:
        arr = list(np.asarray(gaps) / rate)
        lat_s, span_s, perm_s = _serve_session(P, ctx, mats, arr)
        lat_p, span_p, perm_p = _serve_plain(P, ctx, mats, arr)
        same = all(np.array_equal(a, b) for a, b in zip(perm_s, perm_p))
        p50s, p99s = quantiles(lat_s)
        p50p, p99p = quantiles(lat_p)
        rows.append({"rate_per_s": rate,
                     "session": {"reorders_per_s": len(mats) / span_s, "p50_ms": p50s, "p99_ms": p99s},
                     "plain": {"reorders_per_s": len(mats) / span_p, "p50_ms": p50p, "p99_ms": p99p},
                     "speedup": span_p / span_s, "session_equals_plain": bool(same)})
        log(json.dumps(rows[-1]))
    return rows


def measure_grid3d(P, ctx, m, args, ws, stream, flush, dev, cpu: bool):
    """One full reorder of the 128^3 grid (device-resident, L2 flushed
    between steps; e2e through pbrcm_reorder from pinned host buffers)."""
    import torch
    n, nnz = m.n, m.nnz
    rp_d = torch.from_numpy(m.row_ptr.view(np.int32)).to(dev)
    ci_d = torch.from_numpy(m.col_idx.view(np.int32)).to(dev)
    perm_d = torch.empty(n, dtype=torch.int32, device=dev)

    def step():
        with torch.cuda.stream(stream):
            flush.zero_()
        _, r = P.reorder_device(rp_d, ci_d, perm_d, reverse=True, ctx=ctx, stream=stream)
        return r

    for _ in range(max(3, args.warmup)):
        res = step()
    ms = []
    for _ in range(args.steps):
        res = step()
        ms.append(res["device_ms"])
    pm = perm_d.cpu().numpy().astype(np.uint32)
    rp_h = torch.from_numpy(m.row_ptr.view(np.int32)).pin_memory()
    ci_h = torch.from_numpy(m.col_idx.view(np.int32)).pin_memory()
    perm_h = torch.empty(n, dtype=torch.int32).pin_memory()
    rp_np, ci_np, perm_np = (x.numpy().view(np.uint32) for x in (rp_h, ci_h, perm_h))
    P.reorder(rp_np, ci_np, ctx=ctx, perm_out=perm_np)
    e2e = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        stream.synchronize()
        t1 = time.perf_counter()
        P.reorder(rp_np, ci_np, ctx=ctx, perm_out=perm_np)
        e2e.append((time.perf_counter() - t1) * 1e3)
    assert np.array_equal(perm_np, pm), "e2e permutation differs from the device-path permutation"
    t_dev = max_over_ranks(ws, sum(ms) / 1e3)
    t_e2e = max_over_ranks(ws, sum(e2e) / 1e3)
    peak, peak_kind = measured_peak()
    abytes = reorder_bytes(n, nnz, res["peripheral_passes"])
    achieved = abytes / (statistics.mean(ms) / 1e3) / 1e9
    out = {
        "workload": "grid3d_128^3_7pt_rcm", "n": n, "nnz": nnz, "value": ws * args.steps / t_dev,
        "unit": "reorders/s", "ms_per_step": t_dev * 1e3 / args.steps,
        "l2": "flushed (256 MiB write) between steps",
        "e2e": {"value": ws * args.steps / t_e2e, "unit": "reorders/s", "h2d_bytes_per_step": 4 * (n + 1) + 4 * nnz,
                "d2h_bytes_per_step": 4 * n + 64},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "kernel": "k_reorder_team<256,1024>",
                     "algorithmic_bytes_per_launch": abytes,
                     "traffic": profile_value("k_reorder_team_grid3d_128.md", "traffic_bytes_per_launch")},
        "result": {"start": res["start_node"], "passes": res["peripheral_passes"], "ecc": res["eccentricity"],
                   "levels": res["levels"], "bandwidth": res["bandwidth"], "profile": res["profile"]},
    }
    # the latency view: the reorder is a chain of dependent BFS levels (each
    # search pass and the final pass walk about `levels` of them; the last
    # search pass runs beside the final pass), so time per level of that chain
    # says more than the HBM fraction
    chain = res["peripheral_passes"] * res["levels"]
    out["level_chain"] = {"levels": chain, "us_per_level": t_dev * 1e6 / args.steps / max(1, chain),
                          "what": "passes x levels of the final order (the last search pass runs beside the "
                                  "final pass); device time per level of that chain"}
    if cpu:
        try:
            threads = os.cpu_count() or 1
            ms_b, kind, thr = reference_single(m.row_ptr, m.col_idx, 3, threads)
            ms_s, _, _ = reference_single(m.row_ptr, m.col_idx, 1, 1)
            out["cpu_baseline"] = {
                "value": 1e3 / statistics.median(ms_b), "unit": "reorders/s", "cores": thr, "kind": kind,
                "sample": "3 full reorders: findPeripheral + RealCPU::rcm<true> with CPU_BATCH (batch 512) on every "
                          "host thread (its reported mean of 25 internal repetitions), median",
                "serial_rcm_seq": {"value": 1e3 / statistics.median(ms_s), "unit": "reorders/s", "cores": 1,
                                   "sample": "1 full reorder: findPeripheral + rcm_seq<true> (mean of 25)"}}
        except Exception as e:  # reported, never required
            out["cpu_baseline"] = {"value": None, "kind": "unavailable", "sample": str(e)[:200]}
    return out


def run_mixed(args, ws, rank, local, extras: bool = True):
    import torch

    import parallelbatchrcm_b200 as P

    if getattr(args, "lean", False):
        return run_batch_lean(args, ws, rank, local)

    count = int(os.environ.get("PBRCM_BENCH_COUNT", "4096"))
    serve_n = int(os.environ.get("PBRCM_BENCH_SERVE", "160")) if ws == 1 and extras else 0
    rates = [float(x) for x in os.environ.get("PBRCM_BENCH_RATES", "400,100000").split(",")]
    t0 = time.time()
    specs = mixed_specs(count, ws, rank)
    mats = generate(specs)
    sum_n = sum(int(rp.shape[0] - 1) for rp, _ in mats)
    sum_nnz = sum(int(ci.shape[0]) for _, ci in mats)
    log(f"[rank {rank}] generated {count} matrices: sum n={sum_n} sum nnz={sum_nnz} in {time.time() - t0:.1f}s")
    serve_mats, gaps = [], []
    if serve_n:
        sspecs = gen.poisson_stream_specs(serve_n, rate_per_s=1.0, seed=99)
        gaps = [t for t, _ in sspecs]
        serve_mats = generate([s for _, s in sspecs])
    g3 = gen.grid3d(128, 128, 128, seed=12345) if extras else None
    log(f"[rank {rank}] inputs ready in {time.time() - t0:.1f}s")

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    ctx = P.Context(local)
    stream = torch.cuda.Stream(device=dev)
    dmats = _upload(mats, dev)
    db = P.PreparedBatch(dmats, device=True)  # descriptors of the resident buffers, built once
    torch.cuda.synchronize()

    # batched: W untimed, K timed (CUDA events on the launching stream)
    for _ in range(args.warmup):
        _batched_step(P, ctx, db, stream)
    barrier(ws)
    torch.cuda.synchronize()
    times = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            ms, res = _batched_step(P, ctx, db, stream)
            times.append(ms)
        torch.cuda.synchronize()
    barrier(ws)
    torch.cuda.synchronize()
    assert all(r["status"] == 0 for r in res), [r for r in res if r["status"] != 0][:3]
    t_batch = max_over_ranks(ws, sum(times) / 1e3)
    value = ws * count * args.steps / t_batch
    bperm = [p.cpu().numpy().view(np.uint32).copy() for _, _, p in dmats]
    lat50, lat99 = quantiles([r["device_ms"] for r in res])

    # plain one-at-a-time on the same matrices
    lat = _plain_pass(P, ctx, dmats, stream)
    plain_same = all(np.array_equal(a, p.cpu().numpy().view(np.uint32)) for a, (_, _, p) in zip(bperm, dmats))
    t_plain = max_over_ranks(ws, sum(lat) / 1e3)
    plain_value = ws * count / t_plain
    p50, p99 = quantiles(lat)

    # e2e through pbrcm_reorder_batch from pinned host buffers (one pinned
    # slab, the matrices and permutations as views into it)
    hm, hp, slab = pinned_views(mats)
    hb = P.PreparedBatch(hm, perms_out=hp)  # the descriptors of the fixed pinned staging, built once
    P.reorder_batch(hb, reverse=True, ctx=ctx)
    e2e_steps = max(2, args.steps // 2)
    barrier(ws)
    e2e = []
    for _ in range(e2e_steps):
        t1 = time.perf_counter()
        P.reorder_batch(hb, reverse=True, ctx=ctx)
        e2e.append(time.perf_counter() - t1)
    barrier(ws)
    e2e_same = all(np.array_equal(a, b) for a, b in zip(bperm, hp))
    t_e2e = max_over_ranks(ws, sum(e2e))
    e2e_value = ws * count * e2e_steps / t_e2e

    # roofline of the batch launch: the algorithmic bytes of every matrix's
    # full reorder over the launch's mean event time
    peak, peak_kind = measured_peak()
    abytes = sum(reorder_bytes(int(rp.shape[0] - 1), int(ci.shape[0]), r["peripheral_passes"])
                 for (rp, ci), r in zip(mats, res))
    achieved = abytes / (statistics.mean(times) / 1e3) / 1e9
    traffic = profile_value("k_solo_batch_mixed_batch_4096.md", "traffic_bytes_per_launch")

    serve = None
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device=dev)
    if serve_n:
        rows = measure_serve(P, ctx, serve_mats, gaps, rates)
        serve = {"workload": f"serve_poisson_{serve_n}", "n_range": [1000, 2_000_000], "seed": 99,
                 "admission_cap_gb": 120, "sweep": rows}
    g3_out = None
    if g3 is not None:
        g3_out = measure_grid3d(P, ctx, g3, args, ws, stream, flush, dev,
                                cpu=rank == 0 and ws == 1 and not args.no_cpu_baseline)

    # the 64^2 grid alone (shared-memory engine), the reference's serial code
    # beside it: reported, never required
    g2_out = None
    if extras and rank == 0 and ws == 1:
        try:
            team = _team_context(P, local)
            try:
                g2_out = _small_row(P, _oracle(), ctx, team, gen.grid2d(64, 64, seed=1), "grid2d_64x64",
                                    3, 20, dev, stream)
            finally:
                team.close()
        except Exception as e:
            g2_out = {"workload": "grid2d_64x64", "error": str(e)[:200]}

    cpu = None
    ref_same = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            walls, thr, kind, rperms = reference_stream(mats, reps=1, want_perms=True)
            ref_same = all(np.array_equal(a[::-1], b) for a, b in zip(bperm, rperms))
            cpu = {"value": count / statistics.median(walls), "unit": "reorders/s", "cores": thr, "kind": kind,
                   "sample": f"the same {count} matrices, once: findPeripheral + rcm_seq<true> per matrix "
                             f"(the reference's serial stable path), {thr} host threads each taking the next "
                             f"matrix; wall time of the pool"}
        except Exception as e:  # reported, never required
            cpu = {"value": None, "unit": "reorders/s", "cores": 0, "kind": "unavailable", "sample": str(e)[:200]}

    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": "reorders/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_batch * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded mixed 2-D / 3-D grids and random geometric graphs, shuffled labels)",
        "config": {"workload": f"mixed_batch_{count}", "matrices_per_gpu": count, "sum_n": sum_n,
                   "sum_nnz": sum_nnz, "n_range": [500, 200_000], "mix": "40% 2-D grid, 30% 3-D grid, 30% RGG k 4..12",
                   "seed": 42, "reverse": True, "start": "auto",
                   "l2": f"inputs larger than L2 ({4 * (sum_n + count + sum_nnz) / 1e9:.1f} GB of CSRs)",
                   "parallelism": f"{ws} GPU(s), {count} matrices each, no exchange"},
        "gnnz_per_s": value * (sum_nnz / count) / 1e9,
        "latency_ms": {"what": "per matrix, from the batch's first matrix taken to its result (device clock)",
                       "p50": lat50, "p99": lat99},
        "plain_one_at_a_time": {"value": plain_value, "unit": "reorders/s", "total_ms": t_plain * 1e3,
                                "p50_ms": p50, "p99_ms": p99,
                                "what": "pbrcm_reorder_device per matrix, event-timed"},
        "speedup_vs_plain": value / plain_value,
        "parity": {"batched_equals_plain": bool(plain_same), "e2e_equals_device": bool(e2e_same),
                   "batched_equals_reference": ref_same,
                   "reference": "oracle/_ref: findPeripheral + rcm_seq<true>, every matrix, reversed"},
        "e2e": {"value": e2e_value, "unit": "reorders/s",
                "h2d_bytes_per_step": int(sum(4 * (rp.shape[0] + ci.shape[0]) for rp, ci in mats)),
                "d2h_bytes_per_step": int(4 * sum_n + 64 * count), "steps": e2e_steps,
                "what": "pbrcm_reorder_batch: pinned host CSRs in, permutations to pinned host buffers (a PreparedBatch over the fixed pinned staging)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "kernel": "k_solo_batch (the batch launch)",
                     "algorithmic_bytes_per_launch": abytes, "traffic": traffic},
        "serve": serve,
        "grid3d_128": g3_out,
        "grid2d_64": g2_out,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
        "gpu_launches": 2 * args.steps,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_batch_lean(args, ws, rank, local):
    """Only the batched launches of the default workload (PBRCM_BENCH_COUNT
    matrices): W + K steps of pbrcm_reorder_batch_device, one JSON line with
    their event time.  Made for profiling, where every other leg would add
    thousands of launches."""
    import torch

    import parallelbatchrcm_b200 as P

    count = int(os.environ.get("PBRCM_BENCH_COUNT", "4096"))
    mats = generate(mixed_specs(count, ws, rank))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    ctx = P.Context(local)
    stream = torch.cuda.Stream(device=dev)
    dmats = _upload(mats, dev)
    db = P.PreparedBatch(dmats, device=True)  # descriptors of the resident buffers, built once
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        _batched_step(P, ctx, db, stream)
    times = [_batched_step(P, ctx, db, stream)[0] for _ in range(args.steps)]
    if rank == 0:
        sum_nnz = sum(int(ci.shape[0]) for _, ci in mats)
        print(json.dumps({"metric": METRIC, "value": count * len(times) / (sum(times) / 1e3), "unit": "reorders/s",
                          "ms_per_step": statistics.mean(times), "config": {"workload": f"mixed_batch_{count}",
                                                                            "sum_nnz": sum_nnz, "lean": True}}),
              flush=True)
    return 0


def run_mixed_reference(args, ws, rank):
    """--impl reference on the default workload: the reference's own CPU code
    over the same matrices (rank 0 alone; the other ranks exit 0)."""
    if rank != 0:
        return 0
    count = int(os.environ.get("PBRCM_BENCH_COUNT", "4096"))
    mats = generate(mixed_specs(count, ws, 0))
    sum_nnz = sum(int(ci.shape[0]) for _, ci in mats)
    walls, thr, kind, _ = reference_stream(mats, reps=args.warmup + args.steps)
    timed = walls[args.warmup:] if len(walls) > args.warmup else walls
    t = sum(timed)
    value = count * len(timed) / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "reorders/s", "n_gpus": args.gpus,
        "steps": len(timed), "warmup": args.warmup, "ms_per_step": t * 1e3 / len(timed), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded mixed 2-D / 3-D grids and random geometric graphs, shuffled labels)",
        "config": {"workload": f"mixed_batch_{count}", "matrices_per_gpu": count,
                   "sum_n": sum(int(rp.shape[0]) - 1 for rp, _ in mats), "sum_nnz": sum_nnz,
                   "n_range": [500, 200_000], "mix": "40% 2-D grid, 30% 3-D grid, 30% RGG k 4..12", "seed": 42,
                   "reverse": True, "start": "auto",
                   "l2": f"inputs larger than L2 ({4 * (sum(int(rp.shape[0]) for rp, _ in mats) + sum_nnz) / 1e9:.1f} GB of CSRs)",
                   "parallelism": f"host threads, {count} matrices, no exchange"},
        "gnnz_per_s": value * (sum_nnz / count) / 1e9,
        "cpu_baseline": {"value": value, "unit": "reorders/s", "cores": thr, "kind": kind,
                         "sample": f"each step: the whole stream of {count} matrices, findPeripheral + "
                                   f"rcm_seq<true> per matrix on {thr} host threads"},
        "e2e": {"value": value, "unit": "reorders/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# the other workloads
# ---------------------------------------------------------------------------
def run_single(args, ws, rank, local):
    """The 128^3 grid alone (replicas under torchrun)."""
    import torch

    import parallelbatchrcm_b200 as P

    m = gen.grid3d(128, 128, 128, seed=12345)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    ctx = P.Context(local)
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device=dev)
    barrier(ws)
    with ClockSampler(local) as clk:
        out = measure_grid3d(P, ctx, m, args, ws, stream, flush, dev,
                             cpu=rank == 0 and ws == 1 and not args.no_cpu_baseline)
    barrier(ws)
    if rank != 0:
        return 0
    line = {"metric": "reorders/s (full reorder: start search + RCM + bandwidth)", "value": out.pop("value"),
            "unit": "reorders/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": out.pop("ms_per_step"), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded 128^3 7-point grid pattern, shuffled labels)",
            "config": {"workload": out.pop("workload"), "n": out.pop("n"), "nnz": out.pop("nnz"),
                       "l2": out.pop("l2"), "parallelism": f"replicas x{ws}"},
            "clocks": clk.summary(), "gpu_launches": 2 * args.steps}
    line.update(out)
    print(json.dumps(line), flush=True)
    return 0


def run_single_reference(args, ws, rank):
    if rank != 0:
        return 0
    m = gen.grid3d(128, 128, 128, seed=12345)
    threads = os.cpu_count() or 1
    if args.warmup > 0:
        reference_single(m.row_ptr, m.col_idx, 1, threads)
    ms, kind, cores = reference_single(m.row_ptr, m.col_idx, args.steps, threads)
    t = sum(ms) / 1e3
    value = args.steps / t
    line = {
        "impl": "reference", "metric": "reorders/s (full reorder: start search + RCM + bandwidth)",
        "value": value, "unit": "reorders/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32", "data": "synthetic (seeded 128^3 7-point grid pattern, shuffled labels)",
        "config": {"workload": "grid3d_128^3_7pt_rcm", "n": m.n, "nnz": m.nnz},
        "cpu_baseline": {"value": value, "unit": "reorders/s", "cores": cores, "kind": kind,
                         "sample": f"{args.steps} full reorders: findPeripheral + RealCPU::rcm<true> (CPU_BATCH)"},
        "e2e": {"value": value, "unit": "reorders/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_serve(args, ws, rank, local):
    """The serving sweep alone: PBRCM_SERVE_COUNT requests of the Poisson
    stream at each rate of PBRCM_SERVE_RATES."""
    import torch

    import parallelbatchrcm_b200 as P

    count = int(os.environ.get("PBRCM_SERVE_COUNT", "256"))
    rates = [float(x) for x in os.environ.get("PBRCM_SERVE_RATES", "50,200,1000,100000").split(",")]
    sspecs = gen.poisson_stream_specs(count, rate_per_s=1.0, seed=99)
    gaps = [t for t, _ in sspecs]
    mats = generate([s for _, s in sspecs])
    torch.cuda.set_device(local)
    ctx = P.Context(local)
    _serve_session(P, ctx, mats[:16], [0.0] * 16)
    for rp, ci in mats[:4]:
        P.reorder(rp, ci, ctx=ctx)
    rows = measure_serve(P, ctx, mats, gaps, rates)
    best = rows[-1]
    line = {
        "metric": "reorders/s (serving, continuous batching, Poisson arrivals)",
        "value": best["session"]["reorders_per_s"], "unit": "reorders/s", "n_gpus": ws, "steps": len(rates),
        "warmup": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded Poisson stream of grids / RGGs, n in [1e3, 2e6])",
        "config": {"workload": f"serve_poisson_{count}", "rates": rates, "admission_cap_gb": 120},
        "sweep": rows,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_permute(args, ws, rank, local):
    """The reordered matrix B = P A P^T of the 128^3 grid (float64 values, its
    RCM order) through pbrcm_permute_device, device-resident, L2 flushed
    between steps; reports permutes/s and the HBM bytes the call must move."""
    import torch

    import parallelbatchrcm_b200 as P
    from parallelbatchrcm_b200 import gen

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    m = gen.grid3d(128, 128, 128, seed=12345)
    n, nnz = m.n, m.nnz
    ctx = P.Context(local)
    stream = torch.cuda.Stream(device=dev)
    rp = torch.from_numpy(m.row_ptr.view(np.int32)).to(dev)
    ci = torch.from_numpy(m.col_idx.view(np.int32)).to(dev)
    vals = torch.rand(nnz, dtype=torch.float64, device=dev)
    perm, _ = P.reorder_device(rp, ci, reverse=True, ctx=ctx)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device=dev)

    def step():
        with torch.cuda.stream(stream):
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = P.permute_device(rp, ci, perm, vals, ctx=ctx, stream=stream)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), out

    for _ in range(max(3, args.warmup)):
        step()
    ms = [step()[0] for _ in range(args.steps)]
    ms_med = statistics.median(ms)
    # inputs row_ptr, col_idx, values, perm; outputs row_ptr, col_idx, values
    abytes = 4 * (n + 1) + 4 * nnz + 8 * nnz + 4 * n + 4 * (n + 1) + 4 * nnz + 8 * nnz
    peak = None
    try:
        peak = measured_peak()[0]
    except (OSError, ValueError, TypeError, KeyError):
        peak = None
    achieved = abytes / (ms_med / 1e3) / 1e9
    line = {
        "metric": "permutes/s (B = P A P^T, float64 values)", "value": 1e3 / ms_med, "unit": "permutes/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_med, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32+f64", "data": "synthetic (seeded 128^3 grid, RCM order)",
        "config": {"workload": "grid3d_128^3_permute_f64", "n": n, "nnz": nnz,
                   "l2": "flushed (256 MiB write) between steps"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak if peak else None, "algorithmic_bytes": abytes,
                     "includes": "the CSR check and one stream synchronisation of the call"},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_connect(args, ws, rank, local):
    """The loader's connectivity repair on the device (pbrcm_connect_device)
    for a 4M-node random geometric graph of 1-3 nearest neighbours per point
    (about 160k components; the rgg generator with its components left
    apart); inputs
    device-resident, L2 flushed between steps.  e2e: the host CSR copied in,
    joined, and the joined CSR copied back every step.  cpu_baseline: the
    oracle's restatement of the reference's repair on one host core."""
    import torch

    import parallelbatchrcm_b200 as P
    from parallelbatchrcm_b200 import gen

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    m = gen.rgg(4_000_000, kmin=1, kmax=3, long_frac=0.0, connect=False)
    n, nnz = m.n, m.nnz
    ctx = P.Context(local)
    stream = torch.cuda.Stream(device=dev)
    rp = torch.from_numpy(m.row_ptr.view(np.int32)).to(dev)
    ci = torch.from_numpy(m.col_idx.view(np.int32)).to(dev)
    _, oci, links = P.connect_device(rp, ci, ctx=ctx, stream=stream)
    cap = oci.numel()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device=dev)

    def step():
        with torch.cuda.stream(stream):
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        P.connect_device(rp, ci, cap=cap, ctx=ctx, stream=stream)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    for _ in range(max(3, args.warmup)):
        step()
    ms_med = statistics.median([step() for _ in range(args.steps)])

    h_rp = torch.from_numpy(m.row_ptr.view(np.int32)).pin_memory()
    h_ci = torch.from_numpy(m.col_idx.view(np.int32)).pin_memory()
    o_rp = torch.empty(n + 1, dtype=torch.int32).pin_memory()
    o_ci = torch.empty(cap, dtype=torch.int32).pin_memory()

    def e2e_step():
        with torch.cuda.stream(stream):
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        with torch.cuda.stream(stream):
            d_rp = h_rp.to(dev, non_blocking=True)
            d_ci = h_ci.to(dev, non_blocking=True)
        orp, oci2, _ = P.connect_device(d_rp, d_ci, cap=cap, ctx=ctx, stream=stream)
        with torch.cuda.stream(stream):
            o_rp.copy_(orp, non_blocking=True)
            o_ci[:oci2.numel()].copy_(oci2, non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    for _ in range(3):
        e2e_step()
    e2e_ms = statistics.median([e2e_step() for _ in range(args.steps)])

    cpu = None
    if not args.no_cpu_baseline:
        O = _oracle()
        t0 = time.perf_counter()
        reps = 0
        while reps < 3 or time.perf_counter() - t0 < 2.0:
            O.prepare_csr(m.row_ptr, m.col_idx, check_sym=False)
            reps += 1
        cpu_s = (time.perf_counter() - t0) / reps
        cpu = {"value": 1.0 / cpu_s, "unit": "connects/s", "cores": 1, "kind": "port",
               "sample": f"{reps} full repairs of the same graph"}

    nnz_out = nnz + 2 * links
    # row_ptr and col_idx in and out, the parent array written and read once
    abytes = 4 * (n + 1) + 4 * nnz + 4 * (n + 1) + 4 * nnz_out + 8 * n
    peak = None
    try:
        peak = measured_peak()[0]
    except (OSError, ValueError, TypeError, KeyError):
        peak = None
    achieved = abytes / (ms_med / 1e3) / 1e9
    line = {
        "metric": "connects/s (loader connectivity repair)", "value": 1e3 / ms_med, "unit": "connects/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_med, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded RGG, components apart)",
        "config": {"workload": "rgg_4M_k1-3_connect", "n": n, "nnz": nnz, "links": links,
                   "l2": "flushed (256 MiB write) between steps"},
        "e2e": {"value": 1e3 / e2e_ms, "unit": "connects/s", "h2d_bytes_per_step": 4 * (n + 1) + 4 * nnz,
                "d2h_bytes_per_step": 4 * (n + 1) + 4 * nnz_out},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak if peak else None, "algorithmic_bytes": abytes,
                     "includes": "the CSR check and one stream synchronisation of the call"},
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_wide(args, ws, rank, local):
    """Full reorder of a 2M-node random graph of degree 14 (10 BFS levels, the
    widest 1.46M nodes) through pbrcm_reorder_device, device-resident, L2
    flushed between steps: the default context (the team kernel hands the
    matrix to the level-synchronous engine) beside a team-only context
    (PBRCM_WIDE_DIV=0).  cpu_baseline: the oracle's serial restatement of the
    reference's findPeripheral + rcm_seq<true>, one full reorder."""
    import torch

    import parallelbatchrcm_b200 as P
    from parallelbatchrcm_b200 import gen

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    m = gen.erdos_renyi(2_000_000, 14, seed=2)
    n, nnz = m.n, m.nnz
    ctx = P.Context(local)
    old = os.environ.get("PBRCM_WIDE_DIV")
    os.environ["PBRCM_WIDE_DIV"] = "0"
    try:
        team_ctx = P.Context(local)
    finally:
        if old is None:
            os.environ.pop("PBRCM_WIDE_DIV", None)
        else:
            os.environ["PBRCM_WIDE_DIV"] = old
    stream = torch.cuda.Stream(device=dev)
    rp = torch.from_numpy(m.row_ptr.view(np.int32)).to(dev)
    ci = torch.from_numpy(m.col_idx.view(np.int32)).to(dev)
    perm = torch.empty(n, dtype=torch.int32, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device=dev)

    def step(c):
        with torch.cuda.stream(stream):
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _, res = P.reorder_device(rp, ci, perm, reverse=True, ctx=c, stream=stream)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), res

    for _ in range(max(3, args.warmup)):
        step(ctx)
        step(team_ctx)
    ms, ms_team = [], []
    for _ in range(args.steps):
        t, res = step(ctx)
        ms.append(t)
        ms_team.append(step(team_ctx)[0])
    p_auto = perm.cpu().numpy().copy()
    step(team_ctx)
    same = bool(np.array_equal(p_auto, perm.cpu().numpy()))
    ms_med, team_med = statistics.median(ms), statistics.median(ms_team)
    cpu = None
    if not args.no_cpu_baseline:
        O = _oracle()
        t0 = time.perf_counter()
        O.full_reorder(m.row_ptr, m.col_idx, reverse=True)
        cpu_s = time.perf_counter() - t0
        cpu = {"value": 1.0 / cpu_s, "unit": "reorders/s", "cores": 1, "kind": "port",
               "sample": "1 full reorder of the same graph with the C oracle (serial)"}
    line = {
        "metric": "reorders/s (full reorder: start search + RCM + bandwidth)", "value": 1e3 / ms_med,
        "unit": "reorders/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_med,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded random graph, degree 14)",
        "config": {"workload": "erdos_renyi_2M_d14_rcm", "n": n, "nnz": nnz, "reverse": True, "start": "auto",
                   "l2": "flushed (256 MiB write) between steps"},
        "engine": res["engine"], "levels": res["levels"], "passes": res["peripheral_passes"],
        "team_only": {"value": 1e3 / team_med, "unit": "reorders/s", "ms_per_step": team_med,
                      "same_permutation": same},
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    return 0


def _single_configs():
    """The single-matrix configurations: 64^2 and 128^3 grids, 1M-point RGG."""
    return [("grid2d_64x64", lambda: gen.grid2d(64, 64, seed=1)),
            ("grid3d_128^3", lambda: gen.grid3d(128, 128, 128, seed=12345)),
            ("rgg_1M_k6-14", lambda: gen.rgg(1_000_000, seed=7))]


def run_refgpu(args, ws, rank, local):
    """The reference's own GPU path GPU_SIMPLE (src/device/rcm_gpu.cu,
    compiled unchanged for sm_100a: oracle/_ref/ref_gpu_simple) beside this
    engine on the single-matrix configurations, both from the start node the
    reference's findPeripheral picks (the time of one Cuthill-McKee pass, as
    GPU_SIMPLE::rcm reports it: mean of 20 runs after 5 warm-ups).  Also
    counts where GPU_SIMPLE's order differs from the serial stable one.  The
    reference's GPU_BATCH kernel is not run: its waits are unbounded and it
    traps on an internal overflow (include/device/batchWorker.cuh:213-279,
    539-543)."""
    import torch

    import parallelbatchrcm_b200 as P
    if rank != 0:
        return 0
    O = _oracle()
    torch.cuda.set_device(local)
    ctx = P.Context(local)
    dev = torch.device("cuda", local)
    rows = []
    for name, make in _single_configs():
        m = make()
        start, _, _ = O.peripheral(m.row_ptr, m.col_idx)
        cm = O.cm_order(m.row_ptr, m.col_idx, start)
        ref = O.ref_gpu_simple(m.row_ptr, m.col_idx, start)
        rp = torch.from_numpy(m.row_ptr.view(np.int32)).to(dev)
        ci = torch.from_numpy(m.col_idx.view(np.int32)).to(dev)
        po = torch.empty(m.n, dtype=torch.int32, device=dev)
        ms = []
        for i in range(25):
            _, r = P.reorder_device(rp, ci, po, reverse=False, start=int(start), want_bandwidth=False, ctx=ctx)
            if i >= 5:
                ms.append(r["device_ms"])
        ours = po.cpu().numpy().view(np.uint32)
        row = {"workload": name, "n": m.n, "nnz": m.nnz, "start": int(start),
               "ours_ms": statistics.mean(ms), "ours_equals_serial_stable": bool(np.array_equal(ours, cm)),
               "ours_bandwidth": O.bandwidth(m.row_ptr, m.col_idx, ours)}
        if ref is not None:
            rms, rperm = ref
            row.update({"gpu_simple_ms": rms, "gpu_simple_positions_differing": int((rperm != cm).sum()),
                        "gpu_simple_bandwidth": O.bandwidth(m.row_ptr, m.col_idx, rperm),
                        "speedup": rms / statistics.mean(ms)})
        rows.append(row)
        log(json.dumps(row))
    print(json.dumps({"metric": "ms per Cuthill-McKee pass from a given start (reference GPU_SIMPLE vs ours)",
                      "rows": rows, "gpu_batch": "not run: unbounded device waits and a reachable __trap "
                                                 "(include/device/batchWorker.cuh:213-279, 539-543)"}), flush=True)
    return 0


def _small_configs():
    """Matrices the shared-memory engine takes, the 64^2 grid first."""
    return [("grid2d_64x64", lambda: gen.grid2d(64, 64, seed=1)),
            ("grid2d_32x32", lambda: gen.grid2d(32, 32, seed=2)),
            ("grid3d_16^3", lambda: gen.grid3d(16, 16, 16, seed=4)),
            ("grid2d_90x60", lambda: gen.grid2d(90, 60, seed=6)),
            ("rgg_3000_k4-12", lambda: gen.rgg(3000, kmin=4, kmax=12, seed=5))]


def _team_context(P, local):
    """A context that keeps every single matrix on the team engine."""
    old = os.environ.get("PBRCM_ENGINE")
    os.environ["PBRCM_ENGINE"] = "team"
    try:
        return P.Context(local)
    finally:
        if old is None:
            os.environ.pop("PBRCM_ENGINE")
        else:
            os.environ["PBRCM_ENGINE"] = old


def _small_row(P, O, ctx, team, m, name, warmup, steps, dev, st):
    """One small matrix: full reorders on `ctx` (the shared-memory engine)
    device-resident (CUDA events on `st`, median) and end to end from host
    buffers (pbrcm_reorder's own wall time, median), on `team` (the team
    engine alone), and the reference's own findPeripheral + rcm_seq on one
    host thread; every permutation checked against the oracle."""
    import torch
    ref = O.full_reorder(m.row_ptr, m.col_idx, reverse=True)
    rp = torch.from_numpy(m.row_ptr.view(np.int32)).to(dev)
    ci = torch.from_numpy(m.col_idx.view(np.int32)).to(dev)
    po = torch.empty(m.n, dtype=torch.int32, device=dev)

    def timed(c):
        ts = []
        for i in range(warmup + steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            _, r = P.reorder_device(rp, ci, po, ctx=c, stream=st)
            e1.record(st)
            e1.synchronize()
            if i >= warmup:
                ts.append(e0.elapsed_time(e1))
        ok = np.array_equal(po.cpu().numpy().view(np.uint32), ref["perm"])
        return statistics.median(ts), r["engine"], ok

    ms, engine, ok = timed(ctx)
    tms, tengine, tok = timed(team)
    hp = np.empty(m.n, dtype=np.uint32)
    e2e = []
    for i in range(warmup + steps):
        _, r = P.reorder(m.row_ptr, m.col_idx, ctx=ctx, perm_out=hp)
        if i >= warmup:
            e2e.append(r["total_ms"])
    row = {"workload": name, "n": m.n, "nnz": m.nnz, "engine": engine, "ms": ms,
           "e2e_ms": statistics.median(e2e), "team_ms": tms,
           "equals_oracle": bool(ok and tok and np.array_equal(hp, ref["perm"])), "team_engine": tengine}
    if O.ref_available():
        rr = O.ref_time(m.row_ptr, m.col_idx, 1, 1)[0]
        row.update({"reference_peripheral_ms": rr["peripheral_ms"], "reference_rcm_ms": rr["rcm_ms"],
                    "reference_ms": rr["peripheral_ms"] + rr["rcm_ms"]})
    return row


def run_small(args, ws, rank, local):
    """Small matrices, one at a time (rank 0; _small_row each): the
    shared-memory engine beside the team engine and the reference's serial
    code."""
    import torch

    import parallelbatchrcm_b200 as P
    if rank != 0:
        return 0
    O = _oracle()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = P.Context(local)
    team = _team_context(P, local)
    st = torch.cuda.Stream(device=dev)
    rows = []
    for name, make in _small_configs():
        rows.append(_small_row(P, O, ctx, team, make(), name, args.warmup, args.steps, dev, st))
        log(json.dumps(rows[-1]))
    ctx.close()
    team.close()
    print(json.dumps({"metric": "ms per full reorder of a small matrix: shared-memory engine (device, end to end) "
                                "vs team engine vs the reference's serial CPU code (1 thread)",
                      "rows": rows}), flush=True)
    return 0


def run_cpu(args, ws, rank, local):
    """The reference's CPU paths on the single-matrix configurations, on this
    host: findPeripheral + RealCPU::rcm<true> serial (rcm_seq) and CPU_BATCH
    with 2..nproc threads (batch 512), as src/main.cpp:456-483 runs them; each
    RealCPU::rcm reports the mean of its 25 internal repetitions."""
    if rank != 0:
        return 0
    import platform
    nproc = os.cpu_count() or 1
    threads = [t for t in (1, 2, 4, 8, 16, 32, 64) if t <= nproc]
    if threads[-1] != nproc:
        threads.append(nproc)
    rows = []
    for name, make in _single_configs():
        m = make()
        row = {"workload": name, "n": m.n, "nnz": m.nnz}
        for t in threads:
            ms, kind, _ = reference_single(m.row_ptr, m.col_idx, 1, t)
            row[f"threads_{t}_reorder_ms"] = ms[0]
        O = _oracle()
        rr = O.ref_time(m.row_ptr, m.col_idx, 1, 1)[0]
        row["peripheral_ms"] = rr["peripheral_ms"]
        row["serial_rcm_ms"] = rr["rcm_ms"]
        rows.append(row)
        log(json.dumps(row))
    cpu_model = platform.processor() or ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    cpu_model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    print(json.dumps({"metric": "ms per full reorder on the host (reference CPU code)", "cpu": cpu_model,
                      "nproc": nproc, "rows": rows}), flush=True)
    return 0


def main(args, ws, rank, local):
    if args.impl == "reference":
        if args.workload == "single":
            return run_single_reference(args, ws, rank)
        return run_mixed_reference(args, ws, rank)
    fn = {"mixed": run_mixed, "single": run_single, "serve": run_serve, "permute": run_permute,
          "connect": run_connect, "wide": run_wide, "refgpu": run_refgpu, "cpu": run_cpu,
          "small": run_small}.get(args.workload)
    if args.workload == "batch":
        return run_mixed(args, ws, rank, local, extras=False)
    if fn is None:
        raise ValueError(args.workload)
    return fn(args, ws, rank, local)
