"""Many-matrix and serving benchmarks (``bench.py --workload batch|serve``).

batch  4096 independent matrices, n log-uniform in [500, 200000]: 40% 2-D
       grids, 30% 3-D grids, 30% RGGs with k ~ U{4..12} (seed 42).  Measures
       the one-launch batched engine (pbrcm_reorder_batch_device, CSRs resident
       in HBM) against plain one-matrix-at-a-time GPU RCM (one team launch per
       matrix, pbrcm_reorder_device, same engine), checks that every batched
       permutation equals the one-at-a-time one, and samples matrices against
       the oracle.
serve  Poisson arrivals of requests with n log-uniform in [1000, 2000000]
       over the three generators (seed 99).  The serving session (continuous
       batching) against a plain FIFO worker that reorders one request at a
       time with pbrcm_reorder; both start from host buffers.  Reports
       throughput and p50/p99 latency (arrival -> result) per arrival rate.
"""
from __future__ import annotations

import json
import multiprocessing as mp
import os
import statistics
import sys
import threading
import time

import numpy as np

from . import gen


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def _make(spec):
    m = gen.make_from_spec(spec)
    return m.row_ptr, m.col_idx


def generate(specs, procs: int | None = None):
    """Generates the matrices of `specs` with a spawn-started process pool
    (started before any CUDA call)."""
    procs = procs or max(1, min(len(specs), (os.cpu_count() or 2) - 1, 64))
    if procs == 1 or len(specs) < 8:
        return [_make(s) for s in specs]
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        return pool.map(_make, specs, chunksize=max(1, len(specs) // (procs * 8)))


def _quantiles(v):
    v = sorted(v)
    if not v:
        return None, None
    q = lambda f: v[min(len(v) - 1, int(round(f * (len(v) - 1))))]  # noqa: E731
    return q(0.5), q(0.99)


def shard_by_nnz(nnz, parts: int):
    """Greedy longest-first assignment of matrices to `parts` GPUs by nnz
    (the batch shards by request, with no exchange between GPUs).  Returns
    one sorted index list per part."""
    load = [0] * parts
    out = [[] for _ in range(parts)]
    for i in sorted(range(len(nnz)), key=lambda k: (-int(nnz[k]), k)):
        p = min(range(parts), key=lambda q: (load[q], q))
        out[p].append(i)
        load[p] += int(nnz[i])
    return [sorted(x) for x in out]


def _max_over_ranks(ws, x: float) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_batch(args, ws, rank, local):
    import torch

    import parallelbatchrcm_b200 as P

    total = int(os.environ.get("PBRCM_BATCH_COUNT", "4096"))
    t0 = time.time()
    specs = gen.mixed_batch_specs(count=total, seed=42)
    if ws > 1:
        # every rank builds the same specs and reorders its own shard
        shard = shard_by_nnz([gen.spec_nnz_estimate(s) for s in specs], ws)[rank]
        specs = [specs[i] for i in shard]
    count = len(specs)
    mats = generate(specs)
    sum_n = sum(int(rp.shape[0] - 1) for rp, _ in mats)
    sum_nnz = sum(int(ci.shape[0]) for _, ci in mats)
    log(f"generated {count} matrices: sum n={sum_n} sum nnz={sum_nnz} in {time.time() - t0:.1f}s")
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    ctx = P.Context(local)
    stream = torch.cuda.Stream(device=dev)
    dmats = []
    for rp, ci in mats:
        dmats.append((torch.from_numpy(rp.view(np.int32)).to(dev), torch.from_numpy(ci.view(np.int32)).to(dev),
                      torch.empty(rp.shape[0] - 1, dtype=torch.int32, device=dev)))
    torch.cuda.synchronize()

    def batched():
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        res = P.reorder_batch_device(dmats, reverse=True, ctx=ctx, stream=stream)
        ev1.record(stream)
        ev1.synchronize()
        return ev0.elapsed_time(ev1), res

    for _ in range(args.warmup):
        batched()
    times = []
    for _ in range(args.steps):
        ms, res = batched()
        times.append(ms)
    assert all(r["status"] == 0 for r in res), [r for r in res if r["status"] != 0][:3]
    bperm = [p.cpu().numpy().copy() for _, _, p in dmats]
    batch_ms = statistics.median(times)

    # plain one-at-a-time: one team launch per matrix, same stream
    plain_perm = []
    tplain = 0.0
    lat = []
    for rp_d, ci_d, po in dmats:
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        P.reorder_device(rp_d, ci_d, po, reverse=True, ctx=ctx, stream=stream)
        ev1.record(stream)
        ev1.synchronize()
        lat.append(ev0.elapsed_time(ev1))
        tplain += lat[-1]
        plain_perm.append(po.cpu().numpy().copy())
    same = all(np.array_equal(a, b) for a, b in zip(bperm, plain_perm))

    # oracle sample
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
    import oracle as O
    rng = np.random.default_rng(0)
    sample = rng.choice(count, size=min(64, count), replace=False)
    oracle_ok = all(np.array_equal(bperm[i].view(np.uint32),
                                   O.full_reorder(mats[i][0], mats[i][1], reverse=True)["perm"]) for i in sample)

    # e2e from pinned host buffers through pbrcm_reorder_batch
    hm = [(torch.from_numpy(rp.view(np.int32)).pin_memory().numpy().view(np.uint32),
           torch.from_numpy(ci.view(np.int32)).pin_memory().numpy().view(np.uint32)) for rp, ci in mats]
    P.reorder_batch(hm, reverse=True, ctx=ctx)
    e2e = []
    for _ in range(max(1, args.steps // 2)):
        t1 = time.perf_counter()
        P.reorder_batch(hm, reverse=True, ctx=ctx)
        e2e.append(time.perf_counter() - t1)
    e2e_s = statistics.median(e2e)

    # several GPUs: each reorders its shard; the job takes as long as the
    # slowest shard
    batch_ms = _max_over_ranks(ws, batch_ms)
    tplain = _max_over_ranks(ws, tplain)
    e2e_s = _max_over_ranks(ws, e2e_s)
    if rank != 0:
        return 0
    value = total / (batch_ms / 1e3)
    plain_value = total / (tplain / 1e3)
    line = {
        "metric": "reorders/s (batched, many matrices, one persistent launch)", "value": value,
        "unit": "reorders/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": batch_ms, "higher_is_better": True, "scaling": "strong" if ws > 1 else "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded mixed grids / RGGs)",
        "config": {"workload": f"mixed_batch_{total}", "sum_n": sum_n, "sum_nnz": sum_nnz,
                   "l2": "inputs (GBs) larger than L2",
                   "sharding": "greedy by nnz across GPUs, no exchange" if ws > 1 else "one GPU"},
        "gnnz_per_s": sum_nnz / (batch_ms / 1e3) / 1e9,
        "plain_one_at_a_time": {"value": plain_value, "unit": "reorders/s", "total_ms": tplain,
                                "p50_ms": _quantiles(lat)[0], "p99_ms": _quantiles(lat)[1]},
        "speedup_vs_plain": value / plain_value,
        "batched_equals_plain": bool(same), "oracle_sample_ok": bool(oracle_ok), "oracle_sample": int(len(sample)),
        "e2e": {"value": total / e2e_s, "unit": "reorders/s",
                "h2d_bytes_per_step": int(sum(4 * (rp.shape[0] + ci.shape[0]) for rp, ci in mats)),
                "d2h_bytes_per_step": int(4 * sum_n)},
    }
    print(json.dumps(line), flush=True)
    return 0


def _serve_session(ctx, mats, arrivals, streams):
    import parallelbatchrcm_b200 as P

    sess = P.Session(ctx, streams=streams)
    n = len(mats)
    tick = [None] * n
    t_sub = [0.0] * n
    done_at = [None] * n
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
    pending = set(range(n))
    while pending:
        for i in list(pending):
            if tick[i] is None:
                continue
            out = sess.poll(tick[i])
            if out is not None:
                done_at[i] = time.perf_counter()
                assert out[1]["status"] == 0
                pending.discard(i)
        time.sleep(0.0002)
    th.join()
    lat = [(done_at[i] - (t0 + arrivals[i])) * 1e3 for i in range(n)]
    makespan = max(done_at) - t0
    sess.close()
    return lat, makespan


def _serve_plain(ctx, mats, arrivals):
    import parallelbatchrcm_b200 as P

    n = len(mats)
    done_at = [0.0] * n
    t0 = time.perf_counter() + 0.05
    for i in range(n):
        d = t0 + arrivals[i] - time.perf_counter()
        if d > 0:
            time.sleep(d)
        P.reorder(mats[i][0], mats[i][1], ctx=ctx)
        done_at[i] = time.perf_counter()
    lat = [(done_at[i] - (t0 + arrivals[i])) * 1e3 for i in range(n)]
    return lat, max(done_at) - t0


def run_serve(args, ws, rank, local):
    import torch

    import parallelbatchrcm_b200 as P

    count = int(os.environ.get("PBRCM_SERVE_COUNT", "256"))
    rates = [float(x) for x in os.environ.get("PBRCM_SERVE_RATES", "50,200,1000,100000").split(",")]
    stream_specs = gen.poisson_stream_specs(count, rate_per_s=1.0, seed=99)
    gaps = np.array([t for t, _ in stream_specs])  # arrival times at rate 1/s
    t0 = time.time()
    mats = generate([s for _, s in stream_specs])
    mats = [(rp, ci) for rp, ci in mats]
    log(f"generated {count} requests: sum n={sum(r.shape[0] - 1 for r, _ in mats)} in {time.time() - t0:.1f}s")
    torch.cuda.set_device(local)
    ctx = P.Context(local)
    # warm-up both paths
    _serve_session(ctx, mats[:16], [0.0] * 16, 96)
    for rp, ci in mats[:4]:
        P.reorder(rp, ci, ctx=ctx)
    rows = []
    for rate in rates:
        arr = list(gaps / rate)
        lat_s, span_s = _serve_session(ctx, mats, arr, 96)
        lat_p, span_p = _serve_plain(ctx, mats, arr)
        r = {"rate_per_s": rate,
             "session": {"reorders_per_s": count / span_s, "p50_ms": _quantiles(lat_s)[0],
                         "p99_ms": _quantiles(lat_s)[1]},
             "plain": {"reorders_per_s": count / span_p, "p50_ms": _quantiles(lat_p)[0],
                       "p99_ms": _quantiles(lat_p)[1]}}
        log(json.dumps(r))
        rows.append(r)
    best = rows[-1]
    line = {
        "metric": "reorders/s (serving, continuous batching, Poisson arrivals)",
        "value": best["session"]["reorders_per_s"], "unit": "reorders/s", "n_gpus": ws, "steps": len(rates),
        "warmup": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded Poisson stream of grids / RGGs, n in [1e3, 2e6])",
        "config": {"workload": f"serve_poisson_{count}", "rates": rates, "admission_cap_gb": 120},
        "sweep": rows,
        "speedup_vs_plain_at_max_rate": best["session"]["reorders_per_s"] / best["plain"]["reorders_per_s"],
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
        with open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                               "MEASURED_PEAKS.json")) as f:
            peak = float(json.load(f).get("hbm_gbs"))
    except (OSError, ValueError, TypeError):
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
        sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
        import oracle as O
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
        with open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                               "MEASURED_PEAKS.json")) as f:
            peak = float(json.load(f).get("hbm_gbs"))
    except (OSError, ValueError, TypeError):
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
        sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
        import oracle as O
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


def main(args, ws, rank, local):
    if args.workload == "wide":
        return run_wide(args, ws, rank, local)
    if args.workload == "connect":
        return run_connect(args, ws, rank, local)
    if args.workload == "permute":
        return run_permute(args, ws, rank, local)
    if args.workload == "batch":
        return run_batch(args, ws, rank, local)
    if args.workload == "serve":
        return run_serve(args, ws, rank, local)
    raise ValueError(args.workload)
