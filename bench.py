#!/usr/bin/env python3
"""Benchmark of the B200 RCM engine (one JSON line on rank 0).

Workload (default): one full reorder of the 128^3 7-point Laplacian pattern
(n = 2,097,152, nnz = 14,581,760, labels shuffled with numpy
default_rng(12345)): pseudo-peripheral start search + Cuthill-McKee pass +
reverse + bandwidth/profile, all in one persistent cooperative launch.

  value  reorders/s with the CSR already in HBM (pbrcm_reorder_device),
         device time of each step from CUDA events on the launching stream,
         L2 flushed (256 MiB write) between steps outside the timed events
  e2e    reorders/s through the public host C ABI (pbrcm_reorder) from
         pinned host buffers: H2D of the CSR and D2H of the permutation and
         result inside every step
  roofline  the team kernel's algorithmic bytes per launch / its CUDA-event
         duration, against MEASURED_PEAKS.json hbm_gbs
  cpu_baseline  the reference's own CPU code (oracle/_ref: findPeripheral +
         RealCPU::rcm<true>, CPU_BATCH on all host threads) on one reorder

--impl reference times the reference's CPU implementation alone on the same
workload (rank 0; other ranks exit 0).  Under torchrun each rank runs an
independent replica (the single-matrix path does not shard); value is the
sum over ranks of reorders / the max over ranks of the timed time.

--workload batch|serve|permute|connect|wide run the many-matrix, serving,
P A P^T, connectivity-repair and wide-graph benchmarks instead
(see parallelbatchrcm_b200/workloads.py).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX = NY = NZ = 128
SEED = 12345


def log(*a):
    print(*a, file=sys.stderr, flush=True)


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
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
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
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic():
    """dram__bytes_read.sum + dram__bytes_write.sum of one team-kernel launch on
    this workload, from the committed ncu summary
    (profiles/k_reorder_team_grid3d_128.md), or None."""
    p = os.path.join(ROOT, "profiles", "k_reorder_team_grid3d_128.md")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            if line.startswith("traffic_bytes_per_launch:"):
                return int(line.split(":")[1])
    return None


def algorithmic_bytes(n: int, nnz: int, passes: int) -> int:
    """Algorithmic bytes of one full reorder: per ordered BFS pass (start
    search passes + the final pass) row_ptr 4(n+1) + col_idx 4 nnz + claim
    reset 4n + queue/permutation write 4n + inverse permutation 4n; plus the
    bandwidth pass row_ptr 4(n+1) + col_idx 4 nnz + inverse gathers 4 nnz +
    inverse build 8n."""
    per_pass = 4 * (n + 1) + 4 * nnz + 4 * n + 4 * n + 4 * n
    bw = 4 * (n + 1) + 8 * nnz + 8 * n
    return (passes + 1) * per_pass + bw


def cpu_reference(rp, ci, steps: int, threads: int, timeout: float = 600.0):
    """Times the reference's own CPU code (oracle/_ref/ref_rcm: findPeripheral +
    RealCPU::rcm<true>) if built, else the oracle port (peripheral + serial
    stable CM in C).  Returns (reorder_ms list, kind, cores, sample)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if O.ref_available():
        rows = O.ref_time(rp, ci, threads, steps, timeout=timeout)
        ms = [r["reorder_ms"] for r in rows]
        kind = "reference"
        sample = (f"{steps} full reorder(s) of the 128^3 grid: findPeripheral + RealCPU::rcm<STABLE> "
                  f"({'CPU_BATCH, batch 512' if threads > 1 else 'serial rcm_seq'}, mean of its 25 internal "
                  f"repetitions)")
    else:
        O.build()
        ms = []
        for _ in range(steps):
            t0 = time.perf_counter()
            O.full_reorder(rp, ci)
            ms.append((time.perf_counter() - t0) * 1e3)
        kind, threads = "port", 1
        sample = f"{steps} full reorder(s) of the 128^3 grid with the C oracle (serial)"
    return ms, kind, threads, sample


def run_reference_arm(args, ws, rank):
    if rank != 0:
        return 0
    from parallelbatchrcm_b200 import gen
    m = gen.grid3d(NX, NY, NZ, seed=SEED)
    threads = os.cpu_count() or 1
    if args.warmup > 0:  # one untimed reorder: each step takes seconds on the CPU
        cpu_reference(m.row_ptr, m.col_idx, 1, threads)
    ms, kind, cores, sample = cpu_reference(m.row_ptr, m.col_idx, args.steps, threads)
    t = sum(ms) / 1e3
    value = args.steps / t
    line = {
        "impl": "reference", "metric": "reorders/s (full reorder: start search + RCM + bandwidth)",
        "value": value, "unit": "reorders/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32", "data": "synthetic (seeded 128^3 7-point grid pattern, shuffled labels)",
        "config": {"workload": "grid3d_128^3_7pt_rcm", "n": m.n, "nnz": m.nnz, "l2": "inputs > L2 (CPU path)"},
        "gnnz_per_s": value * m.nnz / 1e9,
        "cpu_baseline": {"value": value, "unit": "reorders/s", "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": "reorders/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, ws, rank, local):
    import torch

    import parallelbatchrcm_b200 as P
    from parallelbatchrcm_b200 import _lib, gen

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    t0 = time.time()
    m = gen.grid3d(NX, NY, NZ, seed=SEED)
    log(f"[rank {rank}] generated {m.name} n={m.n} nnz={m.nnz} in {time.time() - t0:.1f}s")
    n, nnz = m.n, m.nnz
    ctx = P.Context(local)
    stream = torch.cuda.Stream(device=dev)
    rp_d = torch.from_numpy(m.row_ptr.view(np.int32)).to(dev)
    ci_d = torch.from_numpy(m.col_idx.view(np.int32)).to(dev)
    perm_d = torch.empty(n, dtype=torch.int32, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device=dev)

    def step_device():
        with torch.cuda.stream(stream):
            flush.zero_()
        _, res = P.reorder_device(rp_d, ci_d, perm_d, reverse=True, ctx=ctx, stream=stream)
        return res

    for _ in range(args.warmup):
        res = step_device()
    torch.cuda.synchronize()
    # correctness of what is timed: the permutation is a bijection
    pm = perm_d.cpu().numpy().astype(np.uint32)
    assert P.check_permutation(pm) == 0
    barrier(ws)
    torch.cuda.synchronize()
    dev_ms = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            res = step_device()
            dev_ms.append(res["device_ms"])
        torch.cuda.synchronize()
    barrier(ws)
    torch.cuda.synchronize()
    t_dev = max_over_ranks(ws, sum(dev_ms) / 1e3)
    value = ws * args.steps / t_dev
    passes = res["peripheral_passes"]

    # e2e through the host C ABI with pinned buffers
    rp_h = torch.from_numpy(m.row_ptr.view(np.int32)).pin_memory()
    ci_h = torch.from_numpy(m.col_idx.view(np.int32)).pin_memory()
    perm_h = torch.empty(n, dtype=torch.int32).pin_memory()
    rp_np, ci_np, perm_np = (x.numpy().view(np.uint32) for x in (rp_h, ci_h, perm_h))
    for _ in range(max(1, args.warmup)):
        P.reorder(rp_np, ci_np, ctx=ctx, perm_out=perm_np)
    barrier(ws)
    e2e_ms = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        stream.synchronize()
        t1 = time.perf_counter()
        _, r2 = P.reorder(rp_np, ci_np, ctx=ctx, perm_out=perm_np)
        e2e_ms.append((time.perf_counter() - t1) * 1e3)
    barrier(ws)
    t_e2e = max_over_ranks(ws, sum(e2e_ms) / 1e3)
    e2e_value = ws * args.steps / t_e2e
    assert np.array_equal(perm_np, pm), "e2e permutation differs from the device-path permutation"

    if rank != 0:
        return 0
    peak, peak_kind = measured_peak()
    abytes = algorithmic_bytes(n, nnz, passes)
    avg_s = statistics.mean(dev_ms) / 1e3
    achieved = abytes / avg_s / 1e9
    cpu = None
    if not args.no_cpu_baseline:
        try:
            ms, kind, cores, sample = cpu_reference(m.row_ptr, m.col_idx, 1, os.cpu_count() or 1)
            cpu = {"value": 1e3 / statistics.mean(ms), "unit": "reorders/s", "cores": cores, "kind": kind,
                   "sample": sample}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "reorders/s", "cores": 0, "kind": "unavailable", "sample": str(e)[:200]}
    line = {
        "metric": "reorders/s (full reorder: start search + RCM + bandwidth)",
        "value": value, "unit": "reorders/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_dev * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32", "data": "synthetic (seeded 128^3 7-point grid pattern, shuffled labels)",
        "config": {"workload": "grid3d_128^3_7pt_rcm", "n": n, "nnz": nnz, "reverse": True, "start": "auto",
                   "parallelism": f"replicas x{ws}", "l2": "flushed (256 MiB write) between steps",
                   "team": {"variant": _lib.lib_path().rsplit('/', 1)[-1]}},
        "gnnz_per_s": value * nnz / 1e9,
        "latency_ms": {"p50": statistics.median(dev_ms), "max": max(dev_ms)},
        "result": {"start": res["start_node"], "passes": passes, "ecc": res["eccentricity"],
                   "levels": res["levels"], "bandwidth": res["bandwidth"], "profile": res["profile"]},
        "e2e": {"value": e2e_value, "unit": "reorders/s", "h2d_bytes_per_step": 4 * (n + 1) + 4 * nnz,
                "d2h_bytes_per_step": 4 * n + 64, "ms_per_step": statistics.mean(e2e_ms)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": profile_traffic(), "peak_kind": peak_kind, "kernel": "k_reorder_team",
                     "algorithmic_bytes_per_launch": abytes},
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
        "gpu_launches": 2 * args.steps,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="single", choices=["single", "batch", "serve", "permute", "connect", "wide"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    ws, rank, local = dist_init()
    try:
        if args.impl == "reference":
            return run_reference_arm(args, ws, rank)
        if args.workload != "single":
            from parallelbatchrcm_b200 import workloads
            return workloads.main(args, ws, rank, local)
        return run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
