#!/usr/bin/env python3
"""Benchmark of the B200 RCM engine (one JSON line on rank 0).

Default workload (the metric's own configuration): 4,096 independent
matrices, n log-uniform in [500, 200,000] (40% 2-D grids, 30% 3-D grids, 30%
random geometric graphs, seed 42), reordered in one persistent launch.

  value     batched reorders/s, CSRs resident in HBM (pbrcm_reorder_batch_
            device), CUDA events on the launching stream over K steps after W
            warm-up steps; the inputs (4.5 GB) are larger than L2
  e2e       the same through pbrcm_reorder_batch from pinned host buffers:
            H2D of every CSR and D2H of every permutation inside each step
  plain_one_at_a_time   pbrcm_reorder_device per matrix on the same stream
  roofline  algorithmic bytes of every matrix's full reorder / the launch's
            event time, against MEASURED_PEAKS.json hbm_gbs
  serve     the serving session on a Poisson stream vs a plain FIFO worker
  grid3d_128  the single-matrix 128^3 grid (one cooperative launch)
  cpu_baseline  the reference's own findPeripheral + rcm_seq<true>
            (oracle/_ref) over the same matrices on every host thread

--impl reference times the reference's CPU implementation alone on the same
workload (rank 0; other ranks exit 0).  Under torchrun every rank reorders
its own 4,096 matrices (weak scaling; no exchange between GPUs); value is the
sum over ranks of reorders / the max over ranks of the timed time.

--workload single|batch|serve|permute|connect|wide run one part alone;
refgpu times the reference's own GPU_SIMPLE beside this engine, cpu the
reference's serial and CPU_BATCH paths on the single-matrix configurations,
small the shared-memory engine on small matrices (the 64^2 grid first) beside
the team engine and the reference's serial code (bench_workloads.py).
"""
from __future__ import annotations

import argparse
import os
import sys

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from bench_workloads import ClockSampler, barrier, dist_init, max_over_ranks, measured_peak  # noqa: E402,F401


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mixed",
                    choices=["mixed", "single", "batch", "serve", "permute", "connect", "wide", "refgpu", "cpu",
                             "small"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--lean", action="store_true",
                    help="batched launches only (no plain pass, e2e, serving, 128^3 grid or CPU legs): for profiling")
    args = ap.parse_args()
    ws, rank, local = dist_init()
    try:
        import bench_workloads
        return bench_workloads.main(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
