"""The multi-rank plumbing of bench.py on CPU: world_size 2 over gloo, as
torchrun launches it on a GPU node (one rank per GPU, 127.0.0.1 rendezvous).
One matrix does not shard, so the ranks are independent replicas; what they
share is the barrier around the timed region and the max over ranks of the
device time."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE="2",
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    ws, r, _ = bench.dist_init()
    bench.barrier(ws)
    m = bench.max_over_ranks(ws, 1.5 + r)
    out.put((r, ws, m, dist.get_backend()))
    dist.destroy_process_group()


def test_barrier_and_max_over_ranks_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == [(0, 2, 2.5, "gloo"), (1, 2, 2.5, "gloo")]


def test_reference_arm_under_torchrun_two_ranks():
    """`bench.py --impl reference` launched like the driver's N=2 run: rank 0
    alone times the reference's CPU code and prints one JSON line, the other
    rank exits 0 without work."""
    ref = os.path.join(ROOT, "oracle", "_ref", "ref_rcm")
    if not os.path.exists(ref):
        pytest.skip("reference CPU build not present (run the build first)")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"]
    env = dict(os.environ, PBRCM_BENCH_COUNT="48")  # a short stream: this checks the plumbing
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["e2e"]["h2d_bytes_per_step"] == 0


def test_batch_shards_by_nnz():
    sys.path.insert(0, ROOT)
    import bench_workloads as workloads
    from parallelbatchrcm_b200 import gen
    specs = gen.mixed_batch_specs(count=300, seed=42)
    est = [gen.spec_nnz_estimate(s) for s in specs]
    shards = workloads.shard_by_nnz(est, 3)
    assert sorted(i for s in shards for i in s) == list(range(300))
    loads = [sum(est[i] for i in s) for s in shards]
    assert max(loads) - min(loads) <= max(est)  # longest-first greedy bound
    # the estimate is close to the real count
    for s in specs[:20]:
        real = gen.make_from_spec(s).nnz
        assert 0.7 * real <= gen.spec_nnz_estimate(s) <= 1.4 * real, (s, real)
