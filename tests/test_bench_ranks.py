"""The host side of `bench.py --gpus N` on CPU: replicas synchronise with a
barrier and report the slowest rank's time (max over ranks), the whole-job
throughput counts every rank's cells, and under torchrun only rank 0 runs
the reference arm.  Two gloo ranks stand in for two GPUs (the reductions
are the same calls on CPU tensors)."""
import os
import socket
import subprocess
import sys
from datetime import timedelta

import multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ops = bench.RankOps(dist, device="cpu")
        ops.barrier()
        slowest = ops.max(10.0 + 2.5 * rank)  # rank 1 is the slow one
        q.put((rank, slowest, bench.throughput(world, 64 * 64, 20, slowest)))
        ops.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_replicas_report_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r for r, _, _ in results] == [0, 1]
    assert all(m == 12.5 for _, m, _ in results)
    assert all(v == 2 * 64 * 64 * 20 / 12.5e-3 for _, _, v in results)


def test_one_process_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    ops = bench.RankOps(None)
    ops.barrier()
    assert ops.max(3.0) == 3.0
    assert bench.throughput(1, 100, 10, 1.0) == 1e6


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "3",
                          "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0
    assert out.stdout.strip() == ""
