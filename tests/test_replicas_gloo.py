"""The multi-GPU form of the benchmark is independent replicas: every rank
runs the full workload, the job's time is the slowest rank's, and the
reported value is the sum over ranks.  These checks run the rank logic of
bench.py with two gloo ranks on the CPU (no GPU), and check that the
reference arm prints only on rank 0."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        local_ms = 100.0 + 50.0 * rank          # rank 1 is the slow one
        total = bench.max_over_ranks(local_ms, world)
        q.put((rank, total, bench.replica_value(world, 10, total)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_report_the_slowest_rank():
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, total, value in res:
        assert total == 150.0
        assert abs(value - 2 * 10 / 0.150) < 1e-9


def test_single_rank_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(12.5, 1) == 12.5
    assert bench.replica_value(1, 4, 2000.0) == 2.0


def test_reference_arm_prints_only_on_rank_zero():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "3"], capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
