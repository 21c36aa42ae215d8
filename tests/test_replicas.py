"""bench.py --gpus N runs N independent replicas: the aggregation over
ranks (max device time, summed edges) on world_size 2 with gloo, on CPU; and
the reference arm exits without work on ranks other than 0."""
import json
import os
import subprocess
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sys.path.insert(0, ROOT)
        import bench
        t, e = bench.reduce_over_ranks(1.5 + rank, 1000 * (rank + 1), dist, "cpu")
        q.put((rank, t, e))
    finally:
        dist.destroy_process_group()


def test_reduce_over_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 2000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, t, e in got:
        assert t == 2.5 and e == 3000.0  # slowest rank, all ranks' edges


def test_reduce_over_ranks_single_process():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_over_ranks(2.0, 10) == (2.0, 10.0)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "3"],
                       capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
