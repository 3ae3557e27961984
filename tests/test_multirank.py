"""CPU: the N > 1 path of bench.py with two gloo ranks on 127.0.0.1 — every
rank times its own replica, the job's step time is the slowest rank's, and
the whole-job value counts every replica's work."""
import os
import socket
import sys
from datetime import timedelta

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench
    ms = bench.max_over_ranks(100.0 + 50.0 * rank, world, device="cpu")
    dist.barrier()
    q.put((rank, ms, bench.replica_gflops(10**9, ms, world)))
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_step():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [150.0, 150.0]
    # 2 replicas x 2e9 flops in 150 ms
    assert out[0][2] == pytest.approx(2 * 2e9 / 0.150 / 1e9)


def test_single_rank_is_unchanged():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(12.5, 1) == 12.5
    assert bench.replica_gflops(10**9, 1000.0, 1) == pytest.approx(2.0)
