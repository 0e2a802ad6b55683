"""bench.py's multi-rank bookkeeping on CPU: world size 2 over gloo.

Each rank runs its own replica; the job's value is the steps of all ranks over
the slowest rank's time.  Run as two spawned processes on 127.0.0.1.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import bench
        steps = 10 + rank          # ranks may run different step counts
        ms = 100.0 * (rank + 1)    # rank 1 is the slow one
        value, slowest = bench.replica_throughput(world, steps, ms)
        q.put((rank, value, slowest, bench.max_over_ranks(world, rank), bench.sum_over_ranks(world, 1.0)))
    finally:
        dist.destroy_process_group()


def test_replica_throughput_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, value, slowest, mx, sm in res:
        assert slowest == pytest.approx(200.0)
        assert value == pytest.approx((10 + 11) / 0.2)
        assert mx == 1.0 and sm == 2.0


def test_single_rank_needs_no_process_group():
    import bench
    value, slowest = bench.replica_throughput(1, 5, 50.0)
    assert value == pytest.approx(100.0) and slowest == 50.0
