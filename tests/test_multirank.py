"""The N > 1 path of bench.py on CPU: two ranks over gloo (127.0.0.1).

Replicas only: no data-path collective; the timed region's length is the max
over ranks and the value sums the replicas' work.
"""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        local_ms = [12.5, 20.0][rank]
        ms = bench.max_over_ranks(local_ms, dist, "cpu")
        value = bench.replica_value(world, 4096000, 10, ms)
        dist.barrier()
        q.put((rank, ms, value))
    finally:
        dist.destroy_process_group()


def test_two_replicas_max_time_and_summed_work():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms, value in out:
        assert ms == 20.0
        assert value == pytest.approx(2 * 4096000 * 10 / 0.020)


def test_single_rank_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.0, None, "cpu") == 3.0
    assert bench.replica_value(1, 100, 10, 1000.0) == pytest.approx(1000.0)
