"""Host logic of the slab decomposition (openfpm_pdata_b200/decomp.py), on CPU:
the slab geometry (edges, owners, each rank's box) and the transport of packed
rows between ranks, an all-to-all over gloo ranks on 127.0.0.1 (world 2 and 3):
every rank receives, in rank order, exactly the rows the others addressed to it.
The device half (labelling, packing, unpacking in the library) needs a GPU and
is tested in tests/test_gpu_decomp.py.
"""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_slab_geometry():
    sys.path.insert(0, ROOT)
    from openfpm_pdata_b200.decomp import SlabDecomposition
    dec = SlabDecomposition(np.zeros(3), np.array([30.0, 12.0, 12.0]), (1, 1, 0), 2.5, 3)
    assert dec.axis == 0 and dec.periodic and dec.width == 10.0
    assert np.allclose(dec.edges, [0, 10, 20, 30])
    x = np.array([[0.0, 1, 1], [9.999, 1, 1], [10.0, 1, 1], [29.99, 5, 5], [30.0, 5, 5]])
    assert dec.owner(x).tolist() == [0, 0, 1, 2, 2]
    lo, hi, bc = dec.local_box(1)
    assert lo.tolist() == [10, 0, 0] and hi.tolist() == [20, 12, 12] and bc.tolist() == [0, 1, 0]
    s = dec.slab_t()
    assert (s.axis, s.nslabs, s.periodic, s.lo, s.hi, s.ghost) == (0, 3, 1, 0.0, 30.0, 2.5)
    one = SlabDecomposition(np.zeros(3), np.full(3, 8.0), (1, 1, 1), 2.5, 1)
    assert one.local_box(0)[2].tolist() == [1, 1, 1]
    with pytest.raises(ValueError):
        SlabDecomposition(np.zeros(3), np.full(3, 8.0), (1, 1, 1), 2.5, 4)  # slabs narrower than the ghost


def _rank(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    sys.path.insert(0, ROOT)
    from openfpm_pdata_b200.decomp import exchange_rows
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        rb = 12  # rows of three int32: source rank, destination rank, row number
        counts = [(rank + 1) * (d + 2) % 5 for d in range(world)]
        rows = [np.array([rank, d, k], np.int32) for d in range(world) for k in range(counts[d])]
        send = torch.from_numpy(np.concatenate(rows).view(np.uint8).copy() if rows else np.zeros(0, np.uint8))
        recv, rc = exchange_rows(send, counts, rb)
        q.put((rank, rc, recv.numpy().view(np.int32).reshape(-1, 3).tolist()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_exchange_rows_all_to_all(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        r, rc, rows = q.get(timeout=120)
        out[r] = (rc, rows)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    for d in range(world):
        rc, rows = out[d]
        exp = [[s, d, k] for s in range(world) for k in range((s + 1) * (d + 2) % 5)]
        assert rc == [(s + 1) * (d + 2) % 5 for s in range(world)]
        assert rows == exp
