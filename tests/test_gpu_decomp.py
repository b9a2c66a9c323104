"""Slab decomposition with the library computing each rank's forces on the GPU.

Two ranks (gloo processes on the host, exchanging host tensors) share the one
GPU of this run: each builds its extended slab (own particles, then the halo
from the neighbouring slabs) as a vector with the split axis non-periodic and
computes LJ forces with the library's cell list.  Their forces, put together,
equal the library's forces of the whole periodic system within 1e-10 of
(|F| + F_rms).  The kernels of the two ranks never wait on each other.
"""
import os
import socket
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, nside, q):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    sys.path.insert(0, ROOT)
    from openfpm_pdata_b200 import workloads
    from openfpm_pdata_b200.decomp import DistParticles, SlabDecomposition, lj_forces_distributed
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        x, _, L = workloads.lj_lattice(nside, 1.1, 0.05, seed=21)
        n = x.shape[0]
        dec = SlabDecomposition(np.zeros(3), np.full(3, L), (1, 1, 1), 2.5, world)
        dp = DistParticles(dec)
        xs = torch.from_numpy(x) if rank == 0 else torch.zeros((0, 3), dtype=torch.float64)
        gs = torch.arange(n, dtype=torch.int32) if rank == 0 else torch.zeros(0, dtype=torch.int32)
        xl, (gl,) = dp.map(xs, [gs])
        f = lj_forces_distributed(dp, xl)
        q.put((rank, gl.numpy(), f.numpy()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_decomposed_forces_equal_whole_system():
    import torch.multiprocessing as mp
    sys.path.insert(0, ROOT)
    from openfpm_pdata_b200 import workloads
    from openfpm_pdata_b200.decomp import lj_forces_library
    nside, world = 20, 2
    x, _, L = workloads.lj_lattice(nside, 1.1, 0.05, seed=21)
    n = x.shape[0]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, nside, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    f = np.full((n, 3), np.nan)
    for _, gl, fl in out:
        f[gl] = fl
    fw = lj_forces_library(x, np.zeros(3), np.full(3, L), (1, 1, 1))
    frms = np.sqrt((fw ** 2).sum(axis=1).mean())
    assert np.all(np.abs(f - fw) <= 1e-10 * (np.abs(fw) + frms))


def test_library_reads_and_writes_cuda_tensors():
    """The copies of the C ABI take device pointers: forces from a CUDA tensor
    of positions (kept on the GPU) equal those from the host array, bit for bit,
    and so do the one-rank decomposition's forces on CUDA tensors."""
    import torch
    sys.path.insert(0, ROOT)
    from openfpm_pdata_b200 import workloads
    from openfpm_pdata_b200.decomp import DistParticles, SlabDecomposition, lj_forces_distributed, lj_forces_library
    x, _, L = workloads.lj_lattice(14, 1.1, 0.05, seed=23)
    lo, hi = np.zeros(3), np.full(3, L)
    fh = lj_forces_library(x, lo, hi, (1, 1, 1))
    xt = torch.from_numpy(x).cuda()
    fd = lj_forces_library(xt, lo, hi, (1, 1, 1))
    assert fd.is_cuda and np.array_equal(fd.cpu().numpy(), fh)
    dp = DistParticles(SlabDecomposition(lo, hi, (1, 1, 1), 2.5, 1))
    xl, _ = dp.map(xt)
    f1 = lj_forces_distributed(dp, xl)
    assert f1.is_cuda and np.array_equal(f1.cpu().numpy(), fh)


def test_slab_halo_kernel_equals_masks():
    """The library's halo selection (pd_slab_halo) gives the indices of the
    tensor masks, in the same ascending order, for every rank of 2 and 3 slabs;
    positions in host memory are refused before any kernel runs."""
    import torch
    sys.path.insert(0, ROOT)
    from openfpm_pdata_b200 import pd
    from openfpm_pdata_b200.decomp import SlabDecomposition
    rng = np.random.default_rng(4)
    L = 30.0
    x = rng.uniform(0, L, size=(200000, 3))
    xc, xg = torch.from_numpy(x), torch.from_numpy(x).cuda()
    for P in (2, 3):
        dec = SlabDecomposition(np.zeros(3), np.full(3, L), (1, 1, 1), 2.5, P, axis=1)
        for r in range(P):
            host = dec.halo_sends(r, xc)
            dev = dec.halo_sends(r, xg)
            assert [(d, s) for d, _, s in host] == [(d, s) for d, _, s in dev]
            for (_, ih, _), (_, idv, _) in zip(host, dev):
                assert idv.is_cuda and torch.equal(ih, idv.cpu())
    n0, n1 = pd.ctypes.c_long(0), pd.ctypes.c_long(0)
    rc = pd.lib().pd_slab_halo(x.ctypes.data_as(pd.ctypes.c_void_p), x.shape[0], 0, 1.0, 2.0, None, None,
                               pd.ctypes.byref(n0), pd.ctypes.byref(n1), None)
    assert rc == -1  # PD_EINVAL
