"""Slab decomposition of one system over ranks (openfpm_pdata_b200/decomp.py):
`map` puts every particle on the rank owning its position, `ghost_get` delivers
exactly the particles within the ghost of each slab (shifted across periodic
faces, `vector_dist_comm.hpp:1398-1596`), and the forces of the decomposed
system equal those of the whole system.

Ranks are gloo processes on the host (127.0.0.1).  The per-rank forces here
come from a brute-force pair sum over the periodic copies (the library itself
needs a GPU; tests/test_gpu_decomp.py runs the same decomposition with it).
"""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RC = 2.5


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def brute_lj(x, lo, hi, bc, r_cut=RC, eps=1.0, sigma=1.0):
    """LJ forces on every particle of x from all particles of x and their copies
    shifted by -1, 0, +1 box lengths along the periodic axes."""
    x = np.asarray(x, np.float64)
    L = np.asarray(hi, np.float64) - np.asarray(lo, np.float64)
    sh = [np.array([a, b, c], np.float64) * L
          for a in ((-1, 0, 1) if bc[0] else (0,))
          for b in ((-1, 0, 1) if bc[1] else (0,))
          for c in ((-1, 0, 1) if bc[2] else (0,))]
    f = np.zeros_like(x)
    s2 = sigma * sigma
    for s in sh:
        d = x[:, None, :] - (x[None, :, :] + s)
        r2 = (d * d).sum(axis=2)
        if not s.any():
            np.fill_diagonal(r2, np.inf)
        m = r2 < r_cut * r_cut
        r2s = np.where(m, r2, 1.0)
        sr6 = (s2 / r2s) ** 3
        fac = np.where(m, 24.0 * eps * (2.0 * sr6 * sr6 - sr6) / r2s, 0.0)
        f += (fac[:, :, None] * d).sum(axis=1)
    return f


def _system(nside, seed):
    sys.path.insert(0, ROOT)
    from openfpm_pdata_b200 import workloads
    return workloads.lj_lattice(nside, 1.1, 0.05, seed=seed)


def _rank(rank, world, port, nside, bc, q):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    sys.path.insert(0, ROOT)
    from openfpm_pdata_b200.decomp import DistParticles, SlabDecomposition, lj_forces_distributed
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        x, _, L = _system(nside, 5)
        n = x.shape[0]
        dec = SlabDecomposition(np.zeros(3), np.full(3, L), bc, RC, world, axis=0)
        dp = DistParticles(dec)
        # rank 0 holds the whole system at first, the others nothing
        xs = torch.from_numpy(x) if rank == 0 else torch.zeros((0, 3), dtype=torch.float64)
        gs = torch.arange(n, dtype=torch.int32) if rank == 0 else torch.zeros(0, dtype=torch.int32)
        xl, (gl,) = dp.map(xs, [gs])
        xh, (gh,) = dp.ghost_get(xl, [gl])
        f = lj_forces_distributed(dp, xl, force_fn=brute_lj)
        q.put((rank, gl.numpy(), xl.numpy(), f.numpy(), gh.numpy(), xh.numpy()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _run(world, nside, bc):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, nside, bc, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = []
    for _ in range(world):
        out.append(q.get(timeout=90))
    out.sort(key=lambda t: t[0])
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    return out


@pytest.mark.parametrize("world,bc", [(2, (1, 1, 1)), (3, (1, 1, 1)), (3, (0, 1, 1))])
def test_map_ghost_get_and_forces(world, bc):
    nside = 8
    x, _, L = _system(nside, 5)
    n = x.shape[0]
    sys.path.insert(0, ROOT)
    from openfpm_pdata_b200.decomp import SlabDecomposition
    dec = SlabDecomposition(np.zeros(3), np.full(3, L), bc, RC, world, axis=0)
    out = _run(world, nside, bc)
    # map: every particle on exactly one rank, the one whose slab holds it
    ids = np.concatenate([o[1] for o in out])
    assert np.array_equal(np.sort(ids), np.arange(n))
    for rank, gl, xl, _, _, _ in out:
        assert np.array_equal(xl, x[gl])
        assert np.all((xl[:, 0] >= dec.edges[rank]) & (xl[:, 0] < dec.edges[rank + 1]))
    # ghost_get: the halo of each slab is every particle (or its periodic copy along
    # the axis) within the ghost outside the slab
    for rank, _, _, _, gh, xh in out:
        lo, hi = dec.edges[rank] - RC, dec.edges[rank + 1] + RC
        want = []
        for s in ((-L, 0.0, L) if bc[0] else (0.0,)):
            xs = x[:, 0] + s
            inside = (xs >= dec.edges[rank]) & (xs < dec.edges[rank + 1])
            sel = np.nonzero((xs >= lo) & (xs < hi) & ~inside)[0]
            want += [(int(j), float(xs[j])) for j in sel]
        got = sorted((int(j), float(p)) for j, p in zip(gh, xh[:, 0]))
        assert got == sorted(want)
        assert np.array_equal(xh[:, 1:], x[gh][:, 1:])
    # forces of the decomposed system equal those of the whole system
    f = np.zeros((n, 3))
    for _, gl, _, fl, _, _ in out:
        f[gl] = fl
    fw = brute_lj(x, np.zeros(3), np.full(3, L), bc)
    frms = np.sqrt((fw ** 2).sum(axis=1).mean())
    assert np.max(np.abs(f - fw)) <= 1e-12 * frms


def _rank_md(rank, world, port, nside, steps, q):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    sys.path.insert(0, ROOT)
    from openfpm_pdata_b200.decomp import DistParticles, SlabDecomposition, md_distributed
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        from openfpm_pdata_b200 import workloads
        x, v, L = workloads.lj_lattice(nside, 1.1, 0.05, seed=9)
        n = x.shape[0]
        dp = DistParticles(SlabDecomposition(np.zeros(3), np.full(3, L), (1, 1, 1), RC, world, axis=0))
        xs = torch.from_numpy(x) if rank == 0 else torch.zeros((0, 3), dtype=torch.float64)
        vs = torch.from_numpy(v) if rank == 0 else torch.zeros((0, 3), dtype=torch.float64)
        gs = torch.arange(n, dtype=torch.int32) if rank == 0 else torch.zeros(0, dtype=torch.int32)
        xl, (vl, gl) = dp.map(xs, [vs, gs])
        xl, vl, (gl,) = md_distributed(dp, xl, vl, steps, props=[gl], force_fn=brute_lj)
        q.put((rank, gl.numpy(), xl.numpy(), vl.numpy()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_md_over_ranks_follows_the_whole_system():
    """Velocity Verlet with map and ghost_get every step on 2 ranks follows the
    same steps on the whole periodic system (positions within 1e-10)."""
    import torch.multiprocessing as mp
    nside, steps, world = 7, 8, 2
    x, v, L = _system_v(nside, 9)
    n = x.shape[0]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_md, args=(r, world, port, nside, steps, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    xd, vd = np.full((n, 3), np.nan), np.full((n, 3), np.nan)
    for _, gl, xl, vl in out:
        xd[gl], vd[gl] = xl, vl
    lo, hi, bc = np.zeros(3), np.full(3, L), (1, 1, 1)
    h = 0.5 * 0.005
    f = brute_lj(x, lo, hi, bc)
    for _ in range(steps):
        v = v + h * f
        x = x + 0.005 * v
        x = np.mod(x, L)
        f = brute_lj(x, lo, hi, bc)
        v = v + h * f
    d = xd - x
    d -= L * np.round(d / L)
    assert np.max(np.abs(d)) < 1e-10
    assert np.max(np.abs(vd - v)) < 1e-9


def _system_v(nside, seed):
    sys.path.insert(0, ROOT)
    from openfpm_pdata_b200 import workloads
    return workloads.lj_lattice(nside, 1.1, 0.05, seed=seed)


def test_slab_narrower_than_ghost_refused():
    sys.path.insert(0, ROOT)
    from openfpm_pdata_b200.decomp import SlabDecomposition
    with pytest.raises(ValueError):
        SlabDecomposition(np.zeros(3), np.full(3, 8.8), (1, 1, 1), RC, 4, axis=0)


def test_single_rank_is_the_whole_box():
    import torch
    sys.path.insert(0, ROOT)
    from openfpm_pdata_b200.decomp import DistParticles, SlabDecomposition
    x, _, L = _system(6, 7)
    dec = SlabDecomposition(np.zeros(3), np.full(3, L), (1, 1, 1), RC, 1)
    dp = DistParticles(dec)
    xl, _ = dp.map(torch.from_numpy(x))
    assert np.array_equal(xl.numpy(), x)
    xh, _ = dp.ghost_get(xl)
    assert xh.shape[0] == 0
    lo, hi, bc = dec.local_box(0)
    assert np.array_equal(bc, [1, 1, 1]) and hi[0] == L


def test_rows_pack_every_property_type_exactly():
    # positions and properties of any of the packed types and shapes travel as
    # float64 rows and come back bit for bit; other types are refused
    import torch
    sys.path.insert(0, ROOT)
    from openfpm_pdata_b200.decomp import _pack, _unpack
    rng = np.random.default_rng(3)
    n = 257
    x = torch.from_numpy(rng.normal(size=(n, 3)))
    props = [torch.from_numpy(rng.normal(size=n).astype(np.float32)),
             torch.from_numpy(rng.integers(-2 ** 31, 2 ** 31 - 1, size=(n, 2), dtype=np.int64).astype(np.int32)),
             torch.from_numpy(rng.normal(size=(n, 3, 3))),
             torch.zeros((n, 0), dtype=torch.float64)]
    rows, meta = _pack(x, props)
    assert rows.dtype == torch.float64 and rows.shape == (n, 3 + 1 + 2 + 9 + 0)
    x2, p2 = _unpack(rows, meta)
    assert torch.equal(x2, x)
    for a, b in zip(props, p2):
        assert a.dtype == b.dtype and a.shape == b.shape and torch.equal(a, b)
    x0, p0 = _unpack(_pack(x[:0], [p[:0] for p in props])[0], meta)
    assert x0.shape == (0, 3) and [p.shape[0] for p in p0] == [0, 0, 0, 0]
    with pytest.raises(TypeError):
        _pack(x, [torch.zeros(n, dtype=torch.int64)])
