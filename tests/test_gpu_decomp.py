"""Slab decomposition through the library (pd_slab_* in openfpm_pdata_b200/csrc/pd_slab.cu).

Ranks are gloo processes on the host sharing the one GPU of this run: the library
labels, packs and unpacks on the device, gloo moves the packed bytes.  The
kernels of the ranks never wait on each other.  Checked for 2 and 3 slabs,
periodic and non-periodic split axis:
* map: every particle ends on the rank owning it, with its properties (an int32
  id travels as int32, exactly);
* ghost_get: each rank's ghost layer (its periodic images plus the halo from the
  neighbouring slabs) is exactly the multiset of periodic copies of the system
  that lie outside its slab and within the ghost of it (the reference's periodic
  ghost invariants, Vector/tests/vector_dist_unit_test.cpp:631-735, made exact);
* forces: the ranks' LJ forces together equal the single-system library forces
  within 1e-10 of (|F| + F_rms);
* dynamics: 8 velocity-Verlet steps with map and ghost_get every step follow the
  FP64 oracle's trajectory within 1e-9.
"""
import itertools
import os
import socket
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RC = 2.5


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _system(nside, seed):
    sys.path.insert(0, ROOT)
    from openfpm_pdata_b200 import workloads
    return workloads.lj_lattice(nside, 1.1, 0.05, seed=seed)


def _rank(rank, world, port, nside, bc, task, q):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    sys.path.insert(0, ROOT)
    from openfpm_pdata_b200 import pd
    from openfpm_pdata_b200.decomp import DistVector, SlabDecomposition, lj_forces_distributed, md_distributed
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        x, v, L = _system(nside, 5)
        n = x.shape[0]
        dec = SlabDecomposition(np.zeros(3), np.full(3, L), bc, RC, world, axis=0)
        # props: 0 id (int32), 1 velocity, 2 force
        dv = DistVector(dec, props=[(pd.PD_I32, 1), (pd.PD_F64, 3), (pd.PD_F64, 3)])
        if rank == 0:  # rank 0 holds the whole system at first, the others nothing
            dv.vd.resize(n)
            dv.vd.hostToDevicePos(x)
            dv.vd.hostToDeviceProp(0, np.arange(n, dtype=np.int32))
            dv.vd.hostToDeviceProp(1, v)
        dv.map()
        ids = dv.vd.deviceToHostProp(0, with_ghost=False)
        xl = dv.vd.deviceToHostPos(with_ghost=False)
        if task == "exchange":
            lj_forces_distributed(dv, 2, r_cut=RC, ghost_props=[0])
            f = dv.vd.deviceToHostProp(2, with_ghost=False)
            ghosts = dv.vd.deviceToHostPos()[xl.shape[0]:]
            q.put((rank, ids, xl, f, ghosts))
        else:
            md_distributed(dv, 8, 1, 2, dt=0.005, r_cut=RC)
            q.put((rank, dv.vd.deviceToHostProp(0, with_ghost=False), dv.vd.deviceToHostPos(with_ghost=False)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _run(world, nside, bc, task):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, nside, bc, task, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=600) for _ in range(world)), key=lambda t: t[0])
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    return out


def _copies_in(x, L, bc, lo_a, hi_a, g):
    """The periodic copies of x (shifts of -L, 0, L along the periodic axes) outside the
    slab [lo_a, hi_a) x box and inside it enlarged by g (axis 0 is the split axis)."""
    out = []
    shifts = [np.array(s) for s in itertools.product(*[(-1, 0, 1) if b else (0,) for b in bc])]
    for s in shifts:
        y = x + s * L
        inside_big = (y[:, 0] >= lo_a - g) & (y[:, 0] < hi_a + g)
        inside = (y[:, 0] >= lo_a) & (y[:, 0] < hi_a)
        for d in (1, 2):
            inside_big &= (y[:, d] >= -g) & (y[:, d] < L + g)
            inside &= (y[:, d] >= 0) & (y[:, d] < L)
        out.append(y[inside_big & ~inside])
    return np.concatenate(out)


def _sorted_rows(a):
    return a[np.lexsort(a.T[::-1])]


@pytest.mark.parametrize("world,bc", [(2, (1, 1, 1)), (3, (1, 1, 1)), (3, (0, 1, 1))])
def test_decomposed_map_ghost_and_forces(world, bc):
    sys.path.insert(0, ROOT)
    from openfpm_pdata_b200 import pd
    nside = 20
    x, _, L = _system(nside, 5)
    n = x.shape[0]
    out = _run(world, nside, bc, "exchange")
    ids = np.concatenate([o[1] for o in out])
    assert np.array_equal(np.sort(ids), np.arange(n))  # every particle once, its int32 id exact
    w = L / world
    f = np.full((n, 3), np.nan)
    for r, idl, xl, fl, gh in out:
        # map: owned particles are the system's (wrapped) positions in this slab
        assert np.array_equal(xl, x[idl])
        assert np.all((xl[:, 0] >= r * w) & (xl[:, 0] < (r + 1) * w if r < world - 1 else xl[:, 0] <= L))
        # ghost layer: exactly the periodic copies around the slab
        exp = _copies_in(x, L, bc, r * w, (r + 1) * w if r < world - 1 else L, RC)
        assert gh.shape == exp.shape
        assert np.array_equal(_sorted_rows(gh), _sorted_rows(exp))
        f[idl] = fl
    # forces equal the whole system's from the library
    lo, hi = np.zeros(3), np.full(3, L)
    vd = pd.VectorDist(n, lo, hi, np.asarray(bc, np.int32), RC, dtype=np.float64, props=[(pd.PD_F64, 3)])
    vd.hostToDevicePos(x)
    vd.ghost_get()
    cl = vd.getCellListGPU(RC)
    vd.updateCellListGPU(cl)
    vd.lj_forces(0, cl=cl, r_cut=RC)
    fw = vd.deviceToHostProp(0, with_ghost=False)
    frms = np.sqrt((fw ** 2).sum(axis=1).mean())
    assert np.all(np.abs(f - fw) <= 1e-10 * (np.abs(fw) + frms))


def test_decomposed_md_follows_oracle(orc):
    world, nside = 2, 16
    x, v, L = _system(nside, 5)
    out = _run(world, nside, (1, 1, 1), "md")
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    xo, _, _ = orc.md_lj(x, v, lo, hi, bc, RC, RC, 0.0, 1.0, 1.0, 0.005, 1.0, 8)
    for _, idl, xl in out:
        d = xl - xo[idl]
        d -= L * np.round(d / L)
        assert np.max(np.abs(d)) < 1e-9


def test_library_reads_and_writes_cuda_tensors():
    """The copies of the C ABI take device pointers: positions and properties from
    CUDA tensors (kept on the GPU) give the forces of host arrays, bit for bit."""
    import torch
    sys.path.insert(0, ROOT)
    from openfpm_pdata_b200 import pd
    x, v, L = _system(14, 23)
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    out = []
    for dev in (False, True):
        vd = pd.VectorDist(x.shape[0], lo, hi, bc, RC, dtype=np.float64, props=[(pd.PD_F64, 3), (pd.PD_F64, 3)])
        vd.hostToDevicePos(torch.from_numpy(x).cuda() if dev else x)
        vd.hostToDeviceProp(1, torch.from_numpy(v).cuda() if dev else v)
        vd.ghost_get()
        cl = vd.getCellListGPU(RC)
        vd.updateCellListGPU(cl)
        vd.lj_forces(0, cl=cl, r_cut=RC)
        f = vd.deviceToHostProp(0, with_ghost=False, device=dev)
        assert not dev or f.is_cuda
        vv = vd.deviceToHostProp(1, with_ghost=False, device=dev)
        xx = vd.deviceToHostPos(with_ghost=False, device=dev)
        out.append([t.cpu().numpy() if dev else t for t in (f, vv, xx)])
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


def test_slab_halo_kernel_equals_masks():
    """pd_slab_halo (the standalone halo selection) gives the indices of the numpy
    masks in ascending order; positions in host memory are refused."""
    import torch
    sys.path.insert(0, ROOT)
    from openfpm_pdata_b200 import pd
    rng = np.random.default_rng(4)
    x = rng.uniform(0, 30.0, size=(200000, 3))
    xg = torch.from_numpy(x).cuda()
    for axis, lo_thr, hi_thr in ((1, 12.5, 17.5), (0, 2.5, 27.5)):
        a, b = pd.slab_halo(xg, axis, lo_thr, hi_thr)
        assert np.array_equal(a.cpu().numpy(), np.nonzero(x[:, axis] < lo_thr)[0])
        assert np.array_equal(b.cpu().numpy(), np.nonzero(x[:, axis] >= hi_thr)[0])
    n0, n1 = pd.ctypes.c_long(0), pd.ctypes.c_long(0)
    rc = pd.lib().pd_slab_halo(x.ctypes.data_as(pd.ctypes.c_void_p), x.shape[0], 0, 1.0, 2.0, None, None,
                               pd.ctypes.byref(n0), pd.ctypes.byref(n1), None)
    assert rc == -1  # PD_EINVAL
