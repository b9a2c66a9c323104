"""Parity of the CUDA path (libpdgpu.so through its C ABI) with the CPU oracle.

Integer / index results (wrapped coordinates, image sets and records, cell
order, Verlet rows) must be bit-exact; floating-point sums within the stated
tolerances.  Each test names the reference test it mirrors.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

F32, F64 = np.float32, np.float64


@pytest.fixture(scope="module")
def pd():
    from openfpm_pdata_b200 import pd as _pd
    _pd.lib()
    return _pd


def make_vd(pd, pos, lo, hi, bc, ghost, dtype, props=()):
    vd = pd.VectorDist(pos.shape[0], lo, hi, bc, ghost, dtype=dtype, props=props)
    vd.hostToDevicePos(pos.astype(dtype))
    return vd


@pytest.mark.parametrize("dtype", [F32, F64])
def test_map_wrap_bit_exact(pd, orc, dtype):
    """map(RUN_ON_DEVICE) == periodic_l per periodic dimension (apply_bc_each_part)."""
    rng = np.random.default_rng(11)
    lo, hi = np.array([0.0, -1.0, 0.5]), np.array([1.0, 2.0, 3.0])
    bc = np.array([1, 1, 0], np.int32)
    L = hi - lo
    pos = (lo + rng.uniform(-0.4, 1.4, size=(5000, 3)) * L).astype(dtype)
    pos[:10, 0] = dtype(lo[0]) - dtype(1e-7)  # wraps to exactly hi -> round-off fix branch
    vd = make_vd(pd, pos, lo, hi, bc, 0.1, dtype)
    vd.map()
    got = vd.deviceToHostPos()
    exp = orc.wrap(pos, lo.astype(dtype), hi.astype(dtype), bc)
    assert np.array_equal(got.view(np.uint8), exp.view(np.uint8))


@pytest.mark.parametrize("dtype", [F32, F64])
@pytest.mark.parametrize("ghost", [0.05, 0.3])
def test_ghost_get_bit_exact(pd, orc, dtype, ghost):
    """ghost_get on one process: images, their order and (particle, shift) records
    equal the oracle's (vector_dist_gpu_unit_tests.cu:600-888 compares the image
    multiset bit-exact; here the GPU order itself is pinned)."""
    rng = np.random.default_rng(12)
    lo, hi, bc = np.zeros(3), np.ones(3), np.ones(3, np.int32)
    pos = orc.wrap(rng.random((20000, 3)).astype(dtype), lo.astype(dtype), hi.astype(dtype), bc)
    vd = make_vd(pd, pos, lo, hi, bc, ghost, dtype, props=[(pd.PD_F64, 1), (pd.PD_I32, 3)])
    p0 = rng.random(pos.shape[0])
    p1 = rng.integers(0, 1 << 30, size=(pos.shape[0], 3)).astype(np.int32)
    vd.hostToDeviceProp(0, p0)
    vd.hostToDeviceProp(1, p1)
    vd.ghost_get()
    img, src, shf = orc.ghost_get(pos, lo.astype(dtype), hi.astype(dtype), bc, dtype(ghost))
    n = pos.shape[0]
    assert vd.size_local() == n and vd.size_local_with_ghost() == n + img.shape[0]
    allp = vd.deviceToHostPos()
    assert np.array_equal(allp[:n], pos)
    assert np.array_equal(allp[n:].view(np.uint8), img.view(np.uint8))
    gsrc, gshf = vd.ghost_records()
    assert np.array_equal(gsrc, src) and np.array_equal(gshf, shf)
    assert np.array_equal(vd.deviceToHostProp(0)[n:], p0[src])
    assert np.array_equal(vd.deviceToHostProp(1)[n:], p1[src])
    # SKIP_LABELLING replay after a move: images follow their sources
    vd2 = make_vd(pd, pos, lo, hi, bc, ghost, dtype, props=[(pd.PD_F64, 1)])
    vd2.ghost_get()
    moved = (pos + dtype(1e-3)).astype(dtype)
    vd2.hostToDevicePos(moved)
    vd2.hostToDeviceProp(0, p0 * 2)
    vd2.ghost_get(props=[0], opt=pd.SKIP_LABELLING)
    sh = orc.shift_vectors(lo, hi, dtype=dtype)
    exp = (moved[src] - sh[shf]).astype(dtype)
    got = vd2.deviceToHostPos()[n:]
    assert np.array_equal(got, exp)
    assert np.array_equal(vd2.deviceToHostProp(0)[n:], (p0 * 2)[src])
    # NO_POSITION replay: properties only
    vd2.hostToDeviceProp(0, p0 * 3)
    vd2.ghost_get(props=[0], opt=pd.SKIP_LABELLING | pd.NO_POSITION)
    assert np.array_equal(vd2.deviceToHostPos()[n:], exp)
    assert np.array_equal(vd2.deviceToHostProp(0)[n:], (p0 * 3)[src])


def test_ghost_kernels_synthetic_boxes(pd, orc):
    """vector_ghost_process_local_particles (vector_dist_cuda_func_test.cu:19-389)."""
    rng = np.random.default_rng(13)
    pos = rng.random((10000, 3)).astype(F32)
    blo = np.zeros((4, 3))
    bhi = np.ones((4, 3))
    bhi[:, 0] = [0.5, 0.3, 0.2, 0.1]
    sv = np.arange(4, dtype=np.int32)
    vd = make_vd(pd, pos, np.zeros(3), np.ones(3), np.ones(3, np.int32), 0.1, F32,
                 props=[(pd.PD_F32, 1), (pd.PD_F32, 3), (pd.PD_F32, 9)])
    vd.hostToDeviceProp(0, np.arange(10000) + 12345.0)
    cnt = vd.ghost_count_boxes(blo, bhi, sv)
    x = pos[:, 0]
    expect = np.where(x >= 0.5, 0, np.where(x >= 0.3, 1, np.where(x >= 0.2, 2, np.where(x >= 0.1, 3, 4))))
    assert np.array_equal(cnt, expect)
    assert np.array_equal(cnt, orc.ghost_count(pos, blo.astype(F32), bhi.astype(F32), sv))
    shifts = np.zeros((4, 3))
    shifts[:, 0] = [10, 20, 30, 40]
    vd.ghost_get_boxes(blo, bhi, sv, shifts)
    img, src, shf = orc.ghost_images(pos, blo.astype(F32), bhi.astype(F32), sv, shifts.astype(F32))
    got = vd.deviceToHostPos()[10000:]
    assert np.array_equal(got, img)
    gsrc, gshf = vd.ghost_records()
    assert np.array_equal(gsrc, src) and np.array_equal(gshf, shf)
    assert np.array_equal(vd.deviceToHostProp(0)[10000:], np.arange(10000)[src] + 12345.0)


def _clustered(rng, n, L):
    c = rng.uniform(0, L, size=(8, 3))
    pos = c[rng.integers(0, 8, size=n)] + rng.normal(0, L / 20, size=(n, 3))
    return np.mod(pos, L)


@pytest.mark.parametrize("dtype", [F32, F64])
@pytest.mark.parametrize("layout", ["uniform", "clustered"])
def test_celllist_counting_sort_bit_exact(pd, orc, dtype, layout):
    """updateCellListGPU: cell_start and the in-cell order equal the oracle's
    stable counting sort (cell-order contract)."""
    rng = np.random.default_rng(14)
    L = 10.0
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    n = 30000
    pos = rng.uniform(0, L, size=(n, 3)) if layout == "uniform" else _clustered(rng, n, L)
    pos = orc.wrap(pos.astype(dtype), lo.astype(dtype), hi.astype(dtype), bc)
    vd = make_vd(pd, pos, lo, hi, bc, 0.7, dtype)
    vd.ghost_get()
    allp = vd.deviceToHostPos()
    cl = vd.getCellListGPU(0.7)
    vd.updateCellListGPU(cl)
    cs, so = cl.get()
    G = orc.cl_geometry(lo.astype(dtype), hi.astype(dtype), dtype(0.7), dtype(0.7), dtype=dtype)
    v = cl.view()
    assert list(v.div) == list(G.div) and v.ncells == G.ncells
    ecs, eso, _ = orc.cl_build(allp, G)
    assert np.array_equal(cs.astype(np.int64), ecs)
    assert np.array_equal(so, eso)


def test_celllist_reorder_restore(pd, orc):
    """vector_dist_gpu_make_sort (vector_dist_gpu_unit_tests.cu:425-567): CL_GPU_REORDER
    puts positions / properties in cell order, restoreOrder brings them back
    bit-exact, per-cell counts are unchanged."""
    rng = np.random.default_rng(15)
    lo, hi, bc = np.zeros(3), np.ones(3), np.zeros(3, np.int32)
    pos = rng.random((10000, 3)).astype(F32)
    vd = make_vd(pd, pos, lo, hi, bc, 0.1, F32, props=[(pd.PD_F32, 1), (pd.PD_F32, 3), (pd.PD_F32, 3)])
    vd.map()
    p0 = pos.sum(axis=1)
    p1 = np.stack([pos[:, 0] + pos[:, 1], pos[:, 0] + pos[:, 2], pos[:, 1] + pos[:, 2]], axis=1)
    vd.hostToDeviceProp(0, p0)
    vd.hostToDeviceProp(1, p1)
    vd.hostToDeviceProp(2, p1 * 2)
    cl = vd.getCellListGPU(0.1, pd.CL_NON_SYMMETRIC | pd.CL_GPU_REORDER)
    vd.updateCellListGPU(cl, props=[0, 1, 2])
    cs, so = cl.get()
    sp = vd.deviceToHostPos()
    assert np.array_equal(sp, pos[so])
    assert np.array_equal(vd.deviceToHostProp(1), p1[so])
    vd.restoreOrder(cl, props=[0, 1, 2])
    assert np.array_equal(vd.deviceToHostPos(), pos)
    assert np.array_equal(vd.deviceToHostProp(0), p0.astype(F32))
    assert np.array_equal(vd.deviceToHostProp(2), (p1 * 2).astype(F32))
    cl2 = vd.getCellListGPU(0.1)
    vd.updateCellListGPU(cl2)
    cs2, _ = cl2.get()
    assert np.array_equal(cs, cs2)


@pytest.mark.parametrize("sorted_", [False, True])
def test_celllist_force_functor(pd, orc, sorted_):
    """vector_dist_gpu_test[_sorted] (vector_dist_gpu_unit_tests.cu:259-423): the
    calculate_force functor on the GPU cell list equals the CPU walk within the
    reference's 3e-4 (FP32)."""
    rng = np.random.default_rng(55067)
    lo, hi, bc = np.zeros(3), np.ones(3), np.zeros(3, np.int32)
    pos = rng.random((10000, 3)).astype(F32)
    vd = make_vd(pd, pos, lo, hi, bc, 0.1, F32, props=[(pd.PD_F32, 1), (pd.PD_F32, 3), (pd.PD_F32, 3)])
    vd.map()
    vd.ghost_get()
    p0 = pos.sum(axis=1).astype(F32)
    vd.hostToDeviceProp(0, p0)
    opt = pd.CL_NON_SYMMETRIC | (pd.CL_GPU_REORDER if sorted_ else 0)
    cl = vd.getCellListGPU(0.1, opt)
    vd.updateCellListGPU(cl, props=[0])
    vd.test_force(cl, 0, 1, sorted=sorted_)
    if sorted_:
        vd.restoreOrder(cl, props=[1])
    got = vd.deviceToHostProp(1)[:10000]
    allp = vd.deviceToHostPos()
    G = orc.cl_geometry(lo.astype(F32), hi.astype(F32), F32(0.1), F32(0.1), dtype=F32)
    exp = orc.test_force(allp, np.concatenate([p0, np.zeros(allp.shape[0] - 10000, F32)]), 10000, G)
    assert np.max(np.abs(got - exp)) < 3e-4


@pytest.mark.parametrize("dtype", [F32, F64])
def test_verlet_bit_exact(pd, orc, dtype):
    """getVerlet: every row equals the oracle's (same order), which itself equals
    the brute-force sets (vector_dist_NN_tests.cpp:214-330)."""
    rng = np.random.default_rng(16)
    L = 12.0
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    pos = orc.wrap(rng.uniform(0, L, size=(20000, 3)).astype(dtype), lo.astype(dtype), hi.astype(dtype), bc)
    vd = make_vd(pd, pos, lo, hi, bc, 1.6, dtype)
    vd.ghost_get()
    vl = vd.getVerlet(1.6)
    off, idx = vl.get()
    allp = vd.deviceToHostPos()
    G = orc.cl_geometry(lo.astype(dtype), hi.astype(dtype), dtype(1.6), dtype(1.6), dtype=dtype, verlet=True)
    eoff, eidx = orc.verlet(allp, pos.shape[0], G, dtype(1.6))
    assert np.array_equal(off, eoff)
    assert np.array_equal(idx, eidx)


@pytest.mark.parametrize("ng", [10, 23])
def test_verlet_lattice_shells(pd, ng):
    """vector_dist_cell_verlet_test: 7 / 12 / 8 neighbours per shell on the GPU list."""
    sp = F32(1.0) / F32(ng)
    k = np.arange(ng)
    z, y, x = np.meshgrid(k, k, k, indexing="ij")
    pos = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1).astype(F32) * sp
    third = F32(np.sqrt(F32(3.0) * sp * sp))
    ghost = F32(third * F32(1.1))
    vd = make_vd(pd, pos, np.zeros(3), np.ones(3), np.ones(3, np.int32), float(ghost), F32)
    vd.map()
    vd.ghost_get()
    first = F32(sp + sp * F32(0.05))
    second = F32(np.sqrt(F32(2.0) * sp * sp))
    second = F32(second + second * F32(0.05))
    r = F32(third + third * F32(0.05))
    vl = vd.getVerlet(float(r))
    off, idx = vl.get()
    allp = vd.deviceToHostPos()
    n = pos.shape[0]
    assert off.shape[0] == n + 1
    for i in range(0, n, max(1, n // 300)):
        q = allp[idx[off[i]:off[i + 1]]]
        d = np.sqrt(((allp[i][None, :] - q) ** 2).sum(axis=1, dtype=F32)).astype(F32)
        assert (int((d <= first).sum()), int(((d > first) & (d <= second)).sum()), int((d > second).sum())) == (7, 12, 8)


def test_verlet_capacity_growth(pd, orc):
    """Rows longer than the first capacity estimate (dense clusters) are rebuilt
    with a larger capacity, still bit-exact."""
    rng = np.random.default_rng(17)
    L = 20.0
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    pos = np.concatenate([rng.uniform(0, L, size=(2000, 3)), 10 + rng.normal(0, 0.3, size=(3000, 3))])
    pos = orc.wrap(pos, lo, hi, bc)
    vd = make_vd(pd, pos, lo, hi, bc, 1.5, F64)
    vd.ghost_get()
    vl = vd.getVerlet(1.5)
    off, idx = vl.get()
    G = orc.cl_geometry(lo, hi, 1.5, 1.5, verlet=True)
    eoff, eidx = orc.verlet(vd.deviceToHostPos(), pos.shape[0], G, 1.5)
    assert np.diff(eoff).max() > 300
    assert np.array_equal(off, eoff) and np.array_equal(idx, eidx)


def test_lj_forces_fp64(pd, orc):
    """LJ forces, energy and virial from the GPU Verlet list and from the GPU cell
    list against the FP64 oracle: |dF| <= 1e-10 (|F| + F_rms), energies 1e-11 rel."""
    from openfpm_pdata_b200 import workloads
    x, v, L = workloads.lj_lattice(20, 1.1, 0.05, seed=3)
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    vd = make_vd(pd, x, lo, hi, bc, 2.8, F64, props=[(pd.PD_F64, 3)])
    vd.ghost_get()
    vl = vd.getVerlet(2.8)
    pe, vir = vd.lj_forces(0, vl=vl)
    f = vd.deviceToHostProp(0)[: x.shape[0]]
    allp = vd.deviceToHostPos()
    off, idx = vl.get()
    ef, epe, evir = orc.lj_verlet(allp, x.shape[0], off, idx)
    frms = np.sqrt((ef ** 2).sum(axis=1).mean())
    assert np.all(np.abs(f - ef) <= 1e-10 * (np.abs(ef) + frms))
    assert abs(pe - epe.sum()) <= 1e-11 * abs(epe.sum())
    assert abs(vir - evir.sum()) <= 1e-11 * abs(evir.sum())
    cl = vd.getCellListGPU(2.5)
    vd.updateCellListGPU(cl)
    pe2, vir2 = vd.lj_forces(0, cl=cl)
    f2 = vd.deviceToHostProp(0)[: x.shape[0]]
    assert np.all(np.abs(f2 - ef) <= 1e-10 * (np.abs(ef) + frms))
    assert abs(pe2 - epe.sum()) <= 1e-11 * abs(epe.sum())


@pytest.mark.parametrize("cell_list", [False, True])
def test_md_lj_matches_oracle(pd, orc, cell_list):
    """100 velocity-Verlet steps (10^3 lattice, spacing 1.1): per-step KE/PE/virial
    within 1e-9 relative of the FP64 oracle, final positions within 1e-8."""
    from openfpm_pdata_b200 import workloads
    x, v, L = workloads.lj_lattice(10, 1.1, 0.05, seed=9)
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    skin = 0.0 if cell_list else 0.3
    ghost = 2.5 + skin
    vd = make_vd(pd, x, lo, hi, bc, ghost, F64, props=[(pd.PD_F64, 3), (pd.PD_F64, 3)])
    vd.hostToDeviceProp(0, v)
    md = pd.MD(vd, 0, 1, dt=0.005, skin=skin, use_cell_list=cell_list)
    E = md.run(100)
    xo, vo, Eo = orc.md_lj(x, v, lo, hi, bc, ghost, 2.5, skin, 1.0, 1.0, 0.005, 1.0, 100)
    np.testing.assert_allclose(E[:, :3], Eo[1:, :3], rtol=1e-9, atol=1e-9)
    assert np.array_equal(E[:, 3], Eo[1:, 3])
    gid = vd.gid(with_ghost=False)
    xg = vd.deviceToHostPos(with_ghost=False)
    xr = xo[gid]
    d = xg - xr
    d -= L * np.round(d / L)
    assert np.max(np.abs(d)) < 1e-8
    b, s, err = md.stats()
    assert s == 100 and err == 0


@pytest.mark.parametrize("tx", [0, 1, 3, 8])
def test_md_tiled_rows_equal_oracle_sets(pd, orc, tx):
    """The driver's tile-local Verlet rows, translated to global indices, hold
    exactly the oracle's neighbour sets (d2 < (r_cut+skin)^2, self included)
    for the particles and images as stored after the build."""
    from openfpm_pdata_b200 import workloads
    x, v, L = workloads.lj_lattice(14, 1.1, 0.05, seed=31)
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    vd = make_vd(pd, x, lo, hi, bc, 2.8, F64, props=[(pd.PD_F64, 3), (pd.PD_F64, 3)])
    vd.hostToDeviceProp(0, v)
    md = pd.MD(vd, 0, 1, dt=0.005, skin=0.3)
    md.set_tiles(True, tx)
    md.run(0)
    off, idx, tiled = md.verlet()
    assert tiled
    allp = vd.deviceToHostPos()
    n = x.shape[0]
    G = orc.cl_geometry(lo, hi, 2.8, 2.8, verlet=True)
    eoff, eidx = orc.verlet(allp, n, G, 2.8)
    assert np.array_equal(np.diff(off), np.diff(eoff))
    for i in range(n):
        assert np.array_equal(np.sort(idx[off[i]:off[i + 1]]), np.sort(eidx[eoff[i]:eoff[i + 1]]))


@pytest.mark.parametrize("layout", ["uniform", "dense_half", "non_cubic", "wide_tiles"])
def test_md_tiled_rows_random_layouts(pd, orc, layout):
    """The same on layouts that are not lattices: uniform random positions (tile
    sizes fluctuate around the automatic width's target), a box whose left half
    is three times as dense as its right (tiles far above the mean take further
    sweeps of the layered build), a 48 x 30 x 21 box (axes of different cell
    counts), and tiles of 14 cells (about 290 domain particles each: more than
    one sweep of two particles a thread takes)."""
    rng = np.random.default_rng({"uniform": 41, "dense_half": 42, "non_cubic": 43, "wide_tiles": 44}[layout])
    L, n = 40.0, 60000
    box = np.array([48.0, 30.0, 21.0]) if layout == "non_cubic" else np.full(3, L)
    if layout == "dense_half":
        k = 3 * n // 4
        x = np.concatenate([rng.uniform([0, 0, 0], [L / 2, L, L], size=(k, 3)),
                            rng.uniform([L / 2, 0, 0], [L, L, L], size=(n - k, 3))])
    else:
        x = rng.uniform(0.0, 1.0, size=(n, 3)) * box
    lo, hi, bc = np.zeros(3), box.copy(), np.ones(3, np.int32)
    vd = make_vd(pd, x, lo, hi, bc, 2.8, F64, props=[(pd.PD_F64, 3), (pd.PD_F64, 3)])
    vd.hostToDeviceProp(0, np.zeros((n, 3)))
    md = pd.MD(vd, 0, 1, dt=0.005, skin=0.3)
    md.set_tiles(True, 14 if layout == "wide_tiles" else 0)
    md.run(0)
    off, idx, tiled = md.verlet()
    assert tiled
    allp = vd.deviceToHostPos()
    G = orc.cl_geometry(lo, hi, 2.8, 2.8, verlet=True)
    eoff, eidx = orc.verlet(allp, n, G, 2.8)
    assert np.array_equal(np.diff(off), np.diff(eoff))
    for i in range(n):
        assert np.array_equal(np.sort(idx[off[i]:off[i + 1]]), np.sort(eidx[eoff[i]:eoff[i + 1]]))


def test_md_tiled_equals_global_rows(pd):
    """Tiled shared-memory rows and global-index rows give the same trajectory
    energies (different summation order only)."""
    from openfpm_pdata_b200 import workloads
    x, v, L = workloads.lj_lattice(16, 1.1, 0.05, seed=32)
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    out = []
    for tiles in (True, False):
        vd = make_vd(pd, x, lo, hi, bc, 2.8, F64, props=[(pd.PD_F64, 3), (pd.PD_F64, 3)])
        vd.hostToDeviceProp(0, v)
        md = pd.MD(vd, 0, 1, dt=0.005, skin=0.3)
        md.set_tiles(tiles)
        out.append(md.run(40))
        assert md.verlet()[2] == tiles
    np.testing.assert_allclose(out[0][:, :3], out[1][:, :3], rtol=1e-10, atol=1e-10)
    assert np.array_equal(out[0][:, 3], out[1][:, 3])


def test_md_cell_list_both_paths(pd, orc):
    """Cell list every step: a small system runs in one thread-block cluster, a system
    above 65,536 particles through the captured step graph; both follow the FP64
    oracle (per-step energies within 1e-9, positions within 1e-8)."""
    from openfpm_pdata_b200 import workloads
    for side, steps in ((12, 30), (42, 6)):
        x, v, L = workloads.lj_lattice(side, 1.1, 0.05, seed=11)
        lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
        vd = make_vd(pd, x, lo, hi, bc, 2.5, F64, props=[(pd.PD_F64, 3), (pd.PD_F64, 3)])
        vd.hostToDeviceProp(0, v)
        md = pd.MD(vd, 0, 1, dt=0.005, skin=0.0, use_cell_list=True)
        E = md.run(steps)
        xo, vo, Eo = orc.md_lj(x, v, lo, hi, bc, 2.5, 2.5, 0.0, 1.0, 1.0, 0.005, 1.0, steps)
        np.testing.assert_allclose(E[:, :3], Eo[1:, :3], rtol=1e-9, atol=1e-9)
        gid = vd.gid(with_ghost=False)
        d = vd.deviceToHostPos(with_ghost=False) - xo[gid]
        d -= L * np.round(d / L)
        assert np.max(np.abs(d)) < 1e-8, (side, np.max(np.abs(d)))


@pytest.mark.parametrize("cell_list", [False, True])
def test_md_fp32_storage_follows_oracle(pd, orc, cell_list):
    """A vector with FP32 positions and FP32 properties through the tiled Verlet path
    and the cell-list path: 20 steps stay within FP32 accuracy of the FP64 oracle
    (per-step total energy within 1e-4 relative, positions within 1e-4)."""
    from openfpm_pdata_b200 import workloads
    x, v, L = workloads.lj_lattice(10, 1.1, 0.05, seed=13)
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    skin = 0.0 if cell_list else 0.3
    vd = make_vd(pd, x.astype(F32), lo, hi, bc, 2.5 + skin, F32, props=[(pd.PD_F32, 3), (pd.PD_F32, 3)])
    vd.hostToDeviceProp(0, v.astype(F32))
    md = pd.MD(vd, 0, 1, dt=0.005, skin=skin, use_cell_list=cell_list)
    E = md.run(20)
    xo, vo, Eo = orc.md_lj(x.astype(F32).astype(np.float64), v.astype(F32).astype(np.float64), lo, hi, bc,
                           2.5 + skin, 2.5, skin, 1.0, 1.0, 0.005, 1.0, 20)
    tot, toto = E[:, 0] + E[:, 1], Eo[1:, 0] + Eo[1:, 1]
    assert np.max(np.abs(tot - toto) / np.abs(toto)) < 1e-4
    gid = vd.gid(with_ghost=False)
    d = vd.deviceToHostPos(with_ghost=False).astype(np.float64) - xo[gid]
    d -= L * np.round(d / L)
    assert np.max(np.abs(d)) < 1e-4


def test_md_cell_list_graph_recaptured_after_growth(pd):
    """The cell-list step graph holds raw buffer addresses: a second, longer run
    (its energy buffer grows) makes the driver capture it again.  Runs of 3 + 10
    steps equal one run of 13 bit for bit."""
    from openfpm_pdata_b200 import workloads
    x, v, L = workloads.lj_lattice(42, 1.1, 0.05, seed=17)
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    out = []
    for split in (True, False):
        vd = make_vd(pd, x, lo, hi, bc, 2.5, F64, props=[(pd.PD_F64, 3), (pd.PD_F64, 3)])
        vd.hostToDeviceProp(0, v)
        md = pd.MD(vd, 0, 1, dt=0.005, skin=0.0, use_cell_list=True)
        if split:
            E = np.concatenate([md.run(3), md.run(10)])
        else:
            E = md.run(13)
        out.append(E)
        gid = vd.gid(with_ghost=False)
        xs = np.zeros_like(x)
        xs[gid] = vd.deviceToHostPos(with_ghost=False)
        out.append(xs)
    assert np.array_equal(out[0], out[2])
    assert np.array_equal(out[1], out[3])


def test_md_one_run_equals_runs_of_one_step(pd):
    """A run of 24 steps -- whose pair kernels also make the next step's kick and drift
    -- leaves the same positions and velocities, bit for bit, the same rebuild steps and
    the same energies as 24 runs of one step each (separate kick and drift kernels)."""
    from openfpm_pdata_b200 import workloads
    x, v, L = workloads.lj_lattice(20, 1.1, 0.05, seed=33)
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    out = []
    for split in (False, True):
        vd = make_vd(pd, x, lo, hi, bc, 2.8, F64, props=[(pd.PD_F64, 3), (pd.PD_F64, 3)])
        vd.hostToDeviceProp(0, v)
        md = pd.MD(vd, 0, 1, dt=0.005, skin=0.3)
        E = np.concatenate([md.run(1) for _ in range(24)]) if split else md.run(24)
        pos = vd.deviceToHostPos(with_ghost=False)
        vel = vd.deviceToHostProp(0, with_ghost=False)
        out.append((E, pos, vel, md.stats()[0]))
    (E0, p0, v0, b0), (E1, p1, v1, b1) = out
    assert b0 == b1 and b0 >= 3  # rebuilds inside the run
    np.testing.assert_array_equal(E0[:, 3], E1[:, 3])
    np.testing.assert_array_equal(p0, p1)
    np.testing.assert_array_equal(v0, v1)
    np.testing.assert_allclose(E0[:, 1:3], E1[:, 1:3], rtol=1e-13, atol=1e-9)
    np.testing.assert_allclose(E0[:, 0], E1[:, 0], rtol=1e-12)
