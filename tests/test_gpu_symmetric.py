"""Symmetric (half) Verlet lists and ghost_put through the C ABI.

ghost_put<add_/max_/replace_> on one process (vector_dist.hpp:2304-2310 ->
vector_dist_comm.hpp:2086-2182) folds every ghost's value onto its source, the
ghosts of a source in image order: checked bit-exact against a sequential loop.

getVerletSym (vector_dist.hpp:1412-1416) keeps each interacting pair once.  The
tests mirror vector_dist_cell_list_tests.cpp:443-649 (vector_dist_symmetric_cell_list
/ _verlet_list): neighbour counts and neighbour id sets accumulated from the half
list, with the ghosts' share folded by ghost_put<add_>, equal those of the full
list; LJ forces from the half list plus ghost_put<add_> equal the full-list forces
within 1e-10 (|F| + F_rms), energy and virial within 1e-11 relative.
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


def _system(pd, orc, n, L, ghost, dtype, seed, props, bc=(1, 1, 1)):
    rng = np.random.default_rng(seed)
    lo, hi, bcv = np.zeros(3), np.full(3, L), np.asarray(bc, np.int32)
    pos = orc.wrap(rng.uniform(0, L, size=(n, 3)).astype(dtype), lo.astype(dtype), hi.astype(dtype), bcv)
    vd = pd.VectorDist(n, lo, hi, bcv, ghost, dtype=dtype, props=props)
    vd.hostToDevicePos(pos)
    vd.map()
    vd.ghost_get()
    return vd


@pytest.mark.parametrize("op", [1, 2, 3])
@pytest.mark.parametrize("ptype", ["f64", "f32", "i32", "i64"])
def test_ghost_put_bit_exact(pd, orc, op, ptype):
    t, npt = {"f64": (pd.PD_F64, F64), "f32": (pd.PD_F32, F32), "i32": (pd.PD_I32, np.int32),
              "i64": (pd.PD_I64, np.int64)}[ptype]
    vd = _system(pd, orc, 6007, 10.0, 1.3, F64, 31, props=[(t, 2), (pd.PD_F64, 1)])
    n, m = vd.size_local(), vd.size_local_with_ghost()
    src, _ = vd.ghost_records()
    assert m > n and np.bincount(src, minlength=n).max() >= 3  # corner particles have several images
    rng = np.random.default_rng(op * 7 + len(ptype))
    if np.issubdtype(npt, np.integer):
        a = rng.integers(-10**6, 10**6, size=(m, 2)).astype(npt)
    else:
        a = rng.normal(size=(m, 2)).astype(npt)
    b = rng.normal(size=m)
    vd.hostToDeviceProp(0, a)
    vd.hostToDeviceProp(1, b)
    vd.ghost_put([0], op=op)
    got = vd.deviceToHostProp(0)
    assert np.array_equal(got[:n], orc.ghost_put(a, n, src, op))
    assert np.array_equal(got[n:], a[n:])                      # ghosts keep their values
    assert np.array_equal(vd.deviceToHostProp(1), b)           # props outside the mask untouched


def test_ghost_put_needs_ghost_get(pd):
    vd = pd.VectorDist(100, np.zeros(3), np.ones(3), np.ones(3, np.int32), 0.1, dtype=F64, props=[(pd.PD_F64, 1)])
    vd.hostToDevicePos(np.random.default_rng(1).random((100, 3)))
    with pytest.raises(RuntimeError):
        vd.ghost_put([0])
    vd.map()
    vd.ghost_get()
    vd.ghost_put([0])
    with pytest.raises(RuntimeError):
        vd.ghost_put([0], op=7)


@pytest.mark.parametrize("dtype", [F32, F64])
@pytest.mark.parametrize("bc", [(1, 1, 1), (1, 0, 1)])
def test_verlet_sym_rows_are_filtered_full_rows(pd, orc, dtype, bc):
    """Each half row is the full row with the pairs the other side keeps removed
    (same order), and every full-list pair is kept exactly once."""
    r = 1.4
    vd = _system(pd, orc, 8000, 11.0, r, dtype, 41, props=[], bc=bc)
    n = vd.size_local()
    full = vd.getVerlet(r)
    half = vd.getVerletSym(r)
    off, idx = full.get()
    hoff, hidx = half.get()
    allp = vd.deviceToHostPos()
    eoff, eidx = orc.verlet_sym(allp, n, off, idx)
    assert np.array_equal(hoff, eoff)
    assert np.array_equal(hidx, eidx)
    # the full list holds each pair from both sides, plus p itself on row p
    assert off[-1] == 2 * hoff[-1] + n


@pytest.mark.parametrize("dtype", [F32, F64])
def test_verlet_sym_counts_and_ids_fold_to_full(pd, orc, dtype):
    """vector_dist_symmetric_verlet_list: per-particle neighbour count and sorted
    neighbour-id list accumulated from the half list (the partner's share on a
    ghost, folded with ghost_put<add_>) equal the full list's."""
    r = 1.5
    vd = _system(pd, orc, 6000, 9.0, r, dtype, 43, props=[(pd.PD_I32, 1)])
    n, m = vd.size_local(), vd.size_local_with_ghost()
    gid = vd.gid()
    src, _ = vd.ghost_records()
    owner = np.concatenate([np.arange(n), src]).astype(np.int64)  # domain index behind every slot
    full = vd.getVerlet(r)
    half = vd.getVerletSym(r)
    off, idx = full.get()
    hoff, hidx = half.get()
    # counts: the half-list kernel's view (row length on p, +1 on the partner slot)
    cnt = np.zeros(m, np.int32)
    cnt[:n] = np.diff(hoff)
    np.add.at(cnt, hidx, 1)
    vd.hostToDeviceProp(0, cnt)
    vd.ghost_put([0])
    folded = vd.deviceToHostProp(0)[:n]
    assert np.array_equal(folded, np.diff(off).astype(np.int32) - 1)  # the full row also holds p itself
    # id sets: the partner's global id on p, p's global id on the partner's owner
    ids_full = []
    for i in range(n):
        row = idx[off[i]:off[i + 1]]
        ids_full.append(sorted(gid[owner[row[row != i]]].tolist()))
    ids_half = [[] for _ in range(n)]
    for i in range(n):
        for q in hidx[hoff[i]:hoff[i + 1]]:
            ids_half[i].append(int(gid[owner[q]]))
            ids_half[owner[q]].append(int(gid[i]))
    assert all(sorted(ids_half[i]) == ids_full[i] for i in range(n))


def test_lj_sym_plus_ghost_put_equals_full(pd):
    """LJ forces from the half list (reactions on ghosts, folded by ghost_put<add_>)
    equal the full-list forces; energy and virial count each pair once."""
    from openfpm_pdata_b200 import workloads
    x, _, L = workloads.lj_lattice(16, 1.1, 0.05, seed=5)
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    vd = pd.VectorDist(x.shape[0], lo, hi, bc, 2.8, dtype=F64, props=[(pd.PD_F64, 3), (pd.PD_F64, 3)])
    vd.hostToDevicePos(x)
    vd.map()
    vd.ghost_get()
    n = vd.size_local()
    pe, vir = vd.lj_forces(0, vl=vd.getVerlet(2.8))
    ef = vd.deviceToHostProp(0)[:n]
    pe_s, vir_s = vd.lj_forces(1, vl=vd.getVerletSym(2.8))
    vd.ghost_put([1])
    f = vd.deviceToHostProp(1)[:n]
    frms = np.sqrt((ef ** 2).sum(axis=1).mean())
    assert np.all(np.abs(f - ef) <= 1e-10 * (np.abs(ef) + frms))
    assert abs(pe_s - pe) <= 1e-11 * abs(pe)
    assert abs(vir_s - vir) <= 1e-11 * abs(vir)
    # Newton's third law: the folded forces sum to zero
    assert np.all(np.abs(f.sum(axis=0)) <= 1e-9 * frms * n)


def test_lj_sym_narrow_box_two_images(pd):
    """A box narrower than twice the cutoff: a pair interacts directly and through
    a periodic image at once; the half list keeps each of those pairs once."""
    rng = np.random.default_rng(7)
    L = 4.5
    n = 150
    x = rng.uniform(0, L, size=(n, 3))
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    vd = pd.VectorDist(n, lo, hi, bc, 2.6, dtype=F64, props=[(pd.PD_F64, 3), (pd.PD_F64, 3)])
    vd.hostToDevicePos(x)
    vd.map()
    vd.ghost_get()
    nn = vd.size_local()
    pe, vir = vd.lj_forces(0, vl=vd.getVerlet(2.6), r_cut=2.5, sigma=0.6)
    ef = vd.deviceToHostProp(0)[:nn]
    pe_s, vir_s = vd.lj_forces(1, vl=vd.getVerletSym(2.6), r_cut=2.5, sigma=0.6)
    vd.ghost_put([1])
    f = vd.deviceToHostProp(1)[:nn]
    frms = np.sqrt((ef ** 2).sum(axis=1).mean())
    assert np.all(np.abs(f - ef) <= 1e-10 * (np.abs(ef) + frms))
    assert abs(pe_s - pe) <= 1e-11 * abs(pe) and abs(vir_s - vir) <= 1e-11 * abs(vir)


@pytest.mark.parametrize("dtype", [F32, F64])
def test_lj_cell_list_sym_plus_ghost_put_equals_full(pd, dtype):
    """vector_dist_symmetric_cell_list: LJ through getCellListSym (each pair once,
    the reaction on the partner) plus ghost_put<add_> equals LJ through the full
    cell list; FP64 within 1e-10 (|F| + F_rms), FP32 within 1e-4."""
    from openfpm_pdata_b200 import workloads
    x, _, L = workloads.lj_lattice(14, 1.1, 0.05, seed=9)
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    vd = pd.VectorDist(x.shape[0], lo, hi, bc, 2.5, dtype=dtype,
                       props=[(pd.PD_F64 if dtype == F64 else pd.PD_F32, 3)] * 2)
    vd.hostToDevicePos(x.astype(dtype))
    vd.map()
    vd.ghost_get()
    n = vd.size_local()
    cl = vd.getCellListGPU(2.5)
    vd.updateCellListGPU(cl)
    pe, vir = vd.lj_forces(0, cl=cl)
    ef = vd.deviceToHostProp(0)[:n].astype(F64)
    cs = vd.getCellListSym(2.5)
    vd.updateCellListGPU(cs)
    pe_s, vir_s = vd.lj_forces(1, cl=cs)
    vd.ghost_put([1])
    f = vd.deviceToHostProp(1)[:n].astype(F64)
    tol = 1e-10 if dtype == F64 else 1e-4
    frms = np.sqrt((ef ** 2).sum(axis=1).mean())
    assert np.all(np.abs(f - ef) <= tol * (np.abs(ef) + frms))
    assert abs(pe_s - pe) <= tol * abs(pe) and abs(vir_s - vir) <= tol * abs(vir)
