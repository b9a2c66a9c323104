"""Stream compaction through the C ABI: remove_marked and get_indexes_by_type.

remove_marked<prp> (vector_dist_cuda_funcs.cuh:333-412) mirrors
vector_dist_cuda_func_test.cu:945-1088 (vector_dist_remove_marked_type<0..3>);
get_indexes_by_type (:449-481) mirrors vector_dist_gpu_unit_tests.cu:1626-1694
(vector_dist_get_index_set).  Positions, global ids, every property and the
destroyed mark must equal the oracle's bit for bit.
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


def _vd(pd, orc, n, props, seed, dtype=F32, ghost=0.1):
    rng = np.random.default_rng(seed)
    lo, hi, bc = np.zeros(3), np.ones(3), np.ones(3, np.int32)
    pos = orc.wrap(rng.random((n, 3)).astype(dtype), lo.astype(dtype), hi.astype(dtype), bc)
    vd = pd.VectorDist(n, lo, hi, bc, ghost, dtype=dtype, props=props)
    vd.hostToDevicePos(pos)
    vd.map()
    vd.ghost_get()
    return vd, pos


@pytest.mark.parametrize("prp", [0, 1, 2, 3])
def test_remove_marked_reference_case(pd, orc, prp):
    n = 50000
    vd, pos = _vd(pd, orc, n, [(pd.PD_F32, 1), (pd.PD_F32, 1), (pd.PD_I32, 1), (pd.PD_I32, 1)], 11)
    assert vd.size_local_with_ghost() > n
    base = np.arange(1, n + 1)
    cols = [base.astype(F32), base.astype(F32), base.astype(np.int32), base.astype(np.int32)]
    cols[prp] = (base % 3 == 0).astype(cols[prp].dtype)
    for c in range(4):
        vd.hostToDeviceProp(c, cols[c], offset=0)
    gid = vd.gid(with_ghost=False)
    vd.remove_marked(prp)
    out = orc.remove_marked(cols[prp], pos, gid, *cols)
    kpos, kgid, kcols = out[2], out[3], out[4:]
    kcols = list(kcols)
    kcols[prp] = out[1]
    assert vd.size_local() == n - n // 3 == vd.size_local_with_ghost()
    assert np.array_equal(vd.deviceToHostPos(), kpos)
    assert np.array_equal(vd.gid(), kgid)
    for c in range(4):
        assert np.array_equal(vd.deviceToHostProp(c), kcols[c])
        if c != prp:
            assert np.all(vd.deviceToHostProp(c).astype(np.int64) % 3 != 0)
    # nothing marked: nothing removed (the mark is flipped to 1 everywhere)
    m = vd.size_local()
    vd.hostToDeviceProp(prp, np.zeros(m, cols[prp].dtype))
    vd.remove_marked(prp)
    assert vd.size_local() == m and np.all(vd.deviceToHostProp(prp) == 1)
    # everything marked
    vd.hostToDeviceProp(prp, np.ones(m, cols[prp].dtype))
    vd.remove_marked(prp)
    assert vd.size_local() == 0 and vd.size_local_with_ghost() == 0


@pytest.mark.parametrize("mtype", ["f64", "i64", "u32"])
def test_remove_marked_wide_records_and_types(pd, orc, mtype):
    """FP64 positions (32-byte records), vector properties, 64-bit and unsigned
    marks, a ragged size and random marks; then the vector is used again
    (map, ghost_get, getVerlet) and equals the oracle on the kept particles."""
    t, npt = {"f64": (pd.PD_F64, F64), "i64": (pd.PD_I64, np.int64), "u32": (pd.PD_U32, np.uint32)}[mtype]
    n = 70001
    vd, pos = _vd(pd, orc, n, [(pd.PD_F64, 3), (t, 1), (pd.PD_F32, 2)], 12, dtype=F64)
    rng = np.random.default_rng(13)
    v = rng.normal(size=(n, 3))
    mark = (rng.random(n) < 0.3).astype(npt)
    w = rng.normal(size=(n, 2)).astype(F32)
    vd.hostToDeviceProp(0, v)
    vd.hostToDeviceProp(1, mark)
    vd.hostToDeviceProp(2, w)
    gid = vd.gid(with_ghost=False)
    vd.remove_marked(1)
    flipped, kmark, kpos, kgid, kv, kw = orc.remove_marked(mark, pos, gid, v, w)
    assert vd.size_local() == kpos.shape[0] == int((mark == 0).sum())
    assert np.array_equal(vd.deviceToHostPos(), kpos)
    assert np.array_equal(vd.gid(), kgid)
    assert np.array_equal(vd.deviceToHostProp(0), kv)
    assert np.array_equal(vd.deviceToHostProp(1), kmark)
    assert np.array_equal(vd.deviceToHostProp(2), kw)
    vd.map()
    vd.ghost_get()
    vl = vd.getVerlet(0.1)
    off, idx = vl.get()
    allp = vd.deviceToHostPos()
    G = orc.cl_geometry(np.zeros(3), np.ones(3), 0.1, 0.1, verlet=True)
    eoff, eidx = orc.verlet(allp, kpos.shape[0], G, 0.1)
    assert np.array_equal(off, eoff) and np.array_equal(idx, eidx)


def test_remove_marked_empty_and_errors(pd, orc):
    vd = pd.VectorDist(0, np.zeros(3), np.ones(3), np.ones(3, np.int32), 0.1, dtype=F64, props=[(pd.PD_I32, 1)])
    vd.remove_marked(0)
    assert vd.size_local() == 0
    with pytest.raises(RuntimeError):
        vd.remove_marked(3)


def test_get_indexes_by_type(pd, orc):
    """type_is_one on an int property, the other comparisons on a double one,
    `end` inside the domain and past it (ghost slots included)."""
    n = 10000
    vd, _ = _vd(pd, orc, n, [(pd.PD_I32, 1), (pd.PD_F64, 1)], 14, dtype=F64)
    m = vd.size_local_with_ghost()
    rng = np.random.default_rng(15)
    t = (rng.random(m) / 0.5).astype(np.int32)
    d = np.round(rng.normal(size=m) * 4)
    vd.hostToDeviceProp(0, t)
    vd.hostToDeviceProp(1, d)
    ids = vd.get_indexes_by_type(0, 1)
    assert np.array_equal(ids, orc.indexes_by_type(t, n, 0, 1))
    assert np.all(t[ids] == 1)
    for cmp in range(6):
        assert np.array_equal(vd.get_indexes_by_type(1, 2, cmp=cmp), orc.indexes_by_type(d, n, cmp, 2.0))
    assert np.array_equal(vd.get_indexes_by_type(0, 1, end=1234), orc.indexes_by_type(t, 1234, 0, 1))
    assert np.array_equal(vd.get_indexes_by_type(0, 1, end=m), orc.indexes_by_type(t, m, 0, 1))
    assert vd.get_indexes_by_type(0, 7).shape[0] == 0
    # the indexes in device memory (a CUDA tensor) are the same
    dev = vd.get_indexes_by_type(0, 1, device=True)
    assert dev.is_cuda and np.array_equal(dev.cpu().numpy().astype(np.uint32), ids)
