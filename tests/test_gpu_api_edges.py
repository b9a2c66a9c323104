"""Edge cases and the remaining reference-API rows through the C ABI.

reduce_local (vector_dist_cuda_funcs.cuh:247-270), getDomainIteratorGPU and
toKernel (vector_dist.hpp:1958-1979, 2961-2966), resize, an empty vector, a
single particle, and ghost_get with periodic and non-periodic directions mixed
(vector_dist_unit_test.cpp:631-735 checks periodic ghosts; bc per direction is
the reference's `const size_t (&bc)[dim]`).
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


def test_reduce_local_sum_and_max(pd):
    rng = np.random.default_rng(3)
    n = 100003  # ragged: not a multiple of any block size
    vd = pd.VectorDist(n, np.zeros(3), np.ones(3), np.ones(3, np.int32), 0.1, dtype=F64,
                       props=[(pd.PD_F64, 2), (pd.PD_F32, 1), (pd.PD_I32, 1)])
    vd.hostToDevicePos(rng.random((n, 3)))
    a = rng.normal(size=(n, 2))
    b = rng.normal(size=n).astype(np.float32)
    c = rng.integers(-1000, 1000, size=n).astype(np.int32)
    vd.hostToDeviceProp(0, a)
    vd.hostToDeviceProp(1, b)
    vd.hostToDeviceProp(2, c)
    for comp in range(2):
        assert vd.reduce_local(0, comp, pd.RED_ADD) == pytest.approx(a[:, comp].sum(), rel=1e-12, abs=1e-9)
        assert vd.reduce_local(0, comp, pd.RED_MAX) == a[:, comp].max()
    assert vd.reduce_local(1, 0, pd.RED_ADD) == pytest.approx(b.astype(np.float64).sum(), rel=1e-12, abs=1e-9)
    assert vd.reduce_local(1, 0, pd.RED_MAX) == float(b.max())
    assert vd.reduce_local(2, 0, pd.RED_ADD) == float(c.astype(np.int64).sum())
    assert vd.reduce_local(2, 0, pd.RED_MAX) == float(c.max())
    # deterministic: the same bits twice
    assert vd.reduce_local(0, 1, pd.RED_ADD) == vd.reduce_local(0, 1, pd.RED_ADD)


def test_domain_iterator_and_view(pd):
    n = 1000
    rng = np.random.default_rng(4)
    vd = pd.VectorDist(n, np.zeros(3), np.ones(3), np.ones(3, np.int32), 0.1, dtype=F64, props=[(pd.PD_F64, 3)])
    vd.hostToDevicePos(rng.random((n, 3)))
    it = vd.getDomainIteratorGPU(128)
    assert tuple(it.thr) == (128, 1, 1) and tuple(it.wthr) == (8, 1, 1)
    v0 = vd.toKernel()
    assert v0.size_local == n and v0.size == n and v0.n_prop == 1 and v0.stride >= n
    vd.map()
    vd.ghost_get()
    v1 = vd.toKernel()
    m = vd.size_local_with_ghost()
    assert v1.size_local == n and v1.size == m > n and v1.epoch > v0.epoch
    itg = vd.getDomainIteratorGPU(256, with_ghost=True)
    assert itg.wthr[0] * itg.thr[0] >= m and (itg.wthr[0] - 1) * itg.thr[0] < m


def test_resize_keeps_leading_particles(pd):
    rng = np.random.default_rng(5)
    x = rng.random((5000, 3))
    vd = pd.VectorDist(5000, np.zeros(3), np.ones(3), np.ones(3, np.int32), 0.1, dtype=F64, props=[(pd.PD_F64, 1)])
    vd.hostToDevicePos(x)
    vd.resize(20000)
    assert vd.size_local() == 20000
    assert np.array_equal(vd.deviceToHostPos(count=5000, with_ghost=False), x)
    vd.resize(1000)
    assert vd.size_local() == 1000
    assert np.array_equal(vd.deviceToHostPos(with_ghost=False), x[:1000])


def test_empty_vector(pd):
    vd = pd.VectorDist(0, np.zeros(3), np.ones(3), np.ones(3, np.int32), 0.1, dtype=F64, props=[(pd.PD_F64, 3)])
    vd.map()
    vd.ghost_get()
    assert vd.size_local() == 0 and vd.size_local_with_ghost() == 0
    cl = vd.getCellListGPU(0.1)
    vd.updateCellListGPU(cl)
    start, ids = cl.get()[:2]
    assert np.all(np.asarray(start) == 0) and len(ids) == 0
    vl = vd.getVerlet(0.1)
    off, idx = vl.get()
    assert len(idx) == 0
    assert vd.reduce_local(0, 0, pd.RED_ADD) == 0.0


def test_single_particle_corner_images(pd, orc):
    """One particle near a corner of a periodic box has 7 images (every shift
    that reaches it), in shift order."""
    lo, hi, bc = np.zeros(3), np.ones(3), np.ones(3, np.int32)
    x = np.array([[0.01, 0.02, 0.97]])
    vd = pd.VectorDist(1, lo, hi, bc, 0.1, dtype=F64)
    vd.hostToDevicePos(x)
    vd.ghost_get()
    got = vd.deviceToHostPos()[1:]
    img, src, shf = orc.ghost_get(x, lo, hi, bc, 0.1)
    assert got.shape[0] == 7
    assert np.array_equal(got, img)


@pytest.mark.parametrize("bc", [[1, 0, 1], [0, 1, 0], [0, 0, 0]])
def test_ghost_get_mixed_boundaries(pd, orc, bc):
    rng = np.random.default_rng(6)
    lo, hi = np.zeros(3), np.ones(3)
    bc = np.array(bc, np.int32)
    pos = rng.random((20000, 3))
    vd = pd.VectorDist(pos.shape[0], lo, hi, bc, 0.2, dtype=F64)
    vd.hostToDevicePos(pos)
    vd.ghost_get()
    img, src, shf = orc.ghost_get(pos, lo, hi, bc, 0.2)
    got = vd.deviceToHostPos()[pos.shape[0]:]
    assert np.array_equal(got, img)
    gsrc, gshf = vd.ghost_records()
    assert np.array_equal(gsrc, src) and np.array_equal(gshf, shf)


def test_ighost_get_equals_ghost_get(pd):
    """Ighost_get + ghost_wait (vector_dist.hpp:2241-2291) give the images of
    ghost_get bit for bit: the first call overflows its estimated room (no
    previous count) and is redone synchronously, the second fits; the
    SKIP_LABELLING replay refreshes moved sources."""
    rng = np.random.default_rng(9)
    n = 40000
    x = rng.random((n, 3))
    p = rng.normal(size=(n, 3))

    def make():
        vd = pd.VectorDist(n, np.zeros(3), np.ones(3), np.ones(3, np.int32), 0.1, dtype=F64,
                           props=[(pd.PD_F64, 3)])
        vd.hostToDevicePos(x)
        vd.hostToDeviceProp(0, p)
        vd.map()
        return vd
    a, b = make(), make()
    a.ghost_get()
    b.Ighost_get()
    b.ghost_wait()
    assert b.size_local_with_ghost() == a.size_local_with_ghost() > n
    assert np.array_equal(b.deviceToHostPos(), a.deviceToHostPos())
    assert np.array_equal(b.deviceToHostProp(0), a.deviceToHostProp(0))
    assert all(np.array_equal(u, w) for u, w in zip(b.ghost_records(), a.ghost_records()))
    # second exchange after a small move: the room from the first count suffices
    x2 = x + rng.uniform(-0.01, 0.01, size=x.shape)
    for vd in (a, b):
        vd.hostToDevicePos(x2)
        vd.map()
    a.ghost_get()
    b.Ighost_get()
    b.ghost_wait()
    assert np.array_equal(b.deviceToHostPos(), a.deviceToHostPos())
    # replay of the same images after the sources' properties changed
    p2 = rng.normal(size=(n, 3))
    for vd in (a, b):
        vd.hostToDeviceProp(0, p2)
    a.ghost_get([0], opt=pd.RUN_ON_DEVICE | pd.SKIP_LABELLING)
    b.Ighost_get([0], opt=pd.RUN_ON_DEVICE | pd.SKIP_LABELLING)
    b.ghost_wait()
    assert np.array_equal(b.deviceToHostProp(0), a.deviceToHostProp(0))
    # a second Ighost_get, a ghost_get or a map before the wait are refused
    b.Ighost_get()
    with pytest.raises(RuntimeError):
        b.Ighost_get()
    with pytest.raises(RuntimeError):
        b.ghost_get()
    with pytest.raises(RuntimeError):
        b.map()
    b.ghost_wait()
    b.map()


def test_md_spare_storage_across_storage_changes(pd):
    """The MD driver's rebuild reorders into the vector's spare storage and swaps it
    in, carrying every property but the force with its particle (here an int mark
    set before the run selects the same particles after it).  Across a compaction
    (new storage of the same capacity) and a property added afterwards (the spare
    no longer matches), a second driver on the same vector gives the energies of a
    driver on a fresh vector holding the same state, bit for bit (the same kernels
    on the same data)."""
    from openfpm_pdata_b200 import workloads
    x, v, L = workloads.lj_lattice(12, 1.1, 0.05, seed=51)
    n = x.shape[0]
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    props = [(pd.PD_F64, 3), (pd.PD_F64, 3), (pd.PD_I32, 1)]
    vd = pd.VectorDist(n, lo, hi, bc, 2.8, dtype=F64, props=props)
    vd.hostToDevicePos(x)
    vd.hostToDeviceProp(0, v)
    vd.hostToDeviceProp(2, (np.arange(n) % 10 == 3).astype(np.int32))
    md = pd.MD(vd, 0, 1, dt=0.005, skin=0.3)
    md.run(12)
    del md
    # the mark followed its particles through the run's reorders (gid = original index)
    gid = vd.gid(with_ghost=False)
    assert np.array_equal(vd.deviceToHostProp(2, with_ghost=False), (gid % 10 == 3).astype(np.int32))
    vd.remove_marked(2)
    extra = vd.add_prop(pd.PD_F64, 2)
    m = vd.size_local()
    assert m == n - int((np.arange(n) % 10 == 3).sum())
    vd.hostToDeviceProp(extra, np.ones((m, 2)))
    xs = vd.deviceToHostPos(with_ghost=False)
    vs = vd.deviceToHostProp(0, with_ghost=False)
    E1 = pd.MD(vd, 0, 1, dt=0.005, skin=0.3).run(15)
    fresh = pd.VectorDist(m, lo, hi, bc, 2.8, dtype=F64, props=props + [(pd.PD_F64, 2)])
    fresh.hostToDevicePos(xs)
    fresh.hostToDeviceProp(0, vs)
    E2 = pd.MD(fresh, 0, 1, dt=0.005, skin=0.3).run(15)
    assert np.isfinite(E1).all()
    assert np.array_equal(E1, E2)
    assert np.array_equal(vd.deviceToHostProp(extra, with_ghost=False), np.ones((m, 2)))


def test_md_launch_shape(pd):
    """The driver reports the shapes its kernels ran with: the one-cluster step of
    a small cell-list system (16 CTAs, or 8 where 16 cannot be placed) and the
    tile width of the tiled rows."""
    from openfpm_pdata_b200 import workloads
    x, v, L = workloads.lj_lattice(16, 1.0, 0.05, seed=1)
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    vd = pd.VectorDist(x.shape[0], lo, hi, bc, 2.5, dtype=F64, props=[(pd.PD_F64, 3), (pd.PD_F64, 3)])
    vd.hostToDevicePos(x)
    vd.hostToDeviceProp(0, v)
    md = pd.MD(vd, 0, 1, dt=0.005, skin=0.0, r_cut=2.5, use_cell_list=True)
    assert md.launch_shape()["cluster_ctas"] == 0
    md.run(2)
    assert md.launch_shape()["cluster_ctas"] in (8, 16)

    x, v, L = workloads.lj_lattice(24, 1.1, 0.05, seed=2)
    vd = pd.VectorDist(x.shape[0], np.zeros(3), np.full(3, L), bc, 2.8, dtype=F64,
                       props=[(pd.PD_F64, 3), (pd.PD_F64, 3)])
    vd.hostToDevicePos(x)
    vd.hostToDeviceProp(0, v)
    md = pd.MD(vd, 0, 1, dt=0.005, skin=0.3)
    md.set_tiles(True, 7)
    md.run(1)
    s = md.launch_shape()
    assert s["tile_tx"] == 7 and s["threads_per_particle"] == 2 and s["cluster_ctas"] == 0
