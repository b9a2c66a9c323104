"""Parity at the benchmark configurations' own sizes (the reference's GPU-vs-CPU
checks, Vector/cuda/vector_dist_gpu_unit_tests.cu:600-888, at full scale):

* C1 exactly: 16^3 lattice at spacing 1 (jitter 0.05, seed 1), box 16, r_cut 2.5,
  cell list rebuilt every step, 100 velocity-Verlet steps in one thread-block
  cluster launch; per-step energies within 1e-9 relative and positions within
  1e-8 of the FP64 oracle.
* C2 at 4,096,000 particles: 160^3 lattice at spacing 1.1 (box 176), Verlet list
  of radius 2.8; after the first build the rows of a strided sample of 20,000
  particles hold exactly the oracle's neighbour sets, and 3 steps give the
  oracle's energies within 1e-9.
* C3 WCSPH at dp = 1/64 (walls, uneven occupancy): FP64 within 1e-9 of the oracle.
The precision form at 4,096,000 (C2 lattice and C4 clusters) is in test_gpu_mixed.py,
the serving loop (C5) in test_gpu_serving.py.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pd():
    from openfpm_pdata_b200 import pd as _pd
    _pd.lib()
    return _pd


def _vd(pd, x, L, ghost):
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    vd = pd.VectorDist(x.shape[0], lo, hi, bc, ghost, dtype=np.float64, props=[(pd.PD_F64, 3), (pd.PD_F64, 3)])
    vd.hostToDevicePos(x)
    return vd, lo, hi, bc


def test_c1_config_exact(pd, orc):
    from openfpm_pdata_b200 import workloads
    x, v, L = workloads.lj_lattice(16, 1.0, 0.05, seed=1)
    assert x.shape[0] == 4096 and L == 16.0
    vd, lo, hi, bc = _vd(pd, x, L, 2.5)
    vd.hostToDeviceProp(0, v)
    md = pd.MD(vd, 0, 1, dt=0.005, skin=0.0, r_cut=2.5, use_cell_list=True)
    l0 = pd.launch_count()
    E = md.run(100)
    launches = pd.launch_count() - l0
    # the first build, then all 100 steps in the cluster kernel: not the ~28 kernels of a graph step
    assert launches < 50, launches
    xo, vo, Eo = orc.md_lj(x, v, lo, hi, bc, 2.5, 2.5, 0.0, 1.0, 1.0, 0.005, 1.0, 100)
    np.testing.assert_allclose(E[:, :3], Eo[1:, :3], rtol=1e-9, atol=1e-9)
    gid = vd.gid(with_ghost=False)
    d = vd.deviceToHostPos(with_ghost=False) - xo[gid]
    d -= L * np.round(d / L)
    assert np.max(np.abs(d)) < 1e-8


def test_c2_config_full_size(pd, orc):
    from openfpm_pdata_b200 import workloads
    x, v, L = workloads.lj_lattice(160, 1.1, 0.05, seed=2)
    n = x.shape[0]
    assert n == 4096000 and abs(L - 176.0) < 1e-12
    vd, lo, hi, bc = _vd(pd, x, L, 2.8)
    vd.hostToDeviceProp(0, v)
    md = pd.MD(vd, 0, 1, dt=0.005, skin=0.3)
    md.run(0)  # the first list build
    off, idx, tiled = md.verlet()
    assert tiled
    allp = vd.deviceToHostPos()  # real particles, then images, as stored after the build
    sample = np.arange(0, n, n // 20000)[:20000]
    # the oracle's rows of the sample: sample particles first, the other real particles, the images
    perm = np.concatenate([sample, np.setdiff1d(np.arange(n), sample), np.arange(n, allp.shape[0])])
    G = orc.cl_geometry(lo, hi, 2.8, 2.8, verlet=True)
    eoff, eidx = orc.verlet(np.ascontiguousarray(allp[perm]), sample.shape[0], G, 2.8)
    for k, i in enumerate(sample):
        got = np.sort(idx[off[i]:off[i + 1]])
        exp = np.sort(perm[eidx[eoff[k]:eoff[k + 1]]])
        assert np.array_equal(got, exp), i
    del off, idx, allp
    E = md.run(3)
    _, _, Eo = orc.md_lj(x, v, lo, hi, bc, 2.8, 2.5, 0.3, 1.0, 1.0, 0.005, 1.0, 3)
    np.testing.assert_allclose(E[:, :3], Eo[1:, :3], rtol=1e-9, atol=1e-9)


def test_c3_wcsph_fine_resolution(pd, orc):
    """dp = 1/64: 3 wall layers on the floor and four sides, the fluid block, skin 0.3 dp."""
    from openfpm_pdata_b200 import workloads
    dp = 1.0 / 64
    h, c0, rho0, alpha, gz, dt = 1.3 * dp, 20.0, 1000.0, 0.1, -9.81, 1e-4
    x, typ, m, lo, hi = workloads.sph_dam(dp)
    assert x.shape[0] > 100000
    vd = pd.VectorDist(x.shape[0], lo, hi, np.zeros(3, np.int32), 0.0, dtype=np.float64,
                       props=[(pd.PD_F64, 3), (pd.PD_F64, 3), (pd.PD_F64, 1), (pd.PD_F64, 1), (pd.PD_I32, 1)])
    vd.hostToDevicePos(x)
    vd.hostToDeviceProp(0, np.zeros((x.shape[0], 3)))
    vd.hostToDeviceProp(2, np.full(x.shape[0], rho0))
    vd.hostToDeviceProp(4, typ)
    steps = 20
    sph = pd.SPH(vd, 0, 1, 2, 3, 4, h, m, c0, rho0, alpha, gz, dt, skin=0.3 * dp)
    E = sph.run(steps)
    gid = vd.gid(with_ghost=False)
    xs, vs, rs = np.zeros_like(x), np.zeros_like(x), np.zeros(x.shape[0])
    xs[gid] = vd.deviceToHostPos(with_ghost=False)
    vs[gid] = vd.deviceToHostProp(0, with_ghost=False)
    rs[gid] = vd.deviceToHostProp(2, with_ghost=False)
    xo, vo, ro, Eo = orc.md_sph(x, np.zeros_like(x), np.full(x.shape[0], rho0), typ, lo, hi, h, m, c0, rho0, alpha,
                                gz, dt, steps)
    np.testing.assert_allclose(E[:, 0], Eo[:, 0], rtol=1e-9, atol=1e-14)
    np.testing.assert_allclose(E[:, 1], Eo[:, 1], rtol=1e-12)
    assert np.max(np.abs(xs - xo)) < 1e-9
    assert np.max(np.abs(vs - vo)) < 1e-9 * max(1.0, np.abs(vo).max())
    assert np.max(np.abs(rs - ro)) < 1e-9 * rho0
