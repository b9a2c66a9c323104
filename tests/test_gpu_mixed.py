"""Precision form: FP32 cell-local positions and pair math with Kahan-compensated
sums against the FP64 oracle on the same positions.

Force error metric: |F_mixed - F_fp64| / F_rms per particle (F_rms = root mean
square force of the FP64 result).  The bound of this form is 1e-5 on the maximum
over particles: pair displacements are exact (offsets on a power-of-two grid) and
pairs within FP32 rounding of the cutoff are decided in FP64, so only the FP32
pair arithmetic remains.  Where the box length is not a multiple of the offset
quantum (2^-21 for a cell side of 2.8), an image offset is rounded once to the
grid; such boxes are held to 1e-4 on the maximum.  Per-step energies within 2e-5
relative of the FP64 driver over 60 steps (the trajectories separate slowly).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pd():
    from openfpm_pdata_b200 import pd as _pd
    _pd.lib()
    return _pd


def _system(pd, x, v, L, precision):
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    ptype = pd.PD_F32 if precision == pd.PREC_MIXED else pd.PD_F64
    vd = pd.VectorDist(x.shape[0], lo, hi, bc, 2.8, dtype=np.float64, props=[(ptype, 3), (ptype, 3)])
    vd.hostToDevicePos(x)
    vd.hostToDeviceProp(0, v)
    md = pd.MD(vd, 0, 1, dt=0.005, skin=0.3, precision=precision)
    return vd, md


def _force_error(orc, vd, L, n):
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    x = orc.wrap(vd.deviceToHostPos(with_ghost=False), lo, hi, bc)
    img, _, _ = orc.ghost_get(x, lo, hi, bc, 2.8)
    allp = np.concatenate([x, img])
    G = orc.cl_geometry(lo, hi, 2.8, 2.5)
    f64, _, _ = orc.lj_cell(allp, n, G)
    f32 = vd.deviceToHostProp(1, with_ghost=False)[:n].astype(np.float64)
    frms = np.sqrt((f64 ** 2).sum(axis=1).mean())
    err = np.sqrt(((f32 - f64) ** 2).sum(axis=1)) / frms
    return err.mean(), err.max()


@pytest.mark.parametrize("layout", ["lattice", "lattice_on_grid", "clustered"])
def test_mixed_forces_vs_fp64(pd, orc, layout):
    from openfpm_pdata_b200 import workloads
    bound = 1e-5
    if layout == "lattice":
        x, v, L = workloads.lj_lattice(16, 1.1, 0.05, seed=41)  # box 17.6: images rounded to the grid once
        bound = 1e-4
    elif layout == "lattice_on_grid":
        x, v, L = workloads.lj_lattice(16, 1.125, 0.05, seed=41)  # box 18
    else:
        x, v, L = workloads.lj_clustered(4000, 18.0, n_clusters=4, sigma_c=3.0, seed=42)
    vd, md = _system(pd, x, v, L, pd.PREC_MIXED)
    for chunk in range(3):
        md.run(10)
        mean, mx = _force_error(orc, vd, L, x.shape[0])
        print(f"{layout} after {10 * (chunk + 1)} steps: mean {mean:.2e} max {mx:.2e}")
        assert mean < 1e-6 and mx <= bound


def _fp64_gpu_forces(pd, x, L):
    """LJ forces of the FP64 cell-list path at positions x (in the order of x);
    tests/test_gpu_parity.py holds this path to the FP64 oracle."""
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    vd = pd.VectorDist(x.shape[0], lo, hi, bc, 2.5, dtype=np.float64, props=[(pd.PD_F64, 3)])
    vd.hostToDevicePos(x)
    vd.map()
    vd.ghost_get()
    cl = vd.getCellListGPU(2.5)
    vd.updateCellListGPU(cl)
    vd.lj_forces(0, cl=cl, eps=1.0, sigma=1.0, r_cut=2.5)
    f = vd.deviceToHostProp(0, with_ghost=False)
    del cl, vd
    return f


@pytest.mark.parametrize("layout", ["lattice_4M", "clustered_4M"])
def test_mixed_force_error_at_target_size(pd, orc, layout):
    """The precision form on the 4,096,000-particle workloads: the 160^3 lattice
    (spacing 1.1, box 176) and 64 Gaussian clusters (sigma_c 8, minimum distance
    0.8, box 176).  Per-particle max |F32 - F64| / F_rms <= 1e-5 after 10, 20 and
    30 steps, against the FP64 path on the same positions; the FP64 forces of a
    strided sample of 4,000 particles are checked against the oracle's."""
    from openfpm_pdata_b200 import workloads
    if layout == "lattice_4M":
        x, v, L = workloads.lj_lattice(160, 1.1, 0.05, seed=2)
    else:
        x, v, L, _ = workloads.lj_clustered_lib(4096000, 176.0, seed=4)
    n = x.shape[0]
    vd, md = _system(pd, x, v, L, pd.PREC_MIXED)
    for chunk in range(3):
        md.run(10)
        xf = vd.deviceToHostPos(with_ghost=False)
        f32 = vd.deviceToHostProp(1, with_ghost=False).astype(np.float64)
        f64 = _fp64_gpu_forces(pd, xf, L)
        if chunk == 0:
            lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
            xw = orc.wrap(xf, lo, hi, bc)
            sample = np.arange(0, n, n // 4000)[:4000]
            # the oracle's forces on the sample: its particles first, then everything else as neighbours
            rest = np.setdiff1d(np.arange(n), sample)
            img, _, _ = orc.ghost_get(xw, lo, hi, bc, 2.5)
            allp = np.concatenate([xw[sample], xw[rest], img])
            G = orc.cl_geometry(lo, hi, 2.5, 2.5)
            fo, _, _ = orc.lj_cell(allp, sample.shape[0], G)
            frms_o = np.sqrt((f64 ** 2).sum(axis=1).mean())
            assert np.abs(fo - f64[sample]).max() / frms_o < 1e-10
        frms = np.sqrt((f64 ** 2).sum(axis=1).mean())
        err = np.sqrt(((f32 - f64) ** 2).sum(axis=1)) / frms
        print(f"{layout} after {10 * (chunk + 1)} steps: mean {err.mean():.2e} max {err.max():.2e}")
        assert err.max() <= 1e-5


def test_mixed_energies_track_fp64(pd):
    from openfpm_pdata_b200 import workloads
    x, v, L = workloads.lj_lattice(14, 1.1, 0.05, seed=43)
    _, md64 = _system(pd, x, v, L, pd.PREC_FP64)
    _, md32 = _system(pd, x, v, L, pd.PREC_MIXED)
    E64 = md64.run(60)
    E32 = md32.run(60)
    tot64 = E64[:, 0] + E64[:, 1]
    tot32 = E32[:, 0] + E32[:, 1]
    print("max rel total-energy diff", np.max(np.abs(tot32 - tot64) / np.abs(tot64)))
    assert np.max(np.abs(tot32 - tot64) / np.abs(tot64)) < 2e-5
    assert np.max(np.abs(E32[:, 1] - E64[:, 1]) / np.abs(E64[:, 1])) < 2e-5


def test_mixed_one_run_equals_runs_of_one_step(pd):
    """Precision form: a run of 24 steps (a step's closing kick fused with the next
    step's kick and drift of the FP32 offsets) leaves the same positions and
    velocities, bit for bit, and the same rebuild steps as 24 runs of one step each
    (separate kick and kick-drift kernels)."""
    from openfpm_pdata_b200 import workloads
    x, v, L = workloads.lj_lattice(20, 1.1, 0.05, seed=35)
    out = []
    for split in (False, True):
        vd, md = _system(pd, x, v, L, pd.PREC_MIXED)
        E = np.concatenate([md.run(1) for _ in range(24)]) if split else md.run(24)
        out.append((E, vd.deviceToHostPos(with_ghost=False), vd.deviceToHostProp(0, with_ghost=False),
                    md.stats()[0]))
    (E0, p0, v0, b0), (E1, p1, v1, b1) = out
    assert b0 == b1 and b0 >= 3
    np.testing.assert_array_equal(E0[:, 3], E1[:, 3])
    np.testing.assert_array_equal(p0, p1)
    np.testing.assert_array_equal(v0, v1)
    np.testing.assert_allclose(E0[:, :3], E1[:, :3], rtol=1e-12, atol=1e-9)
