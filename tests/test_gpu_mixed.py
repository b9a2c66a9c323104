"""Precision form: FP32 cell-local positions and pair math with Kahan-compensated
sums against the FP64 oracle on the same positions.

Force error metric: |F_mixed - F_fp64| / F_rms per particle (F_rms = root mean
square force of the FP64 result).  Bounds for this form: 1e-5 on the mean and
1e-4 on the maximum over particles.  Per-step energies within 2e-5 relative of
the FP64 driver over 60 steps (the trajectories separate slowly).
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


@pytest.mark.parametrize("layout", ["lattice", "clustered"])
def test_mixed_forces_vs_fp64(pd, orc, layout):
    from openfpm_pdata_b200 import workloads
    if layout == "lattice":
        x, v, L = workloads.lj_lattice(16, 1.1, 0.05, seed=41)
    else:
        x, v, L = workloads.lj_clustered(4000, 18.0, n_clusters=4, sigma_c=3.0, seed=42)
    vd, md = _system(pd, x, v, L, pd.PREC_MIXED)
    for chunk in range(3):
        md.run(10)
        mean, mx = _force_error(orc, vd, L, x.shape[0])
        print(f"{layout} after {10 * (chunk + 1)} steps: mean {mean:.2e} max {mx:.2e}")
        assert mean < 1e-5 and mx < 1e-4


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
