"""WCSPH driver (dam break with fixed walls) against the FP64 oracle.

Same kick-drift-kick scheme and pair set (r < 2h) on both sides.  FP64: per-step
fluid kinetic energy and density sum within 1e-9 relative, final positions /
velocities / densities matched through the original particle ids within 1e-9
of their scale.  FP32 storage: velocities within 2e-3 of the velocity scale and
densities within 1e-5 relative after the same steps.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DP = 1.0 / 32
H = 1.3 * DP
C0, RHO0, ALPHA, GZ, DT = 20.0, 1000.0, 0.1, -9.81, 1e-4


@pytest.fixture(scope="module")
def pd():
    from openfpm_pdata_b200 import pd as _pd
    _pd.lib()
    return _pd


def _run_gpu(pd, x, typ, m, lo, hi, dtype, steps, skin):
    ft = pd.PD_F64 if dtype == np.float64 else pd.PD_F32
    vd = pd.VectorDist(x.shape[0], lo, hi, np.zeros(3, np.int32), 0.0, dtype=dtype,
                       props=[(ft, 3), (ft, 3), (ft, 1), (ft, 1), (pd.PD_I32, 1)])
    vd.hostToDevicePos(x.astype(dtype))
    vd.hostToDeviceProp(0, np.zeros((x.shape[0], 3)))
    vd.hostToDeviceProp(2, np.full(x.shape[0], RHO0))
    vd.hostToDeviceProp(4, typ)
    sph = pd.SPH(vd, 0, 1, 2, 3, 4, H, m, C0, RHO0, ALPHA, GZ, DT, skin=skin)
    E = sph.run(steps)
    gid = vd.gid(with_ghost=False)
    xs = np.zeros_like(x)
    vs = np.zeros_like(x)
    rs = np.zeros(x.shape[0])
    xs[gid] = vd.deviceToHostPos(with_ghost=False)
    vs[gid] = vd.deviceToHostProp(0, with_ghost=False)
    rs[gid] = vd.deviceToHostProp(2, with_ghost=False)
    return E, xs, vs, rs, sph


@pytest.mark.parametrize("skin", [0.0, 0.3 * DP])
def test_sph_fp64_matches_oracle(pd, orc, skin):
    from openfpm_pdata_b200 import workloads
    x, typ, m, lo, hi = workloads.sph_dam(DP)
    steps = 30
    E, xs, vs, rs, sph = _run_gpu(pd, x, typ, m, lo, hi, np.float64, steps, skin)
    xo, vo, ro, Eo = orc.md_sph(x, np.zeros_like(x), np.full(x.shape[0], RHO0), typ, lo, hi, H, m, C0, RHO0,
                                ALPHA, GZ, DT, steps)
    np.testing.assert_allclose(E[:, 0], Eo[:, 0], rtol=1e-9, atol=1e-14)
    np.testing.assert_allclose(E[:, 1], Eo[:, 1], rtol=1e-12)
    assert np.max(np.abs(xs - xo)) < 1e-9
    assert np.max(np.abs(vs - vo)) < 1e-9 * max(1.0, np.abs(vo).max())
    assert np.max(np.abs(rs - ro)) < 1e-9 * RHO0
    assert np.all(vs[typ == 1] == 0) and np.array_equal(xs[typ == 1], x[typ == 1])
    b, s, err = sph.stats()
    assert s == steps and err == 0


def test_sph_fp32_close_to_fp64(pd, orc):
    from openfpm_pdata_b200 import workloads
    x, typ, m, lo, hi = workloads.sph_dam(DP)
    steps = 30
    E, xs, vs, rs, _ = _run_gpu(pd, x, typ, m, lo, hi, np.float32, steps, 0.3 * DP)
    xo, vo, ro, Eo = orc.md_sph(x, np.zeros_like(x), np.full(x.shape[0], RHO0), typ, lo, hi, H, m, C0, RHO0,
                                ALPHA, GZ, DT, steps)
    vscale = np.abs(vo).max()
    print("fp32 max |dv|/vscale", np.max(np.abs(vs - vo)) / vscale, "max |drho|/rho0", np.max(np.abs(rs - ro)) / RHO0)
    assert np.max(np.abs(vs - vo)) < 2e-3 * vscale
    assert np.max(np.abs(rs - ro)) < 1e-5 * RHO0


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_sph_one_run_equals_runs_of_one_step(pd, dtype):
    """A run of 30 steps (each step's closing kick fused with the next step's kick and
    drift in one pass) leaves the same positions, velocities and densities, bit for
    bit, and the same energies as 30 runs of one step each (separate kick and
    kick-drift passes)."""
    from openfpm_pdata_b200 import workloads
    x, typ, m, lo, hi = workloads.sph_dam(DP)
    ft = pd.PD_F64 if dtype == np.float64 else pd.PD_F32
    out = []
    for split in (False, True):
        vd = pd.VectorDist(x.shape[0], lo, hi, np.zeros(3, np.int32), 0.0, dtype=dtype,
                           props=[(ft, 3), (ft, 3), (ft, 1), (ft, 1), (pd.PD_I32, 1)])
        vd.hostToDevicePos(x.astype(dtype))
        vd.hostToDeviceProp(0, np.zeros((x.shape[0], 3)))
        vd.hostToDeviceProp(2, np.full(x.shape[0], RHO0))
        vd.hostToDeviceProp(4, typ)
        sph = pd.SPH(vd, 0, 1, 2, 3, 4, H, m, C0, RHO0, ALPHA, GZ, DT, skin=0.3 * DP)
        E = np.concatenate([sph.run(1) for _ in range(30)]) if split else sph.run(30)
        out.append((E, vd.deviceToHostPos(with_ghost=False), vd.deviceToHostProp(0, with_ghost=False),
                    vd.deviceToHostProp(2, with_ghost=False), sph.stats()[0]))
    (E0, x0, v0, r0, b0), (E1, x1, v1, r1, b1) = out
    assert b0 == b1
    np.testing.assert_array_equal(x0, x1)
    np.testing.assert_array_equal(v0, v1)
    np.testing.assert_array_equal(r0, r1)
    np.testing.assert_array_equal(E0[:, 3], E1[:, 3])
    np.testing.assert_allclose(E0[:, :2], E1[:, :2], rtol=1e-12, atol=1e-14)
