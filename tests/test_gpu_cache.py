"""Device block cache of the library's plain allocation path.

Vectors and drivers created and destroyed one after another take their device
blocks from the blocks the previous ones freed; a run's result does not depend
on whether its blocks were fresh or reused (bit-exact); the cache holds freed
blocks only up to its limit and is emptied on request.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pd():
    from openfpm_pdata_b200 import pd as _pd
    _pd.lib()
    return _pd


def _run(pd, n, seed):
    from openfpm_pdata_b200 import workloads
    x, v, L = workloads.serving_system(n, 0.8, seed=seed)
    vd = pd.VectorDist(n, np.zeros(3), np.full(3, L), np.ones(3, np.int32), 2.8, dtype=np.float64,
                       props=[(pd.PD_F64, 3), (pd.PD_F64, 3)])
    vd.hostToDevicePos(x)
    vd.hostToDeviceProp(0, v)
    md = pd.MD(vd, 0, 1, dt=0.005, skin=0.3)
    E = md.run(10)
    xo = np.zeros_like(x)
    xo[vd.gid(with_ghost=False)] = vd.deviceToHostPos(with_ghost=False)
    del md, vd
    return E, xo


def test_reused_blocks_same_results(pd):
    pd.empty_cache()
    assert pd.set_cache_limit() == 0
    E0, x0 = _run(pd, 20000, 1)           # fresh blocks
    assert pd.set_cache_limit() > 0       # the freed blocks are kept
    for k, n in enumerate([5000, 30000, 12000]):
        _run(pd, n, 2 + k)
    E1, x1 = _run(pd, 20000, 1)           # blocks freed by other runs
    assert np.array_equal(E0, E1)
    assert np.array_equal(x0, x1)
    pd.empty_cache()
    assert pd.set_cache_limit() == 0


def test_limit_bounds_the_cache(pd):
    try:
        assert pd.set_cache_limit(0) == 0  # caching off: every block goes back to the driver
        E0, x0 = _run(pd, 8000, 7)
        assert pd.set_cache_limit() == 0
        pd.set_cache_limit(1 << 20)        # 1 MiB: only small blocks are kept
        E1, x1 = _run(pd, 8000, 7)
        assert 0 <= pd.set_cache_limit() <= (1 << 20)
        assert np.array_equal(E0, E1) and np.array_equal(x0, x1)
    finally:
        pd.set_cache_limit(4 << 30)
        pd.empty_cache()
