"""Failure detection of the bounded device waits, without a GPU fault.

The tile kernels' staging pattern (an mbarrier armed for a bulk copy, a wait of
a bounded number of polls) runs once with the copy issued (completes) and once
without it (nothing completes the phase): the wait gives up, the kernel records
the timeout and returns, the call reports PD_ETIMEOUT, and the context keeps
working for the next calls.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pd():
    from openfpm_pdata_b200 import pd as _pd
    _pd.lib()
    return _pd


def test_bounded_wait_completes_and_gives_up(pd):
    rc, out = pd.selftest_wait(1 << 20, True)
    assert rc == 0 and np.array_equal(out, [1.5, -2.25, 3.0, 4.75])
    rc, out = pd.selftest_wait(2048, False)
    assert rc == -5                                   # PD_ETIMEOUT
    assert "gave up" in pd.lib().pd_last_error().decode()
    # the context is still usable: the staged copy and a small MD run both work
    rc, out = pd.selftest_wait(1 << 20, True)
    assert rc == 0 and np.array_equal(out, [1.5, -2.25, 3.0, 4.75])
    from openfpm_pdata_b200 import workloads
    x, v, L = workloads.lj_lattice(8, 1.1, 0.05, seed=2)
    vd = pd.VectorDist(x.shape[0], np.zeros(3), np.full(3, L), np.ones(3, np.int32), 2.8, dtype=np.float64,
                       props=[(pd.PD_F64, 3), (pd.PD_F64, 3)])
    vd.hostToDevicePos(x)
    vd.hostToDeviceProp(0, v)
    E = pd.MD(vd, 0, 1, dt=0.005, skin=0.3).run(5)
    assert np.isfinite(E).all()


def test_selftest_rejects_bad_arguments(pd):
    rc, _ = pd.selftest_wait(0, True)
    assert rc == -1
