"""The reciprocal of the pair kernels (Newton-Raphson refinement of the
hardware approximation) stays within 2 ulp of the correctly rounded 1/x over
the range of squared pair distances (and far beyond)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_recip_error_bound(dtype):
    from openfpm_pdata_b200 import pd
    rng = np.random.default_rng(5)
    x = np.concatenate([np.exp(rng.uniform(np.log(1e-6), np.log(1e6), 200000)),
                        np.linspace(0.5, 8.0, 100001)]).astype(dtype)
    got = pd.selftest_recip(x)
    exact = (1.0 / x.astype(np.float64))
    ref = exact.astype(dtype)
    ulp = np.spacing(np.abs(ref).astype(dtype))
    err = np.abs(got.astype(np.float64) - exact) / ulp.astype(np.float64)
    assert err.max() <= 2.0, err.max()
