"""pd_celllist_build_static: the cell-list counting sort for callers that cannot
allocate device memory (graph capture in progress, host-owned memory pools,
no device synchronisation allowed).

Checked through the C ABI against the allocating entry point
(pd_celllist_update) on the same positions and grid: the integer outputs
(cell_start, sorted ids) must be identical, on two calls in a row since every
call reuses the one static scratch array.  This file is collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _reference_and_geometry(pd, dtype, n, seed):
    rng = np.random.default_rng(seed)
    L = 6.0
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    pos = rng.uniform(0, L, size=(n, 3)).astype(dtype)
    vd = pd.VectorDist(n, lo, hi, bc, 0.5, dtype=dtype)
    vd.hostToDevicePos(pos)
    vd.map()
    vd.ghost_get()
    cl = vd.getCellListGPU(0.5)
    vd.updateCellListGPU(cl)
    cs, so = cl.get()
    v = cl.view()
    allp = vd.deviceToHostPos()
    return allp, cs, so, v


def _static_build(pd, torch, dtype, allp, v, fill):
    code = pd.PD_F64 if dtype == np.float64 else pd.PD_F32
    pos_d = torch.from_numpy(np.ascontiguousarray(allp)).cuda()
    cs_d = torch.full((v.ncells + 1,), fill, dtype=torch.int32, device="cuda")
    so_d = torch.full((allp.shape[0],), fill, dtype=torch.int32, device="cuda")
    box_lo = (ctypes.c_double * 3)(*v.box_lo)
    sp = (ctypes.c_double * 3)(*v.spacing)
    gs = (ctypes.c_int * 3)(*v.gs)
    rc = pd.lib().pd_celllist_build_static(code, ctypes.c_void_p(pos_d.data_ptr()), allp.shape[0], box_lo, sp, gs,
                                           v.pad, ctypes.c_void_p(cs_d.data_ptr()),
                                           ctypes.c_void_p(so_d.data_ptr()), None)
    torch.cuda.synchronize()
    return rc, cs_d.cpu().numpy(), so_d.cpu().numpy()


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_static_scratch_sort_matches_allocating_sort(dtype):
    import torch
    from openfpm_pdata_b200 import pd
    pd.lib()
    allp, cs, so, v = _reference_and_geometry(pd, dtype, 60000, 77)
    assert v.ncells + 1 <= (1 << 19) and allp.shape[0] <= (1 << 19)
    # two calls in a row: the second finds the first call's contents in the scratch
    for fill in (-1, 7):
        rc, cs2, so2 = _static_build(pd, torch, dtype, allp, v, fill)
        assert rc == 0, pd.lib().pd_last_error()
        assert np.array_equal(cs2, cs)
        assert np.array_equal(so2, so)
    # a different particle set next: nothing of the previous call leaks through
    allp_b, cs_b, so_b, v_b = _reference_and_geometry(pd, dtype, 20000, 78)
    rc, cs3, so3 = _static_build(pd, torch, dtype, allp_b, v_b, -1)
    assert rc == 0
    assert np.array_equal(cs3, cs_b) and np.array_equal(so3, so_b)


def test_static_scratch_rejects_sizes_beyond_limit():
    from openfpm_pdata_b200 import pd
    L = pd.lib()
    box_lo = (ctypes.c_double * 3)(0, 0, 0)
    sp = (ctypes.c_double * 3)(1, 1, 1)
    gs = (ctypes.c_int * 3)(10, 10, 10)
    dummy = ctypes.c_void_p(16)
    rc = L.pd_celllist_build_static(pd.PD_F64, dummy, (1 << 19) + 1, box_lo, sp, gs, 1, dummy, dummy, None)
    assert rc == -1
    assert b"static scratch limit" in L.pd_last_error()
    big = (ctypes.c_int * 3)(100, 100, 100)
    rc = L.pd_celllist_build_static(pd.PD_F64, dummy, 10, box_lo, sp, big, 1, dummy, dummy, None)
    assert rc == -1
