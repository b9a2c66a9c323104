"""pd_celllist_build_static: the cell-list counting sort for callers that cannot
allocate device memory (hosts whose device memory belongs to their own pool,
callers that may not let an allocation synchronise the device).

Checked through the C ABI against the allocating entry point
(pd_celllist_update) on the same positions and grid: the integer outputs
(cell_start, sorted ids) must be identical, on two calls in a row since every
call reuses the one static scratch array.  Also: repeated calls change neither
the device's free memory nor the library's block cache; the optional status
word reports positions outside the grid; cells of more than 32 and more than
512 members (clustered input) keep the stable order.  This file is collected last.
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
    st_d = torch.full((1,), 12345, dtype=torch.int32, device="cuda")
    rc = pd.lib().pd_celllist_build_static(code, ctypes.c_void_p(pos_d.data_ptr()), allp.shape[0], box_lo, sp, gs,
                                           v.pad, ctypes.c_void_p(cs_d.data_ptr()),
                                           ctypes.c_void_p(so_d.data_ptr()), ctypes.c_void_p(st_d.data_ptr()), None)
    torch.cuda.synchronize()
    assert int(st_d.item()) == 0  # every position inside the grid
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
    rc = L.pd_celllist_build_static(pd.PD_F64, dummy, (1 << 19) + 1, box_lo, sp, gs, 1, dummy, dummy, None, None)
    assert rc == -1
    assert b"static scratch limit" in L.pd_last_error()
    big = (ctypes.c_int * 3)(100, 100, 100)
    rc = L.pd_celllist_build_static(pd.PD_F64, dummy, 10, box_lo, sp, big, 1, dummy, dummy, None, None)
    assert rc == -1


def test_static_scratch_crowded_cells_and_status():
    """Clustered input with cells of more than 32 and more than 512 members keeps the
    stable in-cell order; a position outside the grid is reported in the status word."""
    import torch
    from openfpm_pdata_b200 import pd
    L = pd.lib()
    rng = np.random.default_rng(79)
    n = 30000
    # half uniform; a quarter in a tight ball (a cell of thousands) and a quarter in a wide
    # one (cells of tens to a few hundred)
    pos = np.concatenate([rng.uniform(0, 6.0, size=(n // 2, 3)), 4.5 + rng.normal(0, 0.05, size=(n // 4, 3)),
                          2.0 + rng.normal(0, 0.8, size=(n // 4, 3))])
    pos = np.clip(pos, 0.0, 6.0 - 1e-9)
    lo, hi, bc = np.zeros(3), np.full(3, 6.0), np.zeros(3, np.int32)
    vd = pd.VectorDist(n, lo, hi, bc, 0.5, dtype=np.float64)
    vd.hostToDevicePos(pos)
    cl = vd.getCellListGPU(0.5)
    vd.updateCellListGPU(cl)
    cs, so = cl.get()
    counts = np.diff(cs)
    assert counts.max() > 512 and ((counts > 32) & (counts <= 512)).any()
    v = cl.view()
    allp = vd.deviceToHostPos()
    for fill in (-1, 3):
        rc, cs2, so2 = _static_build(pd, torch, np.float64, allp, v, fill)
        assert rc == 0, L.pd_last_error()
        assert np.array_equal(cs2, cs) and np.array_equal(so2, so)
    # one position far outside the grid: clamped into a border cell and reported
    bad = allp.copy()
    bad[5] = (1e3, -1e3, 1e3)
    pos_d = torch.from_numpy(bad).cuda()
    cs_d = torch.zeros(v.ncells + 1, dtype=torch.int32, device="cuda")
    so_d = torch.zeros(bad.shape[0], dtype=torch.int32, device="cuda")
    st_d = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = L.pd_celllist_build_static(pd.PD_F64, ctypes.c_void_p(pos_d.data_ptr()), bad.shape[0],
                                    (ctypes.c_double * 3)(*v.box_lo), (ctypes.c_double * 3)(*v.spacing),
                                    (ctypes.c_int * 3)(*v.gs), v.pad, ctypes.c_void_p(cs_d.data_ptr()),
                                    ctypes.c_void_p(so_d.data_ptr()), ctypes.c_void_p(st_d.data_ptr()), None)
    torch.cuda.synchronize()
    assert rc == 0 and int(st_d.item()) == pd.PD_STATIC_OUT_OF_GRID
    # host buffers are refused before any launch
    h = np.zeros(4, np.int32)
    rc = L.pd_celllist_build_static(pd.PD_F64, ctypes.c_void_p(pos_d.data_ptr()), 4, (ctypes.c_double * 3)(*v.box_lo),
                                    (ctypes.c_double * 3)(*v.spacing), (ctypes.c_int * 3)(*v.gs), v.pad,
                                    h.ctypes.data_as(ctypes.c_void_p), ctypes.c_void_p(so_d.data_ptr()), None, None)
    assert rc == -1 and b"device memory" in L.pd_last_error()


def test_static_scratch_allocates_nothing():
    """After a first call on the device, further calls change neither the device's
    free memory nor the library's block cache, and give the allocating sort's
    outputs."""
    import torch
    from openfpm_pdata_b200 import pd
    L = pd.lib()
    allp, cs, so, v = _reference_and_geometry(pd, np.float64, 50000, 80)
    rc, _, _ = _static_build(pd, torch, np.float64, allp, v, -1)  # the first call on this device
    assert rc == 0
    pos_d = torch.from_numpy(np.ascontiguousarray(allp)).cuda()
    cs_d = torch.full((v.ncells + 1,), -1, dtype=torch.int32, device="cuda")
    so_d = torch.full((allp.shape[0],), -1, dtype=torch.int32, device="cuda")
    args = (pd.PD_F64, ctypes.c_void_p(pos_d.data_ptr()), allp.shape[0], (ctypes.c_double * 3)(*v.box_lo),
            (ctypes.c_double * 3)(*v.spacing), (ctypes.c_int * 3)(*v.gs), v.pad, ctypes.c_void_p(cs_d.data_ptr()),
            ctypes.c_void_p(so_d.data_ptr()), None, None)
    torch.cuda.synchronize()
    held0 = pd.set_cache_limit(-1)
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        cs_d.fill_(-1)
        so_d.fill_(-1)
        rc = L.pd_celllist_build_static(*args)
        torch.cuda.synchronize()
        assert rc == 0, L.pd_last_error()
        assert np.array_equal(cs_d.cpu().numpy(), cs) and np.array_equal(so_d.cpu().numpy(), so)
    assert pd.set_cache_limit(-1) == held0
    assert torch.cuda.mem_get_info()[0] == free0
