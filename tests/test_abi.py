"""Host-side checks that need no GPU: libpdgpu.so loads, exports every entry
point declared in include/*.h, and rejects bad arguments before any launch."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?(?:unsigned\s+)?(?:long\s+)?(?:int|void|char|long|double)\s*\**\s*(pd_\w+)\s*\(", src, re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert len(names) >= 30
    for must in ("pd_create", "pd_map", "pd_ghost_get", "pd_celllist_update", "pd_restore_order",
                 "pd_verlet_update", "pd_lj_forces", "pd_md_run"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from openfpm_pdata_b200 import pd
    L = pd.lib()
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, missing


def test_bad_arguments_rejected_without_gpu():
    from openfpm_pdata_b200 import pd
    L = pd.lib()
    h = ctypes.c_void_p()
    lo = (ctypes.c_double * 3)(0, 0, 0)
    hi = (ctypes.c_double * 3)(1, 1, 1)
    g = (ctypes.c_double * 3)(0.1, 0.1, 0.1)
    bc = (ctypes.c_int * 3)(1, 1, 1)
    assert L.pd_create(2, pd.PD_F64, 10, lo, hi, bc, g, 0, ctypes.byref(h)) == -1   # dim must be 3
    assert L.pd_create(3, 7, 10, lo, hi, bc, g, 0, ctypes.byref(h)) == -1           # dtype
    bad_hi = (ctypes.c_double * 3)(1, 0, 1)
    assert L.pd_create(3, pd.PD_F64, 10, lo, bad_hi, bc, g, 0, ctypes.byref(h)) == -1
    assert L.pd_destroy(None) == -1
    assert L.pd_map(None, 0, None) == -1
    assert b"invalid" in L.pd_last_error()
    # the device block cache: nothing held, emptying it makes no CUDA call
    held = ctypes.c_long(-1)
    assert L.pd_set_cache_limit(ctypes.c_long(-1), ctypes.byref(held)) == 0 and held.value == 0
    assert L.pd_empty_cache() == 0
    # serving entry points refuse a null server
    t = ctypes.c_long(0)
    assert L.pd_srv_submit(None, ctypes.c_long(10), ctypes.c_double(10.0), None, None, 5, ctypes.byref(t)) == -1
    assert L.pd_srv_result(None, ctypes.c_long(0), None, None, None) == -1
    assert L.pd_srv_release(None, ctypes.c_long(0)) == -1
    # the slab halo selection refuses positions that are not in device memory
    import numpy as np
    x = np.zeros((4, 3))
    a, b = ctypes.c_long(0), ctypes.c_long(0)
    assert L.pd_slab_halo(x.ctypes.data_as(ctypes.c_void_p), ctypes.c_long(4), 0, ctypes.c_double(1.0),
                          ctypes.c_double(2.0), None, None, ctypes.byref(a), ctypes.byref(b), None) == -1
    assert L.pd_slab_halo(None, ctypes.c_long(4), 0, ctypes.c_double(1.0), ctypes.c_double(2.0), None, None,
                          ctypes.byref(a), ctypes.byref(b), None) == -1
    # the no-allocation cell-list build refuses host buffers before any launch
    cs = np.zeros(1001, np.int32)
    so = np.zeros(4, np.int32)
    box_lo = (ctypes.c_double * 3)(0, 0, 0)
    sp = (ctypes.c_double * 3)(0.1, 0.1, 0.1)
    gs = (ctypes.c_int * 3)(10, 10, 10)
    assert L.pd_celllist_build_static(pd.PD_F64, x.ctypes.data_as(ctypes.c_void_p), ctypes.c_long(4), box_lo, sp,
                                      gs, 1, cs.ctypes.data_as(ctypes.c_void_p), so.ctypes.data_as(ctypes.c_void_p),
                                      None, None) == -1
    assert b"pd_celllist_build_static" in L.pd_last_error()


def test_package_fails_loudly_without_library(tmp_path, monkeypatch):
    from openfpm_pdata_b200 import pd
    monkeypatch.setattr(pd, "LIB_PATH", str(tmp_path / "missing.so"))
    monkeypatch.setattr(pd, "_lib", None)
    with pytest.raises(ImportError):
        pd.lib()
