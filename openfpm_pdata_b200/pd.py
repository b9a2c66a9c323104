"""ctypes binding of libpdgpu.so, mirroring the reference's vector_dist GPU API.

Names follow the reference (Vector/vector_dist.hpp): ``map``,
``ghost_get``, ``getCellListGPU``, ``updateCellListGPU``, ``restoreOrder``,
``getVerlet``, ``updateVerlet``, ``getDomainIteratorGPU``, ``toKernel``,
``hostToDevicePos`` / ``deviceToHostPos`` and the property variants.  Errors
raise ``PdError`` carrying the library's message, like the reference's
ACTION_ON_ERROR.  There is no CPU fallback: importing this module on a host
without the built library raises.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpdgpu.so")

PD_F32, PD_F64, PD_I32, PD_U32, PD_I64 = 1, 2, 3, 4, 5
NON_PERIODIC, PERIODIC = 0, 1
NO_POSITION, WITH_POSITION, NO_CHANGE_ELEMENTS = 1, 2, 4
SKIP_LABELLING = KEEP_PROPERTIES = 512
RUN_ON_DEVICE = 1024
CL_SYMMETRIC, CL_NON_SYMMETRIC = 1, 2
CL_GPU_REORDER_POSITION, CL_GPU_REORDER_PROPERTY = 64, 128
CL_GPU_REORDER = CL_GPU_REORDER_POSITION | CL_GPU_REORDER_PROPERTY
RED_ADD, RED_MAX = 1, 2
PUT_ADD, PUT_MAX, PUT_REPLACE = 1, 2, 3
CMP_EQ, CMP_NE, CMP_LT, CMP_LE, CMP_GT, CMP_GE = range(6)
VTK_WRITER, CSV_WRITER, FORMAT_BINARY = 0, 1, 2
PD_STATIC_OUT_OF_GRID = 1  # status of pd_celllist_build_static: a position outside the grid

_NP = {PD_F32: np.float32, PD_F64: np.float64, PD_I32: np.int32, PD_U32: np.uint32, PD_I64: np.int64}
_CODES = {-1: "PD_EINVAL", -2: "PD_ENOMEM", -3: "PD_ECUDA", -4: "PD_ESTALE", -5: "PD_ETIMEOUT",
          -6: "PD_EOVERFLOW", -7: "PD_ESTATE", -8: "PD_EIO"}


class PdError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{_CODES.get(code, code)}: {msg}")
        self.code = code


class View(ctypes.Structure):
    _fields_ = [("pos", ctypes.c_void_p), ("prop", ctypes.c_void_p * 16), ("prop_type", ctypes.c_int * 16),
                ("prop_ncomp", ctypes.c_int * 16), ("n_prop", ctypes.c_int), ("dtype", ctypes.c_int),
                ("stride", ctypes.c_long), ("size_local", ctypes.c_long), ("size", ctypes.c_long),
                ("epoch", ctypes.c_long)]


class CLView(ctypes.Structure):
    _fields_ = [("cell_start", ctypes.c_void_p), ("sorted_ids", ctypes.c_void_p), ("dom_sort_ids", ctypes.c_void_p),
                ("ncells", ctypes.c_long), ("gs", ctypes.c_int * 3), ("div", ctypes.c_int * 3),
                ("pad", ctypes.c_int), ("nn_box", ctypes.c_int), ("box_lo", ctypes.c_double * 3),
                ("spacing", ctypes.c_double * 3), ("ghost_marker", ctypes.c_long), ("n_part", ctypes.c_long)]


class Launch(ctypes.Structure):
    _fields_ = [("wthr", ctypes.c_uint * 3), ("thr", ctypes.c_uint * 3)]


class LJParams(ctypes.Structure):
    _fields_ = [("eps", ctypes.c_double), ("sigma", ctypes.c_double), ("r_cut", ctypes.c_double)]


PREC_FP64, PREC_MIXED = 0, 1


class SPHParams(ctypes.Structure):
    _fields_ = [("h", ctypes.c_double), ("mass", ctypes.c_double), ("c0", ctypes.c_double),
                ("rho0", ctypes.c_double), ("alpha", ctypes.c_double), ("gz", ctypes.c_double),
                ("rho_prop", ctypes.c_int), ("drho_prop", ctypes.c_int), ("type_prop", ctypes.c_int)]


class SlabT(ctypes.Structure):
    """pd_slab_t: slab r of nslabs along `axis` is [lo + r w, lo + (r+1) w), w = (hi - lo) / nslabs."""
    _fields_ = [("axis", ctypes.c_int), ("nslabs", ctypes.c_int), ("periodic", ctypes.c_int),
                ("lo", ctypes.c_double), ("hi", ctypes.c_double), ("ghost", ctypes.c_double)]


class MDParams(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_double), ("mass", ctypes.c_double), ("skin", ctypes.c_double),
                ("vel_prop", ctypes.c_int), ("force_prop", ctypes.c_int), ("use_cell_list", ctypes.c_int),
                ("precision", ctypes.c_int)]


_lib = None


def lib():
    """Load libpdgpu.so; raises if it was not built (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
                              "(make -C openfpm_pdata_b200/csrc)")
        L = ctypes.CDLL(LIB_PATH)
        vp, lp, ip, dp = ctypes.c_void_p, ctypes.c_long, ctypes.c_int, ctypes.POINTER(ctypes.c_double)
        P = ctypes.POINTER
        sig = {
            "pd_last_error": ([], ctypes.c_char_p),
            "pd_device_info": ([P(ctypes.c_int), P(ctypes.c_long), P(ctypes.c_long)], ip),
            "pd_create": ([ip, ip, lp, dp, dp, P(ctypes.c_int), dp, ip, P(vp)], ip),
            "pd_destroy": ([vp], ip),
            "pd_add_prop": ([vp, ip, ip, P(ctypes.c_int)], ip),
            "pd_size": ([vp, P(ctypes.c_long), P(ctypes.c_long)], ip),
            "pd_resize": ([vp, lp], ip),
            "pd_h2d_pos": ([vp, vp, lp, lp, vp], ip),
            "pd_d2h_pos": ([vp, vp, lp, lp, vp], ip),
            "pd_h2d_prop": ([vp, ip, vp, lp, lp, vp], ip),
            "pd_d2h_prop": ([vp, ip, vp, lp, lp, vp], ip),
            "pd_map": ([vp, ip, vp], ip),
            "pd_ghost_get": ([vp, ctypes.c_ulong, ip, vp], ip),
            "pd_ghost_records": ([vp, vp, vp, lp, P(ctypes.c_long)], ip),
            "pd_ghost_count_boxes": ([vp, vp, vp, ip, vp, vp], ip),
            "pd_ghost_get_boxes": ([vp, vp, vp, ip, vp, ip, vp], ip),
            "pd_view": ([vp, P(View)], ip),
            "pd_domain_iterator": ([vp, ip, ip, P(Launch)], ip),
            "pd_reduce": ([vp, ip, ip, ip, vp, dp], ip),
            "pd_d2h_gid": ([vp, vp, lp, lp, vp], ip),
            "pd_celllist_create": ([vp, ctypes.c_double, ip, ip, ctypes.c_double, P(vp)], ip),
            "pd_celllist_destroy": ([vp], ip),
            "pd_celllist_update": ([vp, vp, ctypes.c_ulong, vp], ip),
            "pd_restore_order": ([vp, vp, ctypes.c_ulong, vp], ip),
            "pd_celllist_view": ([vp, P(CLView)], ip),
            "pd_celllist_get": ([vp, vp, vp, vp], ip),
            "pd_test_force": ([vp, vp, ip, ip, ip, vp], ip),
            "pd_verlet_create": ([vp, ctypes.c_double, P(vp)], ip),
            "pd_verlet_create_sym": ([vp, ctypes.c_double, P(vp)], ip),
            "pd_ghost_put": ([vp, ctypes.c_ulong, ip, vp], ip),
            "pd_ighost_get": ([vp, ctypes.c_ulong, ip, vp], ip),
            "pd_ghost_wait": ([vp, vp], ip),
            "pd_remove_marked": ([vp, ip, vp], ip),
            "pd_save": ([vp, ctypes.c_char_p], ip),
            "pd_selftest_wait": ([ctypes.c_long, ip, vp, vp], ip),
            "pd_measure_fma_rate": ([ip, P(ctypes.c_double)], ip),
            "pd_load": ([vp, ctypes.c_char_p], ip),
            "pd_write": ([vp, ctypes.c_char_p, ctypes.c_char_p, ip], ip),
            "pd_write_frame": ([vp, ctypes.c_char_p, ctypes.c_long, ctypes.c_char_p, ip], ip),
            "pd_get_indexes_by_type": ([vp, ip, ip, ctypes.c_longlong, ctypes.c_long, vp, ctypes.c_long,
                                        P(ctypes.c_long), vp], ip),
            "pd_verlet_destroy": ([vp], ip),
            "pd_verlet_update": ([vp, vp, vp], ip),
            "pd_verlet_get": ([vp, vp, vp, lp, vp], ip),
            "pd_lj_forces": ([vp, vp, vp, P(LJParams), ip, vp, dp], ip),
            "pd_md_create": ([vp, P(LJParams), P(MDParams), P(vp)], ip),
            "pd_md_destroy": ([vp], ip),
            "pd_md_run": ([vp, ip, vp, vp], ip),
            "pd_md_stats": ([vp, P(ctypes.c_long), P(ctypes.c_long), P(ctypes.c_int)], ip),
            "pd_md_set_timing": ([vp, ip], ip),
            "pd_md_timers": ([vp, P(ctypes.c_double), P(ctypes.c_long)], ip),
            "pd_launch_count": ([], ctypes.c_ulonglong),
            "pd_empty_cache": ([], ip),
            "pd_slab_halo": ([vp, lp, ip, ctypes.c_double, ctypes.c_double, vp, vp, P(ctypes.c_long),
                              P(ctypes.c_long), vp], ip),
            "pd_set_cache_limit": ([lp, P(ctypes.c_long)], ip),
            "pd_md_list_stats": ([vp, P(ctypes.c_long), P(ctypes.c_double), P(ctypes.c_int)], ip),
            "pd_md_launch_shape": ([vp, P(ctypes.c_int), P(ctypes.c_int), P(ctypes.c_int)], ip),
            "pd_celllist_build_static": ([ip, vp, lp, dp, dp, P(ctypes.c_int), ip, vp, vp, vp, vp], ip),
            "pd_slab_map_label": ([vp, P(SlabT), P(ctypes.c_long), vp], ip),
            "pd_slab_halo_label": ([vp, P(SlabT), ip, P(ctypes.c_long), vp], ip),
            "pd_slab_row_bytes": ([vp, ctypes.c_ulong, P(ctypes.c_long)], ip),
            "pd_slab_pack": ([vp, ctypes.c_ulong, vp, lp, vp], ip),
            "pd_slab_map_unpack": ([vp, ctypes.c_ulong, vp, lp, vp], ip),
            "pd_slab_halo_unpack": ([vp, ctypes.c_ulong, vp, lp, vp], ip),
            "pd_md_set_tiles": ([vp, ip, ip, ip], ip),
            "pd_md_set_block": ([vp, ip], ip),
            "pd_sph_create": ([vp, P(SPHParams), P(MDParams), P(vp)], ip),
            "pd_srv_create": ([lp, ip, P(LJParams), ctypes.c_double, ctypes.c_double, P(vp)], ip),
            "pd_srv_destroy": ([vp], ip),
            "pd_srv_set_tuning": ([vp, ip, ip, ip, ip], ip),
            "pd_srv_set_shape": ([vp, ip, ip, ip, ip], ip),
            "pd_srv_submit": ([vp, lp, ctypes.c_double, vp, vp, ip, P(ctypes.c_long)], ip),
            "pd_srv_tick": ([vp, P(ctypes.c_int), P(ctypes.c_int)], ip),
            "pd_srv_state": ([vp, lp, P(ctypes.c_int)], ip),
            "pd_srv_result": ([vp, lp, vp, vp, vp], ip),
            "pd_srv_release": ([vp, lp], ip),
            "pd_srv_stats": ([vp, P(ctypes.c_long), P(ctypes.c_long), P(ctypes.c_long), P(ctypes.c_long),
                              P(ctypes.c_double)], ip),
            "pd_srv_tuned": ([vp, vp, vp, vp, vp, ip, P(ctypes.c_int)], ip),
            "pd_srv_timers": ([vp, vp], ip),
            "pd_srv_completed": ([vp, vp, ip, P(ctypes.c_int)], ip),
            "pd_gen_clustered": ([lp, ctypes.c_double, ip, ctypes.c_double, ctypes.c_double, ctypes.c_ulong, ip, vp,
                                  P(ctypes.c_long)], ip),
            "pd_selftest_recip": ([ip, vp, vp, lp], ip),
            "pd_md_verlet_get": ([vp, vp, vp, lp, P(ctypes.c_int)], ip),
        }
        for name, (args, res) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def check(rc):
    if rc != 0:
        raise PdError(rc, lib().pd_last_error().decode(errors="replace"))
    return rc


def _d3(x):
    a = (ctypes.c_double * 3)(*[float(v) for v in np.broadcast_to(np.asarray(x, dtype=np.float64), (3,))])
    return a


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _is_cuda_tensor(a):
    return getattr(a, "is_cuda", False) and hasattr(a, "data_ptr")


def _check_tensor(a, dtype):
    import torch
    want = torch.float64 if np.dtype(dtype) == np.float64 else torch.float32
    if a.dtype != want:
        raise TypeError("tensor of %s expected, got %s" % (want, a.dtype))


def launch_count():
    """Kernels launched by libpdgpu.so so far."""
    return int(lib().pd_launch_count())


def empty_cache():
    """Return the device blocks the library keeps for reuse to the driver."""
    check(lib().pd_empty_cache())


def slab_halo(x, axis, lo_thr, hi_thr):
    """Halo selection of a slab on a CUDA tensor of positions [n, 3] (float64):
    (ascending indices with x[:, axis] < lo_thr, those with x[:, axis] >= hi_thr)
    as int64 CUDA tensors, computed by the library."""
    import torch
    x = x.contiguous()
    _check_tensor(x, np.float64)
    n = x.shape[0]
    lo = torch.empty(max(n, 1), dtype=torch.int32, device=x.device)
    hi = torch.empty(max(n, 1), dtype=torch.int32, device=x.device)
    a, b = ctypes.c_long(0), ctypes.c_long(0)
    check(lib().pd_slab_halo(ctypes.c_void_p(x.data_ptr()), int(n), int(axis), float(lo_thr), float(hi_thr),
                             ctypes.c_void_p(lo.data_ptr()), ctypes.c_void_p(hi.data_ptr()), ctypes.byref(a),
                             ctypes.byref(b), None))
    return lo[: a.value].to(torch.int64), hi[: b.value].to(torch.int64)


def set_cache_limit(limit_bytes=-1):
    """Set the limit of the device block cache (-1: unchanged); returns the bytes held."""
    held = ctypes.c_long(0)
    check(lib().pd_set_cache_limit(int(limit_bytes), ctypes.byref(held)))
    return held.value


def selftest_recip(x):
    """The pair kernels' reciprocal evaluated on the GPU for the values x."""
    x = np.ascontiguousarray(x)
    code = PD_F64 if x.dtype == np.float64 else PD_F32
    out = np.zeros_like(x)
    check(lib().pd_selftest_recip(code, _ptr(x), _ptr(out), int(x.size)))
    return out


def device_info():
    sm, fr, tot = ctypes.c_int(0), ctypes.c_long(0), ctypes.c_long(0)
    check(lib().pd_device_info(ctypes.byref(sm), ctypes.byref(fr), ctypes.byref(tot)))
    return sm.value, fr.value, tot.value


class CellList:
    """CellList_gpu handle (getCellListGPU / updateCellListGPU / restoreOrder)."""

    def __init__(self, vd, r_cut, opt=CL_NON_SYMMETRIC, nn_box=1, enlarge=None):
        self.vd = vd
        h = ctypes.c_void_p()
        enl = float(np.float32(1.013)) if enlarge is None else float(enlarge)
        check(lib().pd_celllist_create(vd.h, float(r_cut), int(opt), int(nn_box), enl, ctypes.byref(h)))
        self.h = h

    def view(self):
        v = CLView()
        check(lib().pd_celllist_view(self.h, ctypes.byref(v)))
        return v

    def get(self):
        """(cell_start[ncells+1], sorted_ids[n]) on the host."""
        v = self.view()
        cs = np.zeros(v.ncells + 1, np.int32)
        so = np.zeros(max(v.n_part, 1), np.int32)
        check(lib().pd_celllist_get(self.h, _ptr(cs), _ptr(so), None))
        return cs, so[: v.n_part]

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.pd_celllist_destroy(self.h)
            self.h = None


class VerletList:
    """VerletList handle (getVerlet / updateVerlet)."""

    def __init__(self, vd, r_cut, sym=False):
        self.vd = vd
        self.sym = bool(sym)
        h = ctypes.c_void_p()
        create = lib().pd_verlet_create_sym if sym else lib().pd_verlet_create
        check(create(vd.h, float(r_cut), ctypes.byref(h)))
        self.h = h

    def get(self):
        """CSR (offsets[n+1], idx) of the list on the host."""
        n = self.vd.size_local()
        counts = np.zeros(max(n, 1), np.int32)
        check(lib().pd_verlet_get(self.h, _ptr(counts), None, 0, None))
        counts = counts[:n]
        off = np.zeros(n + 1, np.int64)
        off[1:] = np.cumsum(counts)
        idx = np.zeros(max(int(off[-1]), 1), np.int32)
        check(lib().pd_verlet_get(self.h, _ptr(counts), _ptr(idx), int(idx.shape[0]), None))
        return off, idx[: off[-1]]

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.pd_verlet_destroy(self.h)
            self.h = None


def _prop_table(path):
    """(type, ncomp) list of a checkpoint file (the header layout of pd_save)."""
    with open(path, "rb") as f:
        head = f.read(120)
        nprops = int(np.frombuffer(head[8:24], np.uint32)[3])
        t = np.frombuffer(f.read(8 * nprops), np.int32).reshape(-1, 2)
    return [(int(a), int(b)) for a, b in t]


class VectorDist:
    """vector_dist_gpu<3, St, aggregate<...>> on one GPU.

    ``props`` is a list of (type, ncomp) with type in PD_F32/PD_F64/PD_I32/PD_U32/PD_I64.
    """

    def __init__(self, n, lo, hi, bc, ghost, dtype=np.float64, props=()):
        self.dtype = np.dtype(dtype)
        code = PD_F64 if self.dtype == np.float64 else PD_F32
        bcs = (ctypes.c_int * 3)(*[int(b) for b in np.broadcast_to(np.asarray(bc), (3,))])
        h = ctypes.c_void_p()
        check(lib().pd_create(3, code, int(n), _d3(lo), _d3(hi), bcs, _d3(ghost), 0, ctypes.byref(h)))
        self.h = h
        self.props = []
        for t, nc in props:
            self.add_prop(t, nc)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.pd_destroy(self.h)
            self.h = None

    def add_prop(self, t, ncomp):
        pid = ctypes.c_int(-1)
        check(lib().pd_add_prop(self.h, int(t), int(ncomp), ctypes.byref(pid)))
        self.props.append((t, ncomp))
        return pid.value

    def size_local(self):
        a, b = ctypes.c_long(0), ctypes.c_long(0)
        check(lib().pd_size(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value

    def size_local_with_ghost(self):
        a, b = ctypes.c_long(0), ctypes.c_long(0)
        check(lib().pd_size(self.h, ctypes.byref(a), ctypes.byref(b)))
        return b.value

    def resize(self, n):
        check(lib().pd_resize(self.h, int(n)))

    # -- host <-> device
    def hostToDevicePos(self, x, offset=0):
        """positions [n][3] from a host array, or from a CUDA tensor of the
        vector's dtype without a host round trip"""
        if _is_cuda_tensor(x):
            x = x.contiguous().reshape(-1, 3)
            _check_tensor(x, self.dtype)
            check(lib().pd_h2d_pos(self.h, ctypes.c_void_p(x.data_ptr()), int(offset), int(x.shape[0]), None))
            return
        x = np.ascontiguousarray(x, dtype=self.dtype).reshape(-1, 3)
        check(lib().pd_h2d_pos(self.h, _ptr(x), int(offset), int(x.shape[0]), None))

    def deviceToHostPos(self, offset=0, count=None, with_ghost=True, out=None, device=False):
        """positions [n][3]; `out` (e.g. pinned memory) receives them when given;
        device=True returns a CUDA tensor (copied on the GPU)"""
        n = (self.size_local_with_ghost() if with_ghost else self.size_local()) - offset if count is None else count
        if device:
            import torch
            t = torch.empty((max(n, 0), 3), dtype=torch.float64 if self.dtype == np.float64 else torch.float32,
                            device="cuda")
            if n:
                check(lib().pd_d2h_pos(self.h, ctypes.c_void_p(t.data_ptr()), int(offset), int(n), None))
            return t
        if out is None:
            out = np.zeros((n, 3), self.dtype)
        elif out.dtype != self.dtype or not out.flags.c_contiguous or out.size < 3 * n:
            raise ValueError("deviceToHostPos: out must be C-contiguous, of the vector's dtype, with room for n x 3")
        if n:
            check(lib().pd_d2h_pos(self.h, _ptr(out), int(offset), int(n), None))
        return out

    def hostToDeviceProp(self, p, a, offset=0):
        """property p from [n] or [n][ncomp] host data, or from a CUDA tensor of the
        property's type (transposed on the GPU, no host round trip)"""
        t, nc = self.props[p]
        if _is_cuda_tensor(a):
            import torch
            want = getattr(torch, np.dtype(_NP[t]).name)
            if a.dtype != want:
                raise TypeError(f"hostToDeviceProp: a {want} tensor is expected, got {a.dtype}")
            cm = a.reshape(-1, nc).t().contiguous()
            check(lib().pd_h2d_prop(self.h, int(p), ctypes.c_void_p(cm.data_ptr()), int(offset), int(cm.shape[1]),
                                    None))
            return
        a = np.asarray(a, dtype=_NP[t]).reshape(-1, nc)
        cm = np.ascontiguousarray(a.T)
        check(lib().pd_h2d_prop(self.h, int(p), _ptr(cm), int(offset), int(a.shape[0]), None))

    def hostToDevicePropSoA(self, p, cm, offset=0):
        """property p from component-major host data [ncomp][n] (the ABI's layout: no
        transpose, so pinned memory is copied directly)"""
        t, nc = self.props[p]
        if cm.dtype != _NP[t] or not cm.flags.c_contiguous or cm.shape[0] != nc:
            raise ValueError("hostToDevicePropSoA: C-contiguous [ncomp][n] array of the property's type expected")
        check(lib().pd_h2d_prop(self.h, int(p), _ptr(cm), int(offset), int(cm.shape[1]), None))

    def deviceToHostPropSoA(self, p, out=None, offset=0, count=None, with_ghost=True):
        """property p as component-major [ncomp][n] (into `out` when given)"""
        t, nc = self.props[p]
        n = (self.size_local_with_ghost() if with_ghost else self.size_local()) - offset if count is None else count
        if out is None:
            out = np.zeros((nc, n), _NP[t])
        elif out.dtype != _NP[t] or not out.flags.c_contiguous or out.shape != (nc, n):
            raise ValueError("deviceToHostPropSoA: C-contiguous [ncomp][n] output of the property's type expected")
        if n:
            check(lib().pd_d2h_prop(self.h, int(p), _ptr(out), int(offset), int(n), None))
        return out

    def deviceToHostProp(self, p, offset=0, count=None, with_ghost=True, device=False):
        """property p as [n] or [n][ncomp]; device=True returns a CUDA tensor
        (copied on the GPU, no host round trip)"""
        t, nc = self.props[p]
        n = (self.size_local_with_ghost() if with_ghost else self.size_local()) - offset if count is None else count
        if device:
            import torch
            cm = torch.empty((nc, max(n, 0)), dtype=getattr(torch, np.dtype(_NP[t]).name), device="cuda")
            if n:
                check(lib().pd_d2h_prop(self.h, int(p), ctypes.c_void_p(cm.data_ptr()), int(offset), int(n), None))
            return cm.t().contiguous() if nc > 1 else cm[0].clone()
        cm = np.zeros((nc, n), _NP[t])
        if n:
            check(lib().pd_d2h_prop(self.h, int(p), _ptr(cm), int(offset), int(n), None))
        return cm.T.copy() if nc > 1 else cm[0].copy()

    def gid(self, with_ghost=True):
        n = self.size_local_with_ghost() if with_ghost else self.size_local()
        out = np.zeros(max(n, 1), np.int64)
        check(lib().pd_d2h_gid(self.h, _ptr(out), 0, int(n), None))
        return out[:n]

    # -- slab decomposition over ranks (pd_slab_*): label, pack, (transport), unpack
    def slab_map_label(self, slab):
        """map labelling: the rows per destination rank (a list)."""
        c = (ctypes.c_long * slab.nslabs)()
        check(lib().pd_slab_map_label(self.h, ctypes.byref(slab), c, None))
        return list(c)

    def slab_halo_label(self, slab, rank):
        """ghost_get labelling of `rank`: the halo rows per destination rank (a list)."""
        c = (ctypes.c_long * slab.nslabs)()
        check(lib().pd_slab_halo_label(self.h, ctypes.byref(slab), int(rank), c, None))
        return list(c)

    def slab_row_bytes(self, mask):
        b = ctypes.c_long(0)
        check(lib().pd_slab_row_bytes(self.h, ctypes.c_ulong(mask), ctypes.byref(b)))
        return b.value

    def slab_pack(self, mask, rows):
        """the labelled rows packed into a new CUDA uint8 tensor [rows * row_bytes]"""
        import torch
        out = torch.empty(max(rows * self.slab_row_bytes(mask), 1), dtype=torch.uint8, device="cuda")
        check(lib().pd_slab_pack(self.h, ctypes.c_ulong(mask), ctypes.c_void_p(out.data_ptr()), int(rows), None))
        return out[: rows * self.slab_row_bytes(mask)]

    def slab_map_unpack(self, mask, recv, n):
        check(lib().pd_slab_map_unpack(self.h, ctypes.c_ulong(mask), ctypes.c_void_p(recv.data_ptr() if n else 0),
                                       int(n), None))

    def slab_halo_unpack(self, mask, recv, n):
        check(lib().pd_slab_halo_unpack(self.h, ctypes.c_ulong(mask), ctypes.c_void_p(recv.data_ptr() if n else 0),
                                        int(n), None))

    # -- reference API
    def map(self, opt=RUN_ON_DEVICE):
        check(lib().pd_map(self.h, int(opt), None))

    def ghost_get(self, props=None, opt=RUN_ON_DEVICE):
        mask = (1 << 64) - 1 if props is None else sum(1 << p for p in props)
        check(lib().pd_ghost_get(self.h, ctypes.c_ulong(mask), int(opt), None))

    def Ighost_get(self, props=None, opt=RUN_ON_DEVICE, stream=None):
        """Ighost_get<prp...>(opt): enqueue the ghost exchange without waiting for it."""
        mask = (1 << 64) - 1 if props is None else sum(1 << p for p in props)
        check(lib().pd_ighost_get(self.h, ctypes.c_ulong(mask), int(opt), stream))

    def ghost_wait(self, stream=None):
        check(lib().pd_ghost_wait(self.h, stream))

    def ghost_put(self, props=None, op=PUT_ADD):
        """ghost_put<op_, prp...>(): merge every ghost's values onto its source."""
        mask = (1 << 64) - 1 if props is None else sum(1 << p for p in props)
        check(lib().pd_ghost_put(self.h, ctypes.c_ulong(mask), int(op), None))

    def ghost_records(self):
        n = ctypes.c_long(0)
        check(lib().pd_ghost_records(self.h, None, None, 0, ctypes.byref(n)))
        m = n.value
        src = np.zeros(max(m, 1), np.int32)
        shf = np.zeros(max(m, 1), np.int32)
        check(lib().pd_ghost_records(self.h, _ptr(src), _ptr(shf), m, ctypes.byref(n)))
        return src[:m], shf[:m]

    def ghost_count_boxes(self, blo, bhi, sv):
        nb = len(sv)
        boxes = np.ascontiguousarray(np.concatenate([np.asarray(blo, np.float64).reshape(nb, 3),
                                                     np.asarray(bhi, np.float64).reshape(nb, 3)], axis=1))
        svv = np.ascontiguousarray(sv, np.int32)
        out = np.zeros(max(self.size_local(), 1), np.int32)
        check(lib().pd_ghost_count_boxes(self.h, _ptr(boxes), _ptr(svv), nb, _ptr(out), None))
        return out[: self.size_local()]

    def ghost_get_boxes(self, blo, bhi, sv, shifts):
        nb = len(sv)
        boxes = np.ascontiguousarray(np.concatenate([np.asarray(blo, np.float64).reshape(nb, 3),
                                                     np.asarray(bhi, np.float64).reshape(nb, 3)], axis=1))
        svv = np.ascontiguousarray(sv, np.int32)
        sh = np.ascontiguousarray(shifts, np.float64).reshape(-1, 3)
        check(lib().pd_ghost_get_boxes(self.h, _ptr(boxes), _ptr(svv), nb, _ptr(sh), sh.shape[0], None))

    def toKernel(self):
        v = View()
        check(lib().pd_view(self.h, ctypes.byref(v)))
        return v

    def getDomainIteratorGPU(self, n_thr=1024, with_ghost=False):
        it = Launch()
        check(lib().pd_domain_iterator(self.h, int(n_thr), int(with_ghost), ctypes.byref(it)))
        return it

    def remove_marked(self, p):
        """remove_marked<p>(): drop the domain particles whose property p is non-zero."""
        check(lib().pd_remove_marked(self.h, int(p), None))

    def get_indexes_by_type(self, p, value, cmp=CMP_EQ, end=None, device=False):
        """get_indexes_by_type<p, functor>(): ascending indexes i < end with prop p `cmp` value;
        device=True returns them in a CUDA int32 tensor (device memory, as the reference's
        vector_gpu), else in a host uint32 array."""
        n = ctypes.c_long(0)
        e = -1 if end is None else int(end)
        cap = self.size_local_with_ghost()
        if device:
            import torch
            t = torch.empty(max(cap, 1), dtype=torch.int32, device="cuda")
            check(lib().pd_get_indexes_by_type(self.h, int(p), int(cmp), int(value), e,
                                               ctypes.c_void_p(t.data_ptr()), cap, ctypes.byref(n), None))
            return t[: n.value]
        ids = np.zeros(max(cap, 1), np.uint32)
        check(lib().pd_get_indexes_by_type(self.h, int(p), int(cmp), int(value), e, _ptr(ids), cap,
                                           ctypes.byref(n), None))
        return ids[: n.value]

    def save(self, path):
        """save(filename): domain particles to a checksummed binary checkpoint."""
        check(lib().pd_save(self.h, os.fsencode(path)))

    def load(self, path):
        """load(filename): replace the particles by a checkpoint's (properties added if none)."""
        check(lib().pd_load(self.h, os.fsencode(path)))
        if not self.props:
            self.props = _prop_table(path)

    def write(self, out, meta="", opt=VTK_WRITER):
        check(lib().pd_write(self.h, os.fsencode(out), meta.encode(), int(opt)))

    def write_frame(self, out, iteration, meta="", opt=VTK_WRITER):
        check(lib().pd_write_frame(self.h, os.fsencode(out), int(iteration), meta.encode(), int(opt)))

    def reduce_local(self, p, comp=0, op=RED_ADD):
        out = ctypes.c_double(0)
        check(lib().pd_reduce(self.h, int(p), int(comp), int(op), None, ctypes.byref(out)))
        return out.value

    def getCellListGPU(self, r_cut, opt=CL_NON_SYMMETRIC, NNIteratorBox=1, ghostEnlargeFactor=None):
        return CellList(self, r_cut, opt, NNIteratorBox, ghostEnlargeFactor)

    def getCellListSym(self, r_cut):
        return CellList(self, r_cut, CL_SYMMETRIC)

    def updateCellListGPU(self, cl, props=None):
        mask = (1 << 64) - 1 if props is None else sum(1 << p for p in props)
        check(lib().pd_celllist_update(self.h, cl.h, ctypes.c_ulong(mask), None))

    def restoreOrder(self, cl, props=None):
        mask = (1 << 64) - 1 if props is None else sum(1 << p for p in props)
        check(lib().pd_restore_order(self.h, cl.h, ctypes.c_ulong(mask), None))

    def getVerlet(self, r_cut):
        vl = VerletList(self, r_cut)
        check(lib().pd_verlet_update(self.h, vl.h, None))
        return vl

    def getVerletSym(self, r_cut):
        vl = VerletList(self, r_cut, sym=True)
        check(lib().pd_verlet_update(self.h, vl.h, None))
        return vl

    def updateVerlet(self, vl):
        check(lib().pd_verlet_update(self.h, vl.h, None))

    def test_force(self, cl, in_prop, out_prop, sorted=False):
        check(lib().pd_test_force(self.h, cl.h, int(in_prop), int(out_prop), int(bool(sorted)), None))

    def lj_forces(self, force_prop, vl=None, cl=None, eps=1.0, sigma=1.0, r_cut=2.5):
        p = LJParams(eps, sigma, r_cut)
        e = (ctypes.c_double * 2)()
        check(lib().pd_lj_forces(self.h, vl.h if vl else None, cl.h if cl else None, ctypes.byref(p),
                                 int(force_prop), None, e))
        return e[0], e[1]


class MD:
    """Velocity-Verlet LJ driver over a VectorDist holding only real particles."""

    def __init__(self, vd, vel_prop, force_prop, dt=0.005, mass=1.0, skin=0.3, eps=1.0, sigma=1.0, r_cut=2.5,
                 use_cell_list=False, precision=PREC_FP64):
        self.vd = vd
        self.lj = LJParams(eps, sigma, r_cut)
        self.mp = MDParams(dt, mass, skin, vel_prop, force_prop, int(bool(use_cell_list)), int(precision))
        h = ctypes.c_void_p()
        check(lib().pd_md_create(vd.h, ctypes.byref(self.lj), ctypes.byref(self.mp), ctypes.byref(h)))
        self.h = h

    def run(self, steps, energies=True):
        E = np.zeros((max(steps, 1), 4)) if energies else None
        check(lib().pd_md_run(self.h, int(steps), None, _ptr(E) if energies else None))
        return E[:steps] if energies else None

    def set_timing(self, on=True):
        check(lib().pd_md_set_timing(self.h, int(bool(on))))

    def timers(self):
        """{phase: (total ms, count)} for integrate, rebuild, images, force."""
        ms = (ctypes.c_double * 4)()
        cnt = (ctypes.c_long * 4)()
        check(lib().pd_md_timers(self.h, ms, cnt))
        return {k: (ms[i], cnt[i]) for i, k in enumerate(("integrate", "rebuild", "images", "force"))}

    def set_tiles(self, on=True, tx=0, threads_per_particle=0):
        check(lib().pd_md_set_tiles(self.h, int(bool(on)), int(tx), int(threads_per_particle)))

    def set_block(self, threads):
        """Threads per CTA (256 or 128) of the precision form's pair kernel."""
        check(lib().pd_md_set_block(self.h, int(threads)))

    def verlet(self):
        """(offsets, idx, tiled) of the driver's current Verlet rows (global indices)."""
        n = self.vd.size_local()
        counts = np.zeros(max(n, 1), np.int32)
        tiled = ctypes.c_int(0)
        check(lib().pd_md_verlet_get(self.h, _ptr(counts), None, 0, ctypes.byref(tiled)))
        off = np.zeros(n + 1, np.int64)
        off[1:] = np.cumsum(counts[:n])
        idx = np.zeros(max(int(off[-1]), 1), np.int32)
        check(lib().pd_md_verlet_get(self.h, _ptr(counts), _ptr(idx), int(idx.shape[0]), ctypes.byref(tiled)))
        return off, idx[: off[-1]], bool(tiled.value)

    def list_stats(self):
        """(domain particles, mean Verlet row length, longest row) of the last build."""
        n, m, x = ctypes.c_long(0), ctypes.c_double(0), ctypes.c_int(0)
        check(lib().pd_md_list_stats(self.h, ctypes.byref(n), ctypes.byref(m), ctypes.byref(x)))
        return n.value, m.value, x.value

    def launch_shape(self):
        """{cluster_ctas, tile_tx, threads_per_particle} of the driver's kernels (see pdgpu.h)."""
        c, t, p = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
        check(lib().pd_md_launch_shape(self.h, ctypes.byref(c), ctypes.byref(t), ctypes.byref(p)))
        return {"cluster_ctas": c.value, "tile_tx": t.value, "threads_per_particle": p.value}

    def stats(self):
        b, s, e = ctypes.c_long(0), ctypes.c_long(0), ctypes.c_int(0)
        check(lib().pd_md_stats(self.h, ctypes.byref(b), ctypes.byref(s), ctypes.byref(e)))
        return b.value, s.value, e.value

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.pd_md_destroy(self.h)
            self.h = None


class SPH(MD):
    """WCSPH driver: props of `vd` are velocity (vel_prop), acceleration
    (acc_prop), density, density rate and type (0 fluid, 1 wall)."""

    def __init__(self, vd, vel_prop, acc_prop, rho_prop, drho_prop, type_prop, h, mass, c0=20.0, rho0=1000.0,
                 alpha=0.1, gz=-9.81, dt=1e-4, skin=0.0):
        self.vd = vd
        self.sp = SPHParams(h, mass, c0, rho0, alpha, gz, rho_prop, drho_prop, type_prop)
        self.mp = MDParams(dt, mass, skin, vel_prop, acc_prop, 0, PREC_FP64)
        hh = ctypes.c_void_p()
        check(lib().pd_sph_create(vd.h, ctypes.byref(self.sp), ctypes.byref(self.mp), ctypes.byref(hh)))
        self.h = hh


class Server:
    """Serving loop: independent periodic LJ systems batched on one GPU."""

    QUEUED, RUNNING, DONE, FAILED = 0, 1, 2, 3

    def __init__(self, hbm_budget_bytes, max_slots=64, dt=0.005, skin=0.3, eps=1.0, sigma=1.0, r_cut=2.5,
                 autotune=True, tx=0, lanes=2, block=256):
        self.lj = LJParams(eps, sigma, r_cut)
        h = ctypes.c_void_p()
        check(lib().pd_srv_create(int(hbm_budget_bytes), int(max_slots), ctypes.byref(self.lj), float(dt),
                                  float(skin), ctypes.byref(h)))
        self.h = h
        self.info = {}
        check(lib().pd_srv_set_tuning(self.h, int(bool(autotune)), int(tx), int(lanes), int(block)))

    def set_shape(self, bucket, tx, lanes, block):
        """The force kernel's launch shape for systems of size bucket floor(log2 N)."""
        check(lib().pd_srv_set_shape(self.h, int(bucket), int(tx), int(lanes), int(block)))

    def submit(self, x, v, box, steps):
        x = np.ascontiguousarray(x, np.float64)
        v = np.ascontiguousarray(v, np.float64)
        t = ctypes.c_long(0)
        check(lib().pd_srv_submit(self.h, x.shape[0], float(box), _ptr(x), _ptr(v), int(steps), ctypes.byref(t)))
        self.info[t.value] = (x.shape[0], int(steps))
        return t.value

    def tick(self):
        a, q = ctypes.c_int(0), ctypes.c_int(0)
        check(lib().pd_srv_tick(self.h, ctypes.byref(a), ctypes.byref(q)))
        return a.value, q.value

    def state(self, ticket):
        st = ctypes.c_int(0)
        check(lib().pd_srv_state(self.h, int(ticket), ctypes.byref(st)))
        return st.value

    def result(self, ticket):
        """(x_final[N,3] in submission order, E[steps,4], (t_submit, t_admit, t_done))."""
        n, steps = self.info[ticket]
        x = np.zeros((n, 3))
        E = np.zeros((steps, 4))
        t = np.zeros(3)
        check(lib().pd_srv_result(self.h, int(ticket), _ptr(x), _ptr(E), _ptr(t)))
        return x, E, tuple(t)

    def release(self, ticket):
        check(lib().pd_srv_release(self.h, int(ticket)))
        self.info.pop(ticket, None)

    def stats(self):
        ps, sd, tk, rb, tm = ctypes.c_long(0), ctypes.c_long(0), ctypes.c_long(0), ctypes.c_long(0), ctypes.c_double(0)
        check(lib().pd_srv_stats(self.h, ctypes.byref(ps), ctypes.byref(sd), ctypes.byref(tk), ctypes.byref(rb),
                                 ctypes.byref(tm)))
        return {"particle_steps": ps.value, "systems_done": sd.value, "ticks": tk.value, "rebuilds": rb.value,
                "tune_ms": tm.value}

    def timers(self):
        """Host wall ms spent in admission (and its slot-reset part), batched steps and retirement."""
        ms = np.zeros(4)
        check(lib().pd_srv_timers(self.h, _ptr(ms)))
        return dict(zip(("admit", "admit_reset", "step", "retire"), ms.tolist()))

    def completed(self, cap=4096):
        """Tickets finished (done or failed) since the last call."""
        out = np.zeros(cap, np.int64)
        n = ctypes.c_int(0)
        check(lib().pd_srv_completed(self.h, _ptr(out), int(cap), ctypes.byref(n)))
        return out[: n.value].tolist()

    def tuned(self):
        """size bucket -> (tile width, lanes per particle, threads per CTA) of the force kernel"""
        b, w, l, k = (np.zeros(64, np.int32) for _ in range(4))
        n = ctypes.c_int(0)
        check(lib().pd_srv_tuned(self.h, _ptr(b), _ptr(w), _ptr(l), _ptr(k), 64, ctypes.byref(n)))
        m = n.value
        return {int(b[i]): (int(w[i]), int(l[i]), int(k[i])) for i in range(m)}

    def run_until_done(self, tickets, max_ticks=100000):
        for _ in range(max_ticks):
            if all(self.state(t) in (self.DONE, self.FAILED) for t in tickets):
                return
            self.tick()
        raise RuntimeError("serving loop did not finish")

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.pd_srv_destroy(self.h)
            self.h = None


def selftest_wait(limit, issue_copy):
    """Bounded-wait self test: (status code, the 4 floats copied through shared memory)."""
    a = np.array([1.5, -2.25, 3.0, 4.75], np.float32)
    out = np.zeros(4, np.float32)
    rc = lib().pd_selftest_wait(int(limit), int(bool(issue_copy)), _ptr(a), _ptr(out))
    return rc, out


def measure_fma_rate(dtype):
    """Measured vector FMA throughput in TFLOP/s (PD_F32 or PD_F64; an FMA is two flops)."""
    out = ctypes.c_double(0)
    check(lib().pd_measure_fma_rate(int(dtype), ctypes.byref(out)))
    return out.value
