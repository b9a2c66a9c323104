"""numpy front end of the CPU oracle (test infrastructure only).

Only the tests, the smoke entry point and bench.py's CPU-baseline leg import
this module; it is the checker, never the thing measured or shipped.  It
loads ``oracle/liboracle.so`` (built by ``oracle/Makefile``) and exposes the
restated reference algorithms with numpy arrays.  Every function names the
reference code it restates in ``pd_oracle.cpp``.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_lp = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_L = ctypes.c_long
_I = ctypes.c_int
_D = ctypes.c_double
_F = ctypes.c_float


def build():
    """Compile liboracle.so with the Makefile next to this file."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        for sfx, rp, R in (("d", _dp, _D), ("f", _fp, _F)):
            getattr(L, "or_wrap_" + sfx).argtypes = [rp, _L, rp, rp, _ip]
            getattr(L, "or_ghost_boxes_" + sfx).argtypes = [rp, rp, _ip, rp, rp, rp, _ip]
            getattr(L, "or_ghost_boxes_" + sfx).restype = _I
            getattr(L, "or_shift_vectors_" + sfx).argtypes = [rp, rp, rp]
            getattr(L, "or_ghost_count_" + sfx).argtypes = [rp, _L, rp, rp, _ip, _I, _ip]
            getattr(L, "or_ghost_images_" + sfx).argtypes = [rp, _L, rp, rp, _ip, _I, rp, rp, _ip, _ip, _L]
            getattr(L, "or_ghost_images_" + sfx).restype = _L
            getattr(L, "or_ghost_get_" + sfx).argtypes = [rp, _L, rp, rp, _ip, rp, rp, _ip, _ip, _L]
            getattr(L, "or_ghost_get_" + sfx).restype = _L
            getattr(L, "or_cl_geometry_" + sfx).argtypes = [rp, rp, rp, R, R, _I, rp, rp, _ip, _ip,
                                                            ctypes.POINTER(ctypes.c_long)]
            getattr(L, "or_cl_build_" + sfx).argtypes = [rp, _L, rp, rp, _ip, _I, _lp, _ip, ctypes.c_void_p]
            getattr(L, "or_verlet_" + sfx).argtypes = [rp, _L, _L, rp, rp, _ip, _I, R, ctypes.c_void_p,
                                                       ctypes.c_void_p, ctypes.c_void_p]
            getattr(L, "or_verlet_" + sfx).restype = _L
            getattr(L, "or_brute_nn_" + sfx).argtypes = [rp, _L, _L, R, ctypes.c_void_p, ctypes.c_void_p,
                                                         ctypes.c_void_p]
            getattr(L, "or_brute_nn_" + sfx).restype = _L
            getattr(L, "or_test_force_" + sfx).argtypes = [rp, rp, _L, _L, rp, rp, _ip, _I, rp]
        L.or_lj_verlet_d.argtypes = [_dp, _L, _lp, _lp, _ip, _D, _D, _D, _dp, _dp, _dp]
        L.or_lj_cell_d.argtypes = [_dp, _L, _L, _dp, _dp, _ip, _I, _D, _D, _D, _dp, _dp, _dp]
        L.or_sph_rates_d.argtypes = [_dp, _dp, _dp, _ip, _L, _lp, _lp, _ip, _D, _D, _D, _D, _D, _D, _dp, _dp]
        L.or_md_lj_d.argtypes = [_dp, _dp, _L, _dp, _dp, _ip, _dp, _D, _D, _D, _D, _D, _D, _I, _dp,
                                 ctypes.POINTER(ctypes.c_double)]
        L.or_md_lj_d.restype = _I
        L.or_md_sph_d.argtypes = [_dp, _dp, _dp, _ip, _L, _dp, _dp, _D, _D, _D, _D, _D, _D, _D, _I, _dp]
        L.or_md_sph_d.restype = _I
        L.or_num_threads.restype = _I
        L.or_set_threads.argtypes = [_I]
        _LIB = L
    return _LIB


def _t(dtype):
    return ("d", np.float64) if np.dtype(dtype) == np.float64 else ("f", np.float32)


def _a(x, dt):
    return np.ascontiguousarray(x, dtype=dt)


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def num_threads():
    return lib().or_num_threads()


def set_threads(n):
    lib().or_set_threads(int(n))


def wrap(pos, lo, hi, bc):
    """map() on one process: periodic_l per periodic dimension (CartDecomposition.hpp:838-845)."""
    s, dt = _t(pos.dtype)
    p = _a(pos, dt).copy()
    getattr(lib(), "or_wrap_" + s)(p, p.shape[0], _a(lo, dt), _a(hi, dt), _a(bc, np.int32))
    return p


def ghost_boxes(lo, hi, bc, g, dtype=np.float64):
    """Local periodic ghost boxes sorted by shift id (ie_loc_ghost.hpp:145-268, vector_dist_comm.hpp:588-668)."""
    s, dt = _t(dtype)
    blo = np.zeros((26, 3), dt)
    bhi = np.zeros((26, 3), dt)
    sv = np.zeros(26, np.int32)
    g = np.broadcast_to(np.asarray(g, dt), (3,))
    nb = getattr(lib(), "or_ghost_boxes_" + s)(_a(lo, dt), _a(hi, dt), _a(bc, np.int32), _a(g, dt), blo, bhi, sv)
    return blo[:nb].copy(), bhi[:nb].copy(), sv[:nb].copy()


def shift_vectors(lo, hi, dtype=np.float64):
    """27 shift vectors indexed by comb.lin() (shift_vect_converter.hpp:36-66)."""
    s, dt = _t(dtype)
    out = np.zeros((27, 3), dt)
    getattr(lib(), "or_shift_vectors_" + s)(_a(lo, dt), _a(hi, dt), out)
    return out


def ghost_count(pos, blo, bhi, sv):
    """num_shift_ghost_each_part over an explicit box list (vector_dist_cuda_funcs.cuh:157-182)."""
    s, dt = _t(pos.dtype)
    out = np.zeros(pos.shape[0], np.int32)
    getattr(lib(), "or_ghost_count_" + s)(_a(pos, dt), pos.shape[0], _a(blo, dt), _a(bhi, dt),
                                          _a(sv, np.int32), len(sv), out)
    return out


def ghost_images(pos, blo, bhi, sv, shifts):
    """shift_ghost_each_part over an explicit box list (vector_dist_cuda_funcs.cuh:184-233)."""
    s, dt = _t(pos.dtype)
    cap = int(ghost_count(pos, blo, bhi, sv).sum())
    img = np.zeros((max(cap, 1), 3), dt)
    src = np.zeros(max(cap, 1), np.int32)
    shf = np.zeros(max(cap, 1), np.int32)
    m = getattr(lib(), "or_ghost_images_" + s)(_a(pos, dt), pos.shape[0], _a(blo, dt), _a(bhi, dt),
                                               _a(sv, np.int32), len(sv), _a(shifts, dt), img, src, shf, cap)
    return img[:m], src[:m], shf[:m]


def ghost_get(pos, lo, hi, bc, g):
    """ghost_get on one process: periodic images of every particle, particle-major, shifts ascending."""
    s, dt = _t(pos.dtype)
    blo, bhi, sv = ghost_boxes(lo, hi, bc, g, dtype=dt)
    return ghost_images(_a(pos, dt), blo, bhi, sv, shift_vectors(lo, hi, dtype=dt))


class CLGeom:
    def __init__(self, box_lo, spacing, div, gs, ncells, pad, dtype):
        self.box_lo, self.spacing, self.div, self.gs = box_lo, spacing, div, gs
        self.ncells, self.pad, self.dtype = ncells, pad, dtype


def cl_geometry(lo, hi, g, r_cut, enlarge=None, pad=1, dtype=np.float64, verlet=False):
    """Cell-list geometry of getCellListGPU / getVerlet (vector_dist.hpp:1222-1260, 1533-1538).

    The reference magnifies the ghost by the float 1.013f in getCellListGPU and by
    the double 1.013 in getVerlet; ``verlet`` selects which.
    """
    s, dt = _t(dtype)
    if enlarge is None:
        enlarge = 1.013 if verlet else float(np.float32(1.013))
    g = np.broadcast_to(np.asarray(g, dt), (3,))
    box_lo = np.zeros(3, dt)
    sp = np.zeros(3, dt)
    div = np.zeros(3, np.int32)
    gs = np.zeros(3, np.int32)
    nc = ctypes.c_long(0)
    getattr(lib(), "or_cl_geometry_" + s)(_a(lo, dt), _a(hi, dt), _a(g, dt), r_cut, enlarge, pad, box_lo, sp, div,
                                          gs, ctypes.byref(nc))
    return CLGeom(box_lo, sp, div, gs, nc.value, pad, dt)


def cl_build(pos, G):
    """Stable counting-sort cell list: (cell_start[ncells+1], sorted ids, cell of each particle)."""
    s, dt = _t(G.dtype)
    n = pos.shape[0]
    cs = np.zeros(G.ncells + 1, np.int64)
    so = np.zeros(max(n, 1), np.int32)
    cp = np.zeros(max(n, 1), np.int64)
    getattr(lib(), "or_cl_build_" + s)(_a(pos, dt), n, G.box_lo, G.spacing, G.div, G.pad, cs, so, _ptr(cp))
    return cs, so[:n], cp[:n]


def verlet(pos, n_dom, G, r):
    """Full Verlet list of [0,n_dom) over all particles, self included (vector_dist.hpp:1514-1547).

    Returns CSR (offsets[n_dom+1], idx).
    """
    s, dt = _t(G.dtype)
    p = _a(pos, dt)
    n_all = p.shape[0]
    f = getattr(lib(), "or_verlet_" + s)
    counts = np.zeros(max(n_dom, 1), np.int64)
    f(p, n_dom, n_all, G.box_lo, G.spacing, G.div, G.pad, r, _ptr(counts), None, None)
    off = np.zeros(n_dom + 1, np.int64)
    off[1:] = np.cumsum(counts[:n_dom])
    idx = np.zeros(max(int(off[-1]), 1), np.int32)
    f(p, n_dom, n_all, G.box_lo, G.spacing, G.div, G.pad, r, None, _ptr(off), _ptr(idx))
    return off, idx[: off[-1]]


def brute_nn(pos, n_dom, r):
    """O(N^2) neighbour lists with d2 < r^2 (vector_dist_NN_tests.cpp:268-280)."""
    s, dt = _t(pos.dtype)
    p = _a(pos, dt)
    f = getattr(lib(), "or_brute_nn_" + s)
    counts = np.zeros(max(n_dom, 1), np.int64)
    f(p, n_dom, p.shape[0], r, _ptr(counts), None, None)
    off = np.zeros(n_dom + 1, np.int64)
    off[1:] = np.cumsum(counts[:n_dom])
    idx = np.zeros(max(int(off[-1]), 1), np.int32)
    f(p, n_dom, p.shape[0], r, None, _ptr(off), _ptr(idx))
    return off, idx[: off[-1]]


def lj_verlet(pos, n_dom, off, idx, eps=1.0, sigma=1.0, rc=2.5):
    """LJ forces / per-particle PE / virial from a CSR Verlet list (FP64)."""
    p = _a(pos, np.float64)
    counts = np.ascontiguousarray(np.diff(off), dtype=np.int64)
    f = np.zeros((n_dom, 3))
    pe = np.zeros(n_dom)
    vir = np.zeros(n_dom)
    lib().or_lj_verlet_d(p, n_dom, _a(off[:-1], np.int64), counts, _a(idx, np.int32), eps, sigma, rc, f, pe, vir)
    return f, pe, vir


def lj_cell(pos, n_dom, G, eps=1.0, sigma=1.0, rc=2.5):
    """LJ forces through the cell-list NN-box walk (FP64)."""
    p = _a(pos, np.float64)
    f = np.zeros((n_dom, 3))
    pe = np.zeros(n_dom)
    vir = np.zeros(n_dom)
    lib().or_lj_cell_d(p, n_dom, p.shape[0], _a(G.box_lo, np.float64), _a(G.spacing, np.float64), G.div, G.pad,
                       eps, sigma, rc, f, pe, vir)
    return f, pe, vir


def test_force(pos, prop0, n_dom, G):
    """The reference's test functor calculate_force (vector_dist_gpu_unit_tests.cu:46-81)."""
    s, dt = _t(G.dtype)
    out = np.zeros((n_dom, 3), dt)
    getattr(lib(), "or_test_force_" + s)(_a(pos, dt), _a(prop0, dt), n_dom, pos.shape[0], G.box_lo, G.spacing,
                                         G.div, G.pad, out)
    return out


def sph_rates(pos, vel, rho, typ, off, idx, h, m, c0, rho0, alpha, gz):
    """WCSPH accelerations and density rates from a CSR neighbour list (FP64)."""
    n = pos.shape[0] if rho.shape[0] == pos.shape[0] else rho.shape[0]
    acc = np.zeros((n, 3))
    drho = np.zeros(n)
    counts = np.ascontiguousarray(np.diff(off), dtype=np.int64)
    lib().or_sph_rates_d(_a(pos, np.float64), _a(vel, np.float64), _a(rho, np.float64), _a(typ, np.int32), n,
                         _a(off[:-1], np.int64), counts, _a(idx, np.int32), h, m, c0, rho0, alpha, gz, acc, drho)
    return acc, drho


def md_sph(x, v, rho, typ, lo, hi, h, m, c0, rho0, alpha, gz, dt, steps):
    """WCSPH kick-drift-kick with fixed walls; returns (x, v, rho, E[steps, 4] = KE, sum rho, 0, 0)."""
    x = _a(x, np.float64).copy()
    v = _a(v, np.float64).copy()
    rho = _a(rho, np.float64).copy()
    E = np.zeros((max(steps, 1), 4))
    rc_ = lib().or_md_sph_d(x, v, rho, _a(typ, np.int32), x.shape[0], _a(lo, np.float64), _a(hi, np.float64), h, m,
                            c0, rho0, alpha, gz, dt, steps, E)
    assert rc_ == 0
    return x, v, rho, E[:steps]


def md_lj(x, v, lo, hi, bc, ghost, rc, skin, eps, sigma, dt, mass, steps, timing=False):
    """Velocity-Verlet LJ MD with a skin Verlet list; returns (x, v, E[steps+1, 4])
    (and the wall time of the step loop, excluding the initial build, if timing)."""
    x = _a(x, np.float64).copy()
    v = _a(v, np.float64).copy()
    E = np.zeros((steps + 1, 4))
    g = np.broadcast_to(np.asarray(ghost, np.float64), (3,))
    t = ctypes.c_double(0.0)
    rc_ = lib().or_md_lj_d(x, v, x.shape[0], _a(lo, np.float64), _a(hi, np.float64), _a(bc, np.int32),
                           _a(g, np.float64), rc, skin, eps, sigma, dt, mass, steps, E, ctypes.byref(t))
    assert rc_ == 0
    return (x, v, E, t.value) if timing else (x, v, E)


# ---------------------------------------------------------------------------
# index / merge restatements in numpy (small, sequential: the order is the spec)

def ghost_put(a, n, src, op):
    """ghost_put<op_> on one process (vector_dist_comm.hpp:2086-2182, merge_prp_v):
    the value of every ghost j (slot n + j) is merged onto its source src[j]; the
    ghosts of one source in ghost order.  op: 1 add_, 2 max_, 3 replace_."""
    out = np.array(a[:n], copy=True)
    for j in np.argsort(np.asarray(src), kind="stable"):
        p = src[j]
        v = a[n + j]
        if op == 1:
            out[p] = out[p] + v
        elif op == 2:
            out[p] = np.maximum(out[p], v)
        else:
            out[p] = v
    return out


def _lex_after(a, b):
    return a[0] > b[0] or (a[0] == b[0] and (a[1] > b[1] or (a[1] == b[1] and a[2] > b[2])))


def verlet_sym(pos, n_dom, off, idx):
    """Symmetric (half) list from the full list (getVerletSym, vector_dist.hpp:1412-1416):
    row p keeps a domain partner q iff q > p and a ghost iff it lies after p in
    (x, y, z) lexicographic order, so each pair -- and each periodic mirror pair --
    appears once.  Rows keep the full list's order.  Returns CSR (offsets, idx)."""
    hoff = np.zeros(n_dom + 1, np.int64)
    rows = []
    for i in range(n_dom):
        row = idx[off[i]:off[i + 1]]
        keep = [q for q in row if (q > i if q < n_dom else _lex_after(pos[q], pos[i]))]
        rows.append(np.asarray(keep, np.int32))
        hoff[i + 1] = hoff[i] + len(keep)
    return hoff, (np.concatenate(rows) if hoff[-1] else np.zeros(0, np.int32))


def remove_marked(mark, *cols):
    """remove_marked<prp> (vector_dist_cuda_funcs.cuh:333-412): the mark is flipped
    (flip_one_to_zero :313-321, x -> x == 0), the particles with a flipped mark of
    1 are kept in order (copy_new_to_old_by_scan :295-311).  Returns (flipped mark
    of all particles, kept flipped mark, kept columns...); when nothing is marked
    the columns come back whole."""
    mark = np.asarray(mark)
    flipped = (mark == 0).astype(mark.dtype)
    keep = flipped != 0
    if keep.all():
        return (flipped, flipped) + tuple(np.asarray(c) for c in cols)
    return (flipped, flipped[keep]) + tuple(np.asarray(c)[keep] for c in cols)


def indexes_by_type(vals, end, cmp, value):
    """get_indexes_by_type<prp, functor> (vector_dist_cuda_funcs.cuh:414-481): the
    ascending indexes p < end with functor::check(vals[p]); here the check is a
    comparison (0 ==, 1 !=, 2 <, 3 <=, 4 >, 5 >=) with `value`."""
    v = np.asarray(vals)[:end]
    ref = np.asarray(value).astype(v.dtype)
    f = [v == ref, v != ref, v < ref, v <= ref, v > ref, v >= ref][cmp]
    return np.nonzero(f)[0].astype(np.uint32)
