// pd_oracle.cpp -- CPU oracle for the single-process OpenFPM pdata particle path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker: tests/, the smoke entry
// point and bench.py's cpu_baseline / reference leg load it.  The product
// library (openfpm_pdata_b200/csrc) never links, loads or calls it.
//
// It restates, in plain C++ (templates over float / double), the algorithm of
// the reference's CPU vector_dist path for one process and one sub-domain:
//   * periodic wrap  ............  CartDecomposition.hpp:838-845 (periodic_l
//                                   from openfpm_data, restated below)
//   * shift vectors  ............  shift_vect_converter.hpp:36-66
//   * local periodic ghost boxes .  ie_loc_ghost.hpp:145-268, sorted by shift id
//                                   as in vector_dist_comm.hpp:588-668
//   * image generation (GPU order)  vector_dist_cuda_funcs.cuh:157-233
//   * image replay ...............  vector_dist_cuda_funcs.cuh:133-155
//   * cell-list geometry .........  vector_dist.hpp:1222-1260 (cl_param_calculate
//                                   of openfpm_data, restated)
//   * cell-list fill / NN box walk  vector_dist.hpp:1093-1159, test walk in
//                                   vector_dist_gpu_unit_tests.cu:121-179
//   * full Verlet list incl. self   vector_dist.hpp:1514-1547 with the pair
//                                   predicate d2 < r_cut^2 of
//                                   vector_dist_NN_tests.cpp:268-296
//   * test pair functor ..........  vector_dist_gpu_unit_tests.cu:46-81
// Physics with no reference source is restated from published methods:
//   * Lennard-Jones 12-6 with plain cutoff, velocity Verlet (Swope et al. 1982)
//   * WCSPH: cubic spline (Monaghan & Lattanzio 1985), Tait EOS (Monaghan 1994),
//     artificial viscosity (Monaghan 1992)
//
// Parity contract shared with the CUDA path (both sides follow it exactly):
//   cell index     ik = clamp(floor((x_k - box_lo_k) / spacing_k) + pad, 0, gs_k-1)
//   linear cell    c = i0 + gs0*(i1 + gs1*i2)                (dimension 0 fastest)
//   in-cell order  ascending particle index (stable counting sort)
//   distance^2     d2 = fma(dz,dz, fma(dy,dy, dx*dx)),  dx = xp - xq
//   pair predicate d2 < r*r                                 (self included)
//   NN box order   dz, dy, dx in [-r, r], dx fastest
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

static const int PERIODIC = 1;

// openfpm::math::periodic_l (openfpm_data, not vendored): bring a coordinate that
// left [p1,p2) by less than one period back inside; the "== p2" round-off fix
// keeps the result half-open.
template <class T> inline T periodic_l(T pos, T p2, T p1) {
    T r = pos;
    if (pos >= p2) {
        r = p1 + (pos - p2);
    } else if (pos < p1) {
        r = p2 - (p1 - pos);
        if (r == p2) r = p1;
    }
    return r;
}

struct Comb {
    int c[3];
    int lin() const { return (c[0] + 1) + 3 * (c[1] + 1) + 9 * (c[2] + 1); }
};
inline Comb comb_from_lin(int l) {
    Comb k;
    k.c[0] = l % 3 - 1;
    k.c[1] = (l / 3) % 3 - 1;
    k.c[2] = l / 9 - 1;
    return k;
}

template <class T> struct GBox {
    T lo[3], hi[3];
    int sv;
};

// Shift vector of combination c: -(hi-lo) where c=+1, +(hi-lo) where c=-1
// (shift_vect_converter.hpp:46-60).
template <class T> inline void shift_vector(const Comb& k, const T lo[3], const T hi[3], T s[3]) {
    for (int d = 0; d < 3; ++d) {
        if (k.c[d] == 1) s[d] = -(hi[d] - lo[d]);
        else if (k.c[d] == -1) s[d] = (hi[d] - lo[d]);
        else s[d] = 0;
    }
}

// Local internal ghost boxes of a single sub-domain equal to the whole domain:
// applyBC replicates the domain shifted by -L*c (ie_loc_ghost.hpp:163-185), each
// replica is enlarged by the ghost and intersected with the domain
// (create_loc_ghost_ibox, :102-143); createShiftBox sorts the boxes by shift id
// (vector_dist_comm.hpp:645-655).  Returns the box count (<= 26).
template <class T>
int ghost_boxes(const T lo[3], const T hi[3], const int bc[3], const T g[3], GBox<T>* out) {
    int nb = 0;
    for (int l = 0; l < 27; ++l) {
        Comb k = comb_from_lin(l);
        if (k.c[0] == 0 && k.c[1] == 0 && k.c[2] == 0) continue;
        bool valid = true;
        for (int d = 0; d < 3; ++d)
            if (k.c[d] != 0 && bc[d] != PERIODIC) valid = false;
        if (!valid) continue;
        GBox<T> b;
        bool empty = false;
        for (int d = 0; d < 3; ++d) {
            T sh;
            if (k.c[d] == 1) sh = -hi[d] + lo[d];
            else if (k.c[d] == -1) sh = hi[d] - lo[d];
            else sh = 0;
            T sl = lo[d] + sh, su = hi[d] + sh;
            T el = sl + (-g[d]), eu = su + g[d];
            T bl = std::max(lo[d], el), bu = std::min(hi[d], eu);
            if (bl >= bu) empty = true;
            b.lo[d] = bl;
            b.hi[d] = bu;
        }
        if (empty) continue;
        b.sv = l;
        out[nb++] = b;
    }
    return nb;
}

// Box::isInsideNP: lo <= x < hi in every dimension.
template <class T> inline bool inside_np(const GBox<T>& b, const T* x) {
    for (int d = 0; d < 3; ++d)
        if (x[d] < b.lo[d] || x[d] >= b.hi[d]) return false;
    return true;
}

// num_shift_ghost_each_part (vector_dist_cuda_funcs.cuh:157-182): number of
// images of a particle; a box whose shift id equals the last accepted one is
// skipped (boxes are sorted by shift id).
template <class T> inline int count_images(const GBox<T>* bx, const int* sv, int nb, const T* x) {
    int n = 0;
    int old = -1;
    for (int i = 0; i < nb; ++i) {
        int s = sv[i];
        if (inside_np(bx[i], x) && s != old) {
            old = s;
            n++;
        }
    }
    return n;
}

// ----------------------------------------------------------------------------
// cell list
template <class T> struct CLGeom {
    T box_lo[3];
    T spacing[3];
    int div[3];
    int pad;
    int gs[3];
    long ncells;
};

// cl_param_calculate (openfpm_data; call site vector_dist.hpp:1246): the
// processor box enlarged by the ghost magnified by `enlarge`; div = floor(len /
// r_cut) + 1 cells of side r_cut; `pad` layers of padding cells on every side.
template <class T>
CLGeom<T> cl_geometry(const T lo[3], const T hi[3], const T g[3], T r_cut, T enlarge, int pad) {
    CLGeom<T> G;
    G.pad = pad;
    G.ncells = 1;
    for (int d = 0; d < 3; ++d) {
        T gl = (-g[d]) * enlarge, gh = g[d] * enlarge;
        T pl = lo[d] + gl, ph = hi[d] + gh;
        long dv = (long)((ph - pl) / r_cut) + 1;
        ph = pl + (T)dv * r_cut;
        G.box_lo[d] = pl;
        G.spacing[d] = (ph - pl) / (T)dv;
        G.div[d] = (int)dv;
        G.gs[d] = (int)dv + 2 * pad;
        G.ncells *= G.gs[d];
    }
    return G;
}

template <class T> inline int cell_coord(const CLGeom<T>& G, int d, T x) {
    long i = (long)std::floor((x - G.box_lo[d]) / G.spacing[d]) + G.pad;
    if (i < 0) i = 0;
    if (i > G.gs[d] - 1) i = G.gs[d] - 1;
    return (int)i;
}
template <class T> inline long cell_of(const CLGeom<T>& G, const T* x) {
    int i0 = cell_coord(G, 0, x[0]), i1 = cell_coord(G, 1, x[1]), i2 = cell_coord(G, 2, x[2]);
    return i0 + (long)G.gs[0] * (i1 + (long)G.gs[1] * i2);
}

// stable counting sort of particles [0,n) by cell
template <class T>
void cl_build(const CLGeom<T>& G, const T* pos, long n, long* cell_start, int* sorted, long* cell_of_p) {
    std::vector<long> cnt(G.ncells + 1, 0);
    for (long i = 0; i < n; ++i) {
        long c = cell_of(G, pos + 3 * i);
        if (cell_of_p) cell_of_p[i] = c;
        cnt[c]++;
    }
    cell_start[0] = 0;
    for (long c = 0; c < G.ncells; ++c) cell_start[c + 1] = cell_start[c] + cnt[c];
    std::vector<long> fill(cell_start, cell_start + G.ncells);
    for (long i = 0; i < n; ++i) {
        long c = cell_of_p ? cell_of_p[i] : cell_of(G, pos + 3 * i);
        sorted[fill[c]++] = (int)i;
    }
}

template <class T> inline T dist2(const T* p, const T* q) {
    T dx = p[0] - q[0], dy = p[1] - q[1], dz = p[2] - q[2];
    return std::fma(dz, dz, std::fma(dy, dy, dx * dx));
}

// Walk the (2r+1)^3 box of cells around particle p's cell and call f(q).
template <class T, class F>
inline void nn_box_walk(const CLGeom<T>& G, const long* cell_start, const int* sorted, const T* xp, int r, F f) {
    int c0 = cell_coord(G, 0, xp[0]), c1 = cell_coord(G, 1, xp[1]), c2 = cell_coord(G, 2, xp[2]);
    for (int dz = -r; dz <= r; ++dz) {
        int z = c2 + dz;
        if (z < 0 || z >= G.gs[2]) continue;
        for (int dy = -r; dy <= r; ++dy) {
            int y = c1 + dy;
            if (y < 0 || y >= G.gs[1]) continue;
            for (int dx = -r; dx <= r; ++dx) {
                int x = c0 + dx;
                if (x < 0 || x >= G.gs[0]) continue;
                long c = x + (long)G.gs[0] * (y + (long)G.gs[1] * z);
                for (long k = cell_start[c]; k < cell_start[c + 1]; ++k) f(sorted[k]);
            }
        }
    }
}

// ----------------------------------------------------------------------------
// Lennard-Jones 12-6, plain cutoff (force on p from q, r = xp - xq)
template <class T> struct LJ {
    T eps, sig2, rc2;
};
template <class T> inline void lj_pair(const LJ<T>& P, T r2, T dx, T dy, T dz, T& fx, T& fy, T& fz, T& pe, T& vir) {
    T ir2 = T(1) / r2;
    T s2 = P.sig2 * ir2;
    T s6 = s2 * s2 * s2;
    T ff = T(24) * P.eps * ir2 * s6 * (T(2) * s6 - T(1));
    fx += ff * dx;
    fy += ff * dy;
    fz += ff * dz;
    pe += T(4) * P.eps * s6 * (s6 - T(1));
    vir += ff * r2;
}

}  // namespace orc

using namespace orc;

// ============================================================================
// C ABI for ctypes.  Positions are AoS xyz (3 values per particle).
template <class T> static void wrap_impl(T* pos, long n, const T* lo, const T* hi, const int* bc) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d)
            if (bc[d] == PERIODIC) pos[3 * i + d] = periodic_l(pos[3 * i + d], hi[d], lo[d]);
}

template <class T>
static int ghost_boxes_impl(const T* lo, const T* hi, const int* bc, const T* g, T* blo, T* bhi, int* sv) {
    GBox<T> b[26];
    int nb = ghost_boxes(lo, hi, bc, g, b);
    for (int i = 0; i < nb; ++i) {
        for (int d = 0; d < 3; ++d) {
            blo[3 * i + d] = b[i].lo[d];
            bhi[3 * i + d] = b[i].hi[d];
        }
        sv[i] = b[i].sv;
    }
    return nb;
}

template <class T>
static void to_boxes(const T* blo, const T* bhi, const int* sv, int nb, std::vector<GBox<T>>& B) {
    B.resize(nb);
    for (int i = 0; i < nb; ++i) {
        for (int d = 0; d < 3; ++d) {
            B[i].lo[d] = blo[3 * i + d];
            B[i].hi[d] = bhi[3 * i + d];
        }
        B[i].sv = sv[i];
    }
}

// num_shift_ghost_each_part over an explicit box list
template <class T>
static void ghost_count_impl(const T* pos, long n, const T* blo, const T* bhi, const int* sv, int nb, int* out) {
    std::vector<GBox<T>> B;
    to_boxes(blo, bhi, sv, nb, B);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) out[i] = count_images(B.data(), sv, nb, pos + 3 * i);
}

// shift_ghost_each_part over an explicit box list, shifts indexed by sv.
// Writes images (AoS) and (src, shift) records in particle-major order; returns count.
template <class T>
static long ghost_images_impl(const T* pos, long n, const T* blo, const T* bhi, const int* sv, int nb,
                              const T* shifts, T* img, int* src, int* shf, long cap) {
    std::vector<GBox<T>> B;
    to_boxes(blo, bhi, sv, nb, B);
    long m = 0;
    for (long p = 0; p < n; ++p) {
        const T* x = pos + 3 * p;
        int old = -1;
        for (int i = 0; i < nb; ++i) {
            int s = sv[i];
            if (inside_np(B[i], x) && s != old) {
                if (m < cap) {
                    for (int d = 0; d < 3; ++d) img[3 * m + d] = x[d] - shifts[3 * s + d];
                    src[m] = (int)p;
                    shf[m] = s;
                }
                old = s;
                m++;
            }
        }
    }
    return m;
}

// ghost_get for one sub-domain equal to the domain (periodic images only)
template <class T>
static long ghost_get_impl(const T* pos, long n, const T* lo, const T* hi, const int* bc, const T* g, T* img,
                           int* src, int* shf, long cap) {
    T blo[78], bhi[78];
    int sv[26];
    int nb = ghost_boxes_impl(lo, hi, bc, g, blo, bhi, sv);
    T shifts[81];
    for (int l = 0; l < 27; ++l) shift_vector(comb_from_lin(l), lo, hi, shifts + 3 * l);
    return ghost_images_impl(pos, n, blo, bhi, sv, nb, shifts, img, src, shf, cap);
}

template <class T>
static void cl_geometry_impl(const T* lo, const T* hi, const T* g, T r_cut, T enlarge, int pad, T* box_lo,
                             T* spacing, int* div, int* gs, long* ncells) {
    CLGeom<T> G = cl_geometry(lo, hi, g, r_cut, enlarge, pad);
    for (int d = 0; d < 3; ++d) {
        box_lo[d] = G.box_lo[d];
        spacing[d] = G.spacing[d];
        div[d] = G.div[d];
        gs[d] = G.gs[d];
    }
    *ncells = G.ncells;
}

template <class T> static CLGeom<T> geom_from(const T* box_lo, const T* spacing, const int* div, int pad) {
    CLGeom<T> G;
    G.pad = pad;
    G.ncells = 1;
    for (int d = 0; d < 3; ++d) {
        G.box_lo[d] = box_lo[d];
        G.spacing[d] = spacing[d];
        G.div[d] = div[d];
        G.gs[d] = div[d] + 2 * pad;
        G.ncells *= G.gs[d];
    }
    return G;
}

template <class T>
static void cl_build_impl(const T* pos, long n, const T* box_lo, const T* spacing, const int* div, int pad,
                          long* cell_start, int* sorted, long* cell_of_p) {
    CLGeom<T> G = geom_from(box_lo, spacing, div, pad);
    cl_build(G, pos, n, cell_start, sorted, cell_of_p);
}

// Full Verlet list for particles [0, n_dom) against all particles [0, n_all),
// self included, built by the cell-list walk.  Pass 1 (idx == NULL) fills
// counts; pass 2 fills idx (CSR, offsets = exclusive scan of counts).
template <class T>
static long verlet_impl(const T* pos, long n_dom, long n_all, const T* box_lo, const T* spacing, const int* div,
                        int pad, T r, long* counts, const long* offsets, int* idx) {
    CLGeom<T> G = geom_from(box_lo, spacing, div, pad);
    std::vector<long> cs(G.ncells + 1);
    std::vector<int> so(n_all);
    cl_build(G, pos, n_all, cs.data(), so.data(), (long*)nullptr);
    T r2 = r * r;
    long tot = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : tot)
    for (long p = 0; p < n_dom; ++p) {
        const T* xp = pos + 3 * p;
        long c = 0;
        long base = idx ? offsets[p] : 0;
        nn_box_walk(G, cs.data(), so.data(), xp, 1, [&](int q) {
            if (dist2(xp, pos + 3 * (long)q) < r2) {
                if (idx) idx[base + c] = q;
                c++;
            }
        });
        if (counts) counts[p] = c;
        tot += c;
    }
    return tot;
}

// O(N^2) neighbour counts/lists (vector_dist_NN_tests.cpp:268-280 brute force)
template <class T>
static long brute_nn_impl(const T* pos, long n_dom, long n_all, T r, long* counts, const long* offsets, int* idx) {
    T r2 = r * r;
    long tot = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : tot)
    for (long p = 0; p < n_dom; ++p) {
        long c = 0;
        for (long q = 0; q < n_all; ++q) {
            if (dist2(pos + 3 * p, pos + 3 * q) < r2) {
                if (idx) idx[offsets[p] + c] = (int)q;
                c++;
            }
        }
        if (counts) counts[p] = c;
        tot += c;
    }
    return tot;
}

// LJ forces on [0,n_dom) from a CSR neighbour list; out: f (AoS), per-particle
// potential energy (half of the pair sum) and virial (half).
template <class T>
static void lj_verlet_impl(const T* pos, long n_dom, const long* offsets, const long* counts, const int* idx, T eps,
                           T sigma, T rc, T* f, T* pe, T* vir) {
    LJ<T> P{eps, sigma * sigma, rc * rc};
#pragma omp parallel for schedule(static)
    for (long p = 0; p < n_dom; ++p) {
        const T* xp = pos + 3 * p;
        T fx = 0, fy = 0, fz = 0, e = 0, w = 0;
        for (long k = offsets[p]; k < offsets[p] + counts[p]; ++k) {
            long q = idx[k];
            if (q == p) continue;
            const T* xq = pos + 3 * q;
            T dx = xp[0] - xq[0], dy = xp[1] - xq[1], dz = xp[2] - xq[2];
            T r2 = std::fma(dz, dz, std::fma(dy, dy, dx * dx));
            if (r2 < P.rc2) lj_pair(P, r2, dx, dy, dz, fx, fy, fz, e, w);
        }
        f[3 * p] = fx;
        f[3 * p + 1] = fy;
        f[3 * p + 2] = fz;
        if (pe) pe[p] = T(0.5) * e;
        if (vir) vir[p] = T(0.5) * w;
    }
}

// LJ forces on [0,n_dom) through the cell-list walk (cell list over [0,n_all))
template <class T>
static void lj_cell_impl(const T* pos, long n_dom, long n_all, const T* box_lo, const T* spacing, const int* div,
                         int pad, T eps, T sigma, T rc, T* f, T* pe, T* vir) {
    CLGeom<T> G = geom_from(box_lo, spacing, div, pad);
    std::vector<long> cs(G.ncells + 1);
    std::vector<int> so(n_all);
    cl_build(G, pos, n_all, cs.data(), so.data(), (long*)nullptr);
    LJ<T> P{eps, sigma * sigma, rc * rc};
#pragma omp parallel for schedule(dynamic, 256)
    for (long p = 0; p < n_dom; ++p) {
        const T* xp = pos + 3 * p;
        T fx = 0, fy = 0, fz = 0, e = 0, w = 0;
        nn_box_walk(G, cs.data(), so.data(), xp, 1, [&](int q) {
            if (q == p) return;
            const T* xq = pos + 3 * (long)q;
            T dx = xp[0] - xq[0], dy = xp[1] - xq[1], dz = xp[2] - xq[2];
            T r2 = std::fma(dz, dz, std::fma(dy, dy, dx * dx));
            if (r2 < P.rc2) lj_pair(P, r2, dx, dy, dz, fx, fy, fz, e, w);
        });
        f[3 * p] = fx;
        f[3 * p + 1] = fy;
        f[3 * p + 2] = fz;
        if (pe) pe[p] = T(0.5) * e;
        if (vir) vir[p] = T(0.5) * w;
    }
}

// The reference's test functor calculate_force (vector_dist_gpu_unit_tests.cu:46-81):
// sum over the NN box of prop0(q) * (xq - xp)/|xq - xp|, q != p, |r| > 1e-6.
template <class T>
static void test_force_impl(const T* pos, const T* prop0, long n_dom, long n_all, const T* box_lo, const T* spacing,
                            const int* div, int pad, T* out) {
    CLGeom<T> G = geom_from(box_lo, spacing, div, pad);
    std::vector<long> cs(G.ncells + 1);
    std::vector<int> so(n_all);
    cl_build(G, pos, n_all, cs.data(), so.data(), (long*)nullptr);
#pragma omp parallel for schedule(dynamic, 256)
    for (long p = 0; p < n_dom; ++p) {
        const T* xp = pos + 3 * p;
        T f[3] = {0, 0, 0};
        nn_box_walk(G, cs.data(), so.data(), xp, 1, [&](int q) {
            if (q == p) return;
            const T* xq = pos + 3 * (long)q;
            T r[3] = {xq[0] - xp[0], xq[1] - xp[1], xq[2] - xp[2]};
            T nrm = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
            if (nrm > T(1e-6)) {
                for (int d = 0; d < 3; ++d) f[d] += prop0[q] * (r[d] / nrm);
            }
        });
        for (int d = 0; d < 3; ++d) out[3 * p + d] = f[d];
    }
}

// ----------------------------------------------------------------------------
// Velocity-Verlet LJ MD with a skin Verlet list, in original particle order.
//   per step:  v += dt/2 f ; x += dt v ;
//              if max_i |x_i - x_build_i| > skin/2 (or skin <= 0): wrap, images,
//                  lists rebuilt, x_build = x ; else images refreshed ;
//              f = F(x) ; v += dt/2 f ; record KE, PE, virial
// E[s*4 + {0,1,2,3}] = KE, PE, virial, rebuilt(0/1) after step s (s = 0 is the initial state).
template <class T> struct MDState {
    long n;
    const T* lo;
    const T* hi;
    const int* bc;
    T g[3];
    T rlist, rc, eps, sigma;
    std::vector<T> pos;  // n real + images
    std::vector<int> src, shf;
    long nimg;
    std::vector<long> off, cnt;
    std::vector<int> idx;
    std::vector<T> xb;
    T shifts[81];
};

template <class T> static void md_rebuild(MDState<T>& S) {
    long n = S.n;
    wrap_impl(S.pos.data(), n, S.lo, S.hi, S.bc);
    // images
    long cap = n * 8 + 1024;
    std::vector<T> img(3 * cap);
    S.src.assign(cap, 0);
    S.shf.assign(cap, 0);
    long m = ghost_get_impl(S.pos.data(), n, S.lo, S.hi, S.bc, S.g, img.data(), S.src.data(), S.shf.data(), cap);
    S.nimg = m;
    S.pos.resize(3 * (n + m));
    std::copy(img.begin(), img.begin() + 3 * m, S.pos.begin() + 3 * n);
    // Verlet list over the cell list geometry of getVerlet (ghost magnified 1.013)
    T blo[3], sp[3];
    int dv[3], gs[3];
    long nc;
    cl_geometry_impl(S.lo, S.hi, S.g, S.rlist, (T)1.013, 1, blo, sp, dv, gs, &nc);
    S.cnt.assign(n, 0);
    verlet_impl(S.pos.data(), n, n + m, blo, sp, dv, 1, S.rlist, S.cnt.data(), (const long*)nullptr, (int*)nullptr);
    S.off.assign(n + 1, 0);
    for (long i = 0; i < n; ++i) S.off[i + 1] = S.off[i] + S.cnt[i];
    S.idx.assign(S.off[n], 0);
    verlet_impl(S.pos.data(), n, n + m, blo, sp, dv, 1, S.rlist, (long*)nullptr, S.off.data(), S.idx.data());
    S.xb.assign(S.pos.begin(), S.pos.begin() + 3 * n);
}

template <class T> static void md_refresh_images(MDState<T>& S) {
    long n = S.n;
#pragma omp parallel for schedule(static)
    for (long k = 0; k < S.nimg; ++k)
        for (int d = 0; d < 3; ++d)
            S.pos[3 * (n + k) + d] = S.pos[3 * (long)S.src[k] + d] - S.shifts[3 * S.shf[k] + d];
}

static double wtime() {
#ifdef _OPENMP
    return omp_get_wtime();
#else
    return 0.0;
#endif
}

template <class T>
static int md_lj_impl(T* x, T* v, long n, const T* lo, const T* hi, const int* bc, const T* ghost, T rc, T skin,
                      T eps, T sigma, T dt, T mass, int steps, double* E, double* t_loop) {
    MDState<T> S;
    S.n = n;
    S.lo = lo;
    S.hi = hi;
    S.bc = bc;
    for (int d = 0; d < 3; ++d) S.g[d] = ghost[d];
    S.rlist = rc + skin;
    S.rc = rc;
    S.eps = eps;
    S.sigma = sigma;
    for (int l = 0; l < 27; ++l) shift_vector(comb_from_lin(l), lo, hi, S.shifts + 3 * l);
    S.pos.assign(x, x + 3 * n);
    std::vector<T> f(3 * n), pe(n), vir(n);
    auto forces = [&]() {
        lj_verlet_impl(S.pos.data(), n, S.off.data(), S.cnt.data(), S.idx.data(), eps, sigma, rc, f.data(), pe.data(),
                       vir.data());
    };
    auto record = [&](int s, int rebuilt) {
        double ke = 0, p = 0, w = 0;
        for (long i = 0; i < n; ++i) {
            ke += 0.5 * (double)mass * ((double)v[3 * i] * v[3 * i] + (double)v[3 * i + 1] * v[3 * i + 1] +
                                        (double)v[3 * i + 2] * v[3 * i + 2]);
            p += pe[i];
            w += vir[i];
        }
        E[4 * s] = ke;
        E[4 * s + 1] = p;
        E[4 * s + 2] = w;
        E[4 * s + 3] = rebuilt;
    };
    md_rebuild(S);
    forces();
    record(0, 1);
    T half = T(0.5) * dt / mass;
    T lim2 = (T(0.5) * skin) * (T(0.5) * skin);
    double t0 = wtime();
    for (int s = 1; s <= steps; ++s) {
        T mx = 0;
#pragma omp parallel for schedule(static) reduction(max : mx)
        for (long i = 0; i < n; ++i) {
            for (int d = 0; d < 3; ++d) {
                v[3 * i + d] += half * f[3 * i + d];
                S.pos[3 * i + d] += dt * v[3 * i + d];
            }
            T dx = S.pos[3 * i] - S.xb[3 * i], dy = S.pos[3 * i + 1] - S.xb[3 * i + 1],
              dz = S.pos[3 * i + 2] - S.xb[3 * i + 2];
            T d2 = std::fma(dz, dz, std::fma(dy, dy, dx * dx));
            mx = std::max(mx, d2);
        }
        int rebuilt = 0;
        if (skin <= 0 || mx > lim2) {
            S.pos.resize(3 * n);
            md_rebuild(S);
            rebuilt = 1;
        } else {
            md_refresh_images(S);
        }
        forces();
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; ++i)
            for (int d = 0; d < 3; ++d) v[3 * i + d] += half * f[3 * i + d];
        record(s, rebuilt);
    }
    if (t_loop) *t_loop = wtime() - t0;
    std::copy(S.pos.begin(), S.pos.begin() + 3 * n, x);
    return 0;
}

// ----------------------------------------------------------------------------
// WCSPH (weakly compressible SPH), full neighbour list, fixed wall particles.
//   kernel:     cubic spline, support 2h (Monaghan & Lattanzio 1985)
//   EOS:        p = B ((rho/rho0)^7 - 1), B = c0^2 rho0 / 7 (Tait; Monaghan 1994)
//   viscosity:  Pi_ab = -alpha c0 h mu/rho_bar for v_ab.r_ab < 0,
//               mu = v_ab.r_ab / (r^2 + 0.01 h^2) (Monaghan 1992)
//   momentum:   dv_a/dt = -sum_b m_b (p_a/rho_a^2 + p_b/rho_b^2 + Pi_ab) gradW_ab + g
//   continuity: drho_a/dt = sum_b m_b v_ab . gradW_ab
// type: 0 = fluid, 1 = wall (walls do not move; their rho evolves, p from EOS)
template <class T> struct SPHP {
    T h, m, c0, rho0, B, alpha, gz, eta2, w3, dw3;
};

template <class T> static SPHP<T> sph_params(T h, T m, T c0, T rho0, T alpha, T gz) {
    SPHP<T> P;
    P.h = h;
    P.m = m;
    P.c0 = c0;
    P.rho0 = rho0;
    P.B = c0 * c0 * rho0 / T(7);
    P.alpha = alpha;
    P.gz = gz;
    P.eta2 = T(0.01) * h * h;
    const T pi = (T)3.14159265358979323846;
    P.w3 = T(1) / (pi * h * h * h);
    P.dw3 = P.w3 / h;
    return P;
}

// dW/dr / r of the cubic spline, q = r/h
template <class T> inline T sph_dwdr_over_r(const SPHP<T>& P, T r) {
    T q = r / P.h;
    T d;
    if (q < T(1)) d = (T(-3) * q + T(2.25) * q * q);
    else if (q < T(2)) d = T(-0.75) * (T(2) - q) * (T(2) - q);
    else d = 0;
    return P.dw3 * d / r;
}

template <class T> inline T sph_eos(const SPHP<T>& P, T rho) {
    T x = rho / P.rho0;
    T x2 = x * x;
    T x7 = x2 * x2 * x2 * x;
    return P.B * (x7 - T(1));
}

template <class T>
static void sph_rates_impl(const T* pos, const T* vel, const T* rho, const int* type, long n, const long* offsets,
                           const long* counts, const int* idx, T h, T m, T c0, T rho0, T alpha, T gz, T* acc,
                           T* drho) {
    SPHP<T> P = sph_params(h, m, c0, rho0, alpha, gz);
    const T two_h = T(2) * h;
    const T r2c = two_h * two_h;
#pragma omp parallel for schedule(static)
    for (long a = 0; a < n; ++a) {
        const T* xa = pos + 3 * a;
        const T* va = vel + 3 * a;
        T pa = sph_eos(P, rho[a]);
        T ra2 = rho[a] * rho[a];
        T ax = 0, ay = 0, az = 0, dr = 0;
        for (long k = offsets[a]; k < offsets[a] + counts[a]; ++k) {
            long b = idx[k];
            if (b == a) continue;
            const T* xb = pos + 3 * b;
            T dx = xa[0] - xb[0], dy = xa[1] - xb[1], dz = xa[2] - xb[2];
            T r2 = std::fma(dz, dz, std::fma(dy, dy, dx * dx));
            if (r2 >= r2c || r2 == T(0)) continue;
            T r = std::sqrt(r2);
            T dwr = sph_dwdr_over_r(P, r);
            T vx = va[0] - vel[3 * b], vy = va[1] - vel[3 * b + 1], vz = va[2] - vel[3 * b + 2];
            T vr = vx * dx + vy * dy + vz * dz;
            T pb = sph_eos(P, rho[b]);
            T pi_ab = 0;
            if (vr < 0) {
                T mu = h * vr / (r2 + P.eta2);
                T rbar = T(0.5) * (rho[a] + rho[b]);
                pi_ab = -alpha * c0 * mu / rbar;
            }
            T coef = -m * (pa / ra2 + pb / (rho[b] * rho[b]) + pi_ab) * dwr;
            ax += coef * dx;
            ay += coef * dy;
            az += coef * dz;
            dr += m * vr * dwr;
        }
        if (type[a] == 0) {
            acc[3 * a] = ax;
            acc[3 * a + 1] = ay;
            acc[3 * a + 2] = az + gz;
        } else {
            acc[3 * a] = acc[3 * a + 1] = acc[3 * a + 2] = 0;
        }
        drho[a] = dr;
    }
}

// WCSPH time integration (kick-drift-kick, the same scheme as the GPU driver):
//   v' = v + dt/2 a ; rho' = rho + dt/2 drho ; x += dt v' (fluid only) ;
//   (a, drho) = rates(x, v', rho') over pairs with r < 2h (cell-list walk) ;
//   v = v' + dt/2 a ; rho = rho' + dt/2 drho.
// Wall particles (type 1) keep v = 0 and do not move; their density evolves.
// E[s] = (kinetic energy of the fluid, sum of densities, 0, 0) after step s.
template <class T>
static int md_sph_impl(T* x, T* v, T* rho, const int* type, long n, const T* lo, const T* hi, T h, T m, T c0, T rho0,
                       T alpha, T gz, T dt, int steps, double* E) {
    const int bc[3] = {0, 0, 0};
    const T g0[3] = {0, 0, 0};
    T r = T(2) * h;
    T blo[3], sp[3];
    int dv[3], gs[3];
    long nc;
    cl_geometry_impl(lo, hi, g0, r, (T)1.013, 1, blo, sp, dv, gs, &nc);
    std::vector<long> cnt(n), off(n + 1);
    std::vector<int> idx;
    std::vector<T> acc(3 * n), drho(n);
    auto rates = [&]() {
        verlet_impl(x, n, n, blo, sp, dv, 1, r, cnt.data(), (const long*)nullptr, (int*)nullptr);
        off[0] = 0;
        for (long i = 0; i < n; ++i) off[i + 1] = off[i] + cnt[i];
        idx.assign(off[n], 0);
        verlet_impl(x, n, n, blo, sp, dv, 1, r, (long*)nullptr, off.data(), idx.data());
        sph_rates_impl(x, v, rho, type, n, off.data(), cnt.data(), idx.data(), h, m, c0, rho0, alpha, gz, acc.data(),
                       drho.data());
    };
    (void)bc;
    rates();
    T half = T(0.5) * dt;
    for (int s = 0; s < steps; ++s) {
        for (long i = 0; i < n; ++i) {
            if (type[i] == 0) {
                for (int d = 0; d < 3; ++d) v[3 * i + d] += half * acc[3 * i + d];
                for (int d = 0; d < 3; ++d) x[3 * i + d] += dt * v[3 * i + d];
            }
            rho[i] += half * drho[i];
        }
        rates();
        double ke = 0, rs = 0;
        for (long i = 0; i < n; ++i) {
            if (type[i] == 0) {
                for (int d = 0; d < 3; ++d) v[3 * i + d] += half * acc[3 * i + d];
                ke += 0.5 * (double)m *
                      ((double)v[3 * i] * v[3 * i] + (double)v[3 * i + 1] * v[3 * i + 1] +
                       (double)v[3 * i + 2] * v[3 * i + 2]);
            }
            rho[i] += half * drho[i];
            rs += rho[i];
        }
        E[4 * s] = ke;
        E[4 * s + 1] = rs;
        E[4 * s + 2] = 0;
        E[4 * s + 3] = 0;
    }
    return 0;
}

extern "C" {

int or_md_sph_d(double* x, double* v, double* rho, const int* type, long n, const double* lo, const double* hi,
                double h, double m, double c0, double rho0, double alpha, double gz, double dt, int steps, double* E) {
    return md_sph_impl(x, v, rho, type, n, lo, hi, h, m, c0, rho0, alpha, gz, dt, steps, E);
}

// -- periodic wrap
void or_wrap_d(double* pos, long n, const double* lo, const double* hi, const int* bc) { wrap_impl(pos, n, lo, hi, bc); }
void or_wrap_f(float* pos, long n, const float* lo, const float* hi, const int* bc) { wrap_impl(pos, n, lo, hi, bc); }

// -- ghost boxes (sorted by shift id) and shift vectors
int or_ghost_boxes_d(const double* lo, const double* hi, const int* bc, const double* g, double* blo, double* bhi,
                     int* sv) {
    return ghost_boxes_impl(lo, hi, bc, g, blo, bhi, sv);
}
int or_ghost_boxes_f(const float* lo, const float* hi, const int* bc, const float* g, float* blo, float* bhi,
                     int* sv) {
    return ghost_boxes_impl(lo, hi, bc, g, blo, bhi, sv);
}
void or_shift_vectors_d(const double* lo, const double* hi, double* shifts) {
    for (int l = 0; l < 27; ++l) shift_vector(comb_from_lin(l), lo, hi, shifts + 3 * l);
}
void or_shift_vectors_f(const float* lo, const float* hi, float* shifts) {
    for (int l = 0; l < 27; ++l) shift_vector(comb_from_lin(l), lo, hi, shifts + 3 * l);
}

// -- image kernels over explicit box lists
void or_ghost_count_d(const double* pos, long n, const double* blo, const double* bhi, const int* sv, int nb,
                      int* out) {
    ghost_count_impl(pos, n, blo, bhi, sv, nb, out);
}
void or_ghost_count_f(const float* pos, long n, const float* blo, const float* bhi, const int* sv, int nb, int* out) {
    ghost_count_impl(pos, n, blo, bhi, sv, nb, out);
}
long or_ghost_images_d(const double* pos, long n, const double* blo, const double* bhi, const int* sv, int nb,
                       const double* shifts, double* img, int* src, int* shf, long cap) {
    return ghost_images_impl(pos, n, blo, bhi, sv, nb, shifts, img, src, shf, cap);
}
long or_ghost_images_f(const float* pos, long n, const float* blo, const float* bhi, const int* sv, int nb,
                       const float* shifts, float* img, int* src, int* shf, long cap) {
    return ghost_images_impl(pos, n, blo, bhi, sv, nb, shifts, img, src, shf, cap);
}
long or_ghost_get_d(const double* pos, long n, const double* lo, const double* hi, const int* bc, const double* g,
                    double* img, int* src, int* shf, long cap) {
    return ghost_get_impl(pos, n, lo, hi, bc, g, img, src, shf, cap);
}
long or_ghost_get_f(const float* pos, long n, const float* lo, const float* hi, const int* bc, const float* g,
                    float* img, int* src, int* shf, long cap) {
    return ghost_get_impl(pos, n, lo, hi, bc, g, img, src, shf, cap);
}

// -- cell list
void or_cl_geometry_d(const double* lo, const double* hi, const double* g, double r_cut, double enlarge, int pad,
                      double* box_lo, double* spacing, int* div, int* gs, long* ncells) {
    cl_geometry_impl(lo, hi, g, r_cut, enlarge, pad, box_lo, spacing, div, gs, ncells);
}
void or_cl_geometry_f(const float* lo, const float* hi, const float* g, float r_cut, float enlarge, int pad,
                      float* box_lo, float* spacing, int* div, int* gs, long* ncells) {
    cl_geometry_impl(lo, hi, g, r_cut, enlarge, pad, box_lo, spacing, div, gs, ncells);
}
void or_cl_build_d(const double* pos, long n, const double* box_lo, const double* spacing, const int* div, int pad,
                   long* cell_start, int* sorted, long* cell_of_p) {
    cl_build_impl(pos, n, box_lo, spacing, div, pad, cell_start, sorted, cell_of_p);
}
void or_cl_build_f(const float* pos, long n, const float* box_lo, const float* spacing, const int* div, int pad,
                   long* cell_start, int* sorted, long* cell_of_p) {
    cl_build_impl(pos, n, box_lo, spacing, div, pad, cell_start, sorted, cell_of_p);
}

// -- neighbour lists
long or_verlet_d(const double* pos, long n_dom, long n_all, const double* box_lo, const double* spacing,
                 const int* div, int pad, double r, long* counts, const long* offsets, int* idx) {
    return verlet_impl(pos, n_dom, n_all, box_lo, spacing, div, pad, r, counts, offsets, idx);
}
long or_verlet_f(const float* pos, long n_dom, long n_all, const float* box_lo, const float* spacing, const int* div,
                 int pad, float r, long* counts, const long* offsets, int* idx) {
    return verlet_impl(pos, n_dom, n_all, box_lo, spacing, div, pad, r, counts, offsets, idx);
}
long or_brute_nn_d(const double* pos, long n_dom, long n_all, double r, long* counts, const long* offsets, int* idx) {
    return brute_nn_impl(pos, n_dom, n_all, r, counts, offsets, idx);
}
long or_brute_nn_f(const float* pos, long n_dom, long n_all, float r, long* counts, const long* offsets, int* idx) {
    return brute_nn_impl(pos, n_dom, n_all, r, counts, offsets, idx);
}

// -- pair kernels
void or_lj_verlet_d(const double* pos, long n_dom, const long* offsets, const long* counts, const int* idx,
                    double eps, double sigma, double rc, double* f, double* pe, double* vir) {
    lj_verlet_impl(pos, n_dom, offsets, counts, idx, eps, sigma, rc, f, pe, vir);
}
void or_lj_cell_d(const double* pos, long n_dom, long n_all, const double* box_lo, const double* spacing,
                  const int* div, int pad, double eps, double sigma, double rc, double* f, double* pe, double* vir) {
    lj_cell_impl(pos, n_dom, n_all, box_lo, spacing, div, pad, eps, sigma, rc, f, pe, vir);
}
void or_test_force_f(const float* pos, const float* prop0, long n_dom, long n_all, const float* box_lo,
                     const float* spacing, const int* div, int pad, float* out) {
    test_force_impl(pos, prop0, n_dom, n_all, box_lo, spacing, div, pad, out);
}
void or_test_force_d(const double* pos, const double* prop0, long n_dom, long n_all, const double* box_lo,
                     const double* spacing, const int* div, int pad, double* out) {
    test_force_impl(pos, prop0, n_dom, n_all, box_lo, spacing, div, pad, out);
}
void or_sph_rates_d(const double* pos, const double* vel, const double* rho, const int* type, long n,
                    const long* offsets, const long* counts, const int* idx, double h, double m, double c0,
                    double rho0, double alpha, double gz, double* acc, double* drho) {
    sph_rates_impl(pos, vel, rho, type, n, offsets, counts, idx, h, m, c0, rho0, alpha, gz, acc, drho);
}

// -- MD driver
int or_md_lj_d(double* x, double* v, long n, const double* lo, const double* hi, const int* bc, const double* ghost,
               double rc, double skin, double eps, double sigma, double dt, double mass, int steps, double* E,
               double* t_loop) {
    return md_lj_impl(x, v, n, lo, hi, bc, ghost, rc, skin, eps, sigma, dt, mass, steps, E, t_loop);
}

int or_num_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
void or_set_threads(int t) {
#ifdef _OPENMP
    if (t > 0) omp_set_num_threads(t);
#else
    (void)t;
#endif
}

}  // extern "C"
