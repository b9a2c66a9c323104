#include <utility>
// pd_celllist.cu -- GPU cell list: geometry, counting-sort build, reorder / restoreOrder,
// and the reference's test pair functor walking getNNIteratorBox.
//
// Build (replaces openfpm_data's CellList_gpu::construct, called from
// updateCellListGPU, vector_dist.hpp:1334-1401):
//   1. hash      cell id of every particle + warp-aggregated atomic count per cell
//                (__match_any_sync groups equal keys: one atomic per distinct key per warp)
//   2. scan      exclusive scan of the counts -> cell_start
//   3. scatter   slot = cell_start[c] + rank returned by the atomic
//   4. stabilise one warp per cell ranks its members by index, so the in-cell
//                order is ascending particle index (bit-identical to a stable sort)
// Geometry: cl_param_calculate of openfpm_data (call site vector_dist.hpp:1246):
// the domain enlarged by the ghost magnified by `enlarge`, div = floor(len/r)+1
// cells of side r, one padding layer per side.
#include "pd_device.cuh"
#include "pd_internal.cuh"

namespace pd {

template <class T> static Grid<T> make_grid(const pd_cl_s* cl) {
    Grid<T> G;
    for (int d = 0; d < 3; ++d) {
        G.lo[d] = (T)cl->box_lo[d];
        G.sp[d] = (T)cl->spacing[d];
        G.gs[d] = cl->gs[d];
    }
    G.pad = cl->pad;
    return G;
}

// geometry in the vector's precision, same operation sequence as the oracle
template <class T> static void geom_t(pd_cl cl, pd_vd h, T r_cut, T enlarge) {
    cl->ncells = 1;
    for (int d = 0; d < 3; ++d) {
        T g = (T)h->g[d];
        T gl = (-g) * enlarge, gh = g * enlarge;
        T pl = (T)h->lo[d] + gl, ph = (T)h->hi[d] + gh;
        long dv = (long)((ph - pl) / r_cut) + 1;
        ph = pl + (T)dv * r_cut;
        cl->box_lo[d] = pl;
        cl->spacing[d] = (ph - pl) / (T)dv;
        cl->div[d] = (int)dv;
        cl->gs[d] = (int)dv + 2 * cl->pad;
        cl->ncells *= cl->gs[d];
    }
}

int cl_geometry(pd_cl cl, pd_vd h, double r_cut, double enlarge, int nn_box) {
    if (!(r_cut > 0) || nn_box < 1 || nn_box > 4) {
        set_error("cell list: r_cut must be > 0 and NNIteratorBox in [1,4]");
        return PD_EINVAL;
    }
    cl->owner = h;
    cl->r_cut = r_cut;
    cl->nn_box = nn_box;
    cl->pad = nn_box;
    cl->enlarge = enlarge;
    if (h->dtype == PD_F64) geom_t<double>(cl, h, r_cut, enlarge);
    else geom_t<float>(cl, h, (float)r_cut, (float)enlarge);
    if (cl->ncells > (1L << 30)) {
        set_error("cell list: %ld cells is too many (r_cut too small for the box)", cl->ncells);
        return PD_EINVAL;
    }
    return PD_OK;
}

// 1. hash + warp-aggregated count
template <class T>
__global__ void k_cl_hash(const typename V4<T>::type* __restrict__ pos, long n_bound,
                          const unsigned int* __restrict__ n_dev, long n_add, Grid<T> G,
                          unsigned int* __restrict__ cnt, unsigned int* __restrict__ cell_of,
                          unsigned int* __restrict__ slot, unsigned int* __restrict__ err) {
    long n = n_dev ? (long)*n_dev + n_add : n_bound;
    if (n > n_bound) n = n_bound;
    unsigned int bad = 0;
    for (long base = blockIdx.x * (long)blockDim.x; base < n; base += (long)gridDim.x * blockDim.x) {
        long i = base + threadIdx.x;
        bool ok = i < n;
        unsigned int act = __ballot_sync(0xffffffffu, ok);
        if (ok) {
            typename V4<T>::type r = ld4(pos, i);
            unsigned int c = (unsigned int)G.cell(r.x, r.y, r.z, bad);
            cell_of[i] = c;
            slot[i] = warp_agg_inc(cnt, c, act);
        }
    }
    if (bad) atomicOr(err, ERR_CELL_RANGE);
}

// 3. scatter to the (unordered) slot inside the cell
__global__ void k_cl_scatter(long n_bound, const unsigned int* __restrict__ n_dev, long n_add,
                             const unsigned int* __restrict__ cell_of, const unsigned int* __restrict__ slot,
                             const unsigned int* __restrict__ start, int* __restrict__ out) {
    long n = n_dev ? (long)*n_dev + n_add : n_bound;
    if (n > n_bound) n = n_bound;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        out[start[cell_of[i]] + slot[i]] = (int)i;
}

// 4. stabilise: one warp per cell puts its members in ascending index order
__global__ void __launch_bounds__(256) k_cl_stabilise(long ncells, const unsigned int* __restrict__ start,
                                                      const int* __restrict__ in, int* __restrict__ out) {
    __shared__ int cell_sort_buf[256 / 32][CELL_SORT_SMEM];
    long warp = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5;
    long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    for (long c = warp; c < ncells; c += nwarps) {
        const unsigned int s = start[c], e = start[c + 1];
        warp_cell_order(in + s, out + s, e - s, cell_sort_buf[threadIdx.x >> 5]);
    }
}

int cl_build(pd_vd h, pd_cl cl, long n_part, const unsigned int* n_part_dev, cudaStream_t st, long first) {
    // n_part: exact count, or (with n_part_dev) an upper bound; the device count is *n_part_dev + n_real
    long nc = cl->ncells;
    PD_TRY(cl->cell_cnt.ensure(sizeof(unsigned int) * (nc + 1)));
    PD_TRY(cl->cell_start.ensure(sizeof(unsigned int) * (nc + 1)));
    long nb = n_part > 0 ? n_part : 1;
    PD_TRY(cl->sorted.ensure(sizeof(int) * nb));
    PD_TRY(cl->sorted_tmp.ensure(sizeof(int) * nb));
    PD_TRY(cl->cell_of.ensure(sizeof(unsigned int) * nb));
    PD_TRY(cl->slot.ensure(sizeof(unsigned int) * nb));
    PD_CUDA(cudaMemsetAsync(cl->cell_cnt.p, 0, sizeof(unsigned int) * (nc + 1), st));
    long n_add = n_part_dev ? h->n_real : 0;
    if (n_part > 0) {
        unsigned g = grid_for(n_part, 256);
        if (h->dtype == PD_F64)
            pd::launch(k_cl_hash<double>, g, 256, 0, st, (const double4*)h->pos + first, n_part, n_part_dev, n_add,
                                                 make_grid<double>(cl), cl->cell_cnt.as<unsigned int>(),
                                                 cl->cell_of.as<unsigned int>(), cl->slot.as<unsigned int>(),
                                                 &h->ctrl->err);
        else
            pd::launch(k_cl_hash<float>, g, 256, 0, st, (const float4*)h->pos + first, n_part, n_part_dev, n_add,
                                                make_grid<float>(cl), cl->cell_cnt.as<unsigned int>(),
                                                cl->cell_of.as<unsigned int>(), cl->slot.as<unsigned int>(),
                                                &h->ctrl->err);
        PD_LAUNCH_CHECK();
    }
    PD_TRY(scan_u32(cl->cell_cnt.as<unsigned int>(), cl->cell_start.as<unsigned int>(), nc + 1, nullptr,
                    h->scan_scratch, st));
    if (n_part > 0) {
        unsigned g = grid_for(n_part, 256);
        pd::launch(k_cl_scatter, g, 256, 0, st, n_part, n_part_dev, n_add, cl->cell_of.as<unsigned int>(),
                                        cl->slot.as<unsigned int>(), cl->cell_start.as<unsigned int>(),
                                        cl->sorted_tmp.as<int>());
        pd::launch(k_cl_stabilise, grid_for(nc * 32, 256), 256, 0, st, nc, cl->cell_start.as<unsigned int>(),
                                                                 cl->sorted_tmp.as<int>(), cl->sorted.as<int>());
        PD_LAUNCH_CHECK();
    }
    cl->n_part = n_part;
    cl->ghost_marker = h->n_real;
    cl->epoch = h->epoch;
    return PD_OK;
}

// reorder: dst[k] = src[sorted[k]] (gather, coalesced writes) for positions, gid and properties
template <class T>
__global__ void k_gather4(const typename V4<T>::type* __restrict__ src, typename V4<T>::type* __restrict__ dst,
                          const int* __restrict__ ids, long n) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x)
        st4(dst, k, ld4(src, ids[k]));
}
template <class E>
__global__ void k_gather(const E* __restrict__ src, E* __restrict__ dst, const int* __restrict__ ids, long n) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x)
        dst[k] = src[ids[k]];
}
// the same for up to GCOLS columns at once (positions, global ids, property components):
// each permutation entry read once; a column's element is 4, 8, 16 or 32 bytes
static constexpr int GCOLS = 16;
struct GatherCols {
    const char* src[GCOLS];
    char* dst[GCOLS];
    int esize[GCOLS];
    int ncol;
    // with FP64 records in column 0: the same records also to xb and as (x, y) / z copies
    double4* xb;
    double2* sxy;
    double* sz;
};
__global__ void k_gather_cols(const int* __restrict__ ids, long n, GatherCols G) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        const long id = ids[k];
        if (G.xb) {
            const double4 x = ld4(reinterpret_cast<const double4*>(G.src[0]), id);
            st4(G.xb, k, x);
            G.sxy[k] = make_double2(x.x, x.y);
            G.sz[k] = x.z;
        }
        for (int c = 0; c < G.ncol; ++c) {
            const int es = G.esize[c];
            if (es == 32) {
                const double2* s2 = reinterpret_cast<const double2*>(G.src[c]) + 2 * id;
                double2* d2 = reinterpret_cast<double2*>(G.dst[c]) + 2 * k;
                const double2 a = __ldg(s2), b = __ldg(s2 + 1);
                d2[0] = a;
                d2[1] = b;
            } else if (es == 16) {
                reinterpret_cast<double2*>(G.dst[c])[k] = __ldg(reinterpret_cast<const double2*>(G.src[c]) + id);
            } else if (es == 8) {
                reinterpret_cast<long long*>(G.dst[c])[k] = __ldg(reinterpret_cast<const long long*>(G.src[c]) + id);
            } else {
                reinterpret_cast<int*>(G.dst[c])[k] = __ldg(reinterpret_cast<const int*>(G.src[c]) + id);
            }
        }
    }
}

// restore: dst[sorted[k]] = src[k]
template <class T>
__global__ void k_scatter4(const typename V4<T>::type* __restrict__ src, typename V4<T>::type* __restrict__ dst,
                           const int* __restrict__ ids, long n) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x)
        st4(dst, ids[k], ld4(src, k));
}
template <class E>
__global__ void k_scatter(const E* __restrict__ src, E* __restrict__ dst, const int* __restrict__ ids, long n) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x)
        dst[ids[k]] = src[k];
}

static int permute(pd_vd h, const int* ids, long n, unsigned long prop_mask, bool with_pos, bool with_gid,
                   bool restore, cudaStream_t st) {
    if (n <= 0) return PD_OK;
    unsigned g = grid_for(n, 256);
    size_t maxb = (size_t)n * h->pos_bytes;
    for (auto& P : h->props) maxb = std::max(maxb, (size_t)n * P.esize);
    PD_TRY(h->tmp2.ensure(maxb));
    if (with_pos) {
        if (h->dtype == PD_F64) {
            if (restore) pd::launch(k_scatter4<double>, g, 256, 0, st, (const double4*)h->pos, h->tmp2.as<double4>(), ids, n);
            else pd::launch(k_gather4<double>, g, 256, 0, st, (const double4*)h->pos, h->tmp2.as<double4>(), ids, n);
        } else {
            if (restore) pd::launch(k_scatter4<float>, g, 256, 0, st, (const float4*)h->pos, h->tmp2.as<float4>(), ids, n);
            else pd::launch(k_gather4<float>, g, 256, 0, st, (const float4*)h->pos, h->tmp2.as<float4>(), ids, n);
        }
        PD_LAUNCH_CHECK();
        PD_CUDA(cudaMemcpyAsync(h->pos, h->tmp2.p, (size_t)n * h->pos_bytes, cudaMemcpyDeviceToDevice, st));
    }
    if (with_gid) {
        if (restore) pd::launch(k_scatter<int>, g, 256, 0, st, h->gid, h->tmp2.as<int>(), ids, n);
        else pd::launch(k_gather<int>, g, 256, 0, st, h->gid, h->tmp2.as<int>(), ids, n);
        PD_LAUNCH_CHECK();
        PD_CUDA(cudaMemcpyAsync(h->gid, h->tmp2.p, sizeof(int) * n, cudaMemcpyDeviceToDevice, st));
    }
    for (size_t p = 0; p < h->props.size(); ++p) {
        if (!(prop_mask & (1ul << p))) continue;
        Prop& P = h->props[p];
        for (int c = 0; c < P.ncomp; ++c) {
            char* base = P.d + (size_t)c * h->cap * P.esize;
            if (P.esize == 8) {
                if (restore) pd::launch(k_scatter<long long>, g, 256, 0, st, (const long long*)base, h->tmp2.as<long long>(), ids, n);
                else pd::launch(k_gather<long long>, g, 256, 0, st, (const long long*)base, h->tmp2.as<long long>(), ids, n);
            } else {
                if (restore) pd::launch(k_scatter<int>, g, 256, 0, st, (const int*)base, h->tmp2.as<int>(), ids, n);
                else pd::launch(k_gather<int>, g, 256, 0, st, (const int*)base, h->tmp2.as<int>(), ids, n);
            }
            PD_LAUNCH_CHECK();
            PD_CUDA(cudaMemcpyAsync(base, h->tmp2.p, (size_t)n * P.esize, cudaMemcpyDeviceToDevice, st));
        }
    }
    return PD_OK;
}

int gather_bytes(const void* src, void* dst, const int* ids, long n, int esize, cudaStream_t st) {
    if (n <= 0) return PD_OK;
    unsigned g = grid_for(n, 256);
    switch (esize) {
        case 1: pd::launch(k_gather<unsigned char>, g, 256, 0, st, (const unsigned char*)src, (unsigned char*)dst, ids, n); break;
        case 4: pd::launch(k_gather<int>, g, 256, 0, st, (const int*)src, (int*)dst, ids, n); break;
        case 8: pd::launch(k_gather<long long>, g, 256, 0, st, (const long long*)src, (long long*)dst, ids, n); break;
        case 16: pd::launch(k_gather4<float>, g, 256, 0, st, (const float4*)src, (float4*)dst, ids, n); break;
        case 32: pd::launch(k_gather4<double>, g, 256, 0, st, (const double4*)src, (double4*)dst, ids, n); break;
        default: set_error("gather_bytes: element size %d", esize); return PD_EINVAL;
    }
    PD_LAUNCH_CHECK();
    return PD_OK;
}

// The gather of a reorder straight into the vector's spare storage, which then
// takes the place of the storage (every column moved once, not gathered into
// scratch and copied back).  Slots from n_part on hold the spare's old contents and
// views taken before are stale: for a caller that rewrites the slots past n_part
// (the images) and moves the epoch on, and not inside a stream capture (the
// capture would keep the first pair of addresses).
static int permute_swap(pd_vd h, const int* ids, long n, unsigned long prop_mask, bool with_pos, bool with_gid,
                        cudaStream_t st, const ReorderExtra* extra, bool* done) {
    if (n <= 0) return PD_OK;
    if (!h->spare_pos || h->spare_cap != h->cap || h->spare_props.size() != h->props.size()) {
        free_storage(h->spare_pos, h->spare_gid, h->spare_props);
        h->spare_pos = nullptr;
        h->spare_gid = nullptr;
        h->spare_props.clear();
        h->spare_cap = 0;
        PD_TRY(alloc_storage(h, h->cap, &h->spare_pos, &h->spare_gid, h->spare_props));
        h->spare_cap = h->cap;
    }
    const unsigned g = grid_for(n, 256);
    // every column moved by one gather kernel per GCOLS columns
    GatherCols G{};
    auto flush = [&]() -> int {
        if (G.ncol == 0) return PD_OK;
        pd::launch(k_gather_cols, g, 256, 0, st, ids, n, G);
        PD_LAUNCH_CHECK();
        G.ncol = 0;
        G.xb = nullptr;  // only with the records in column 0
        G.sxy = nullptr;
        G.sz = nullptr;
        return PD_OK;
    };
    auto add = [&](const void* src, void* dst, int esize) -> int {
        if (G.ncol == GCOLS) PD_TRY(flush());
        G.src[G.ncol] = (const char*)src;
        G.dst[G.ncol] = (char*)dst;
        G.esize[G.ncol] = esize;
        G.ncol++;
        return PD_OK;
    };
    if (with_pos) PD_TRY(add(h->pos, h->spare_pos, (int)h->pos_bytes));
    if (extra && with_pos && h->dtype == PD_F64) {
        // column 0 holds the records: the first launch also writes the extra outputs
        G.xb = extra->xb;
        G.sxy = extra->sxy;
        G.sz = extra->sz;
        if (done) *done = true;
    }
    if (with_gid) PD_TRY(add(h->gid, h->spare_gid, 4));
    for (size_t p = 0; p < h->props.size(); ++p) {
        if (!(prop_mask & (1ul << p))) continue;
        Prop& P = h->props[p];
        for (int c = 0; c < P.ncomp; ++c) {
            const size_t o = (size_t)c * h->cap * P.esize;
            PD_TRY(add(P.d + o, h->spare_props[p] + o, P.esize));
        }
    }
    PD_TRY(flush());
    if (with_pos) std::swap(h->pos, h->spare_pos);
    if (with_gid) std::swap(h->gid, h->spare_gid);
    for (size_t p = 0; p < h->props.size(); ++p)
        if (prop_mask & (1ul << p)) std::swap(h->props[p].d, h->spare_props[p]);
    return PD_OK;
}

int cl_reorder(pd_vd h, pd_cl cl, long n_part, unsigned long prop_mask, bool with_pos, bool with_gid,
               cudaStream_t st, bool swap, const ReorderExtra* extra, bool* done) {
    if (done) *done = false;
    if (swap && !g_capturing && !g_alloc_ctx)
        return permute_swap(h, cl->sorted.as<int>(), n_part, prop_mask, with_pos, with_gid, st, extra, done);
    return permute(h, cl->sorted.as<int>(), n_part, prop_mask, with_pos, with_gid, false, st);
}

// sorted slots of the domain particles, in sorted order (getDomainSortIds)
__global__ void k_dom_flags(const int* __restrict__ sorted, long n, long gm, unsigned int* __restrict__ f) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x)
        f[k] = sorted[k] < gm ? 1u : 0u;
}
__global__ void k_dom_compact(const int* __restrict__ sorted, long n, long gm, const unsigned int* __restrict__ pos,
                              int* __restrict__ out) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x)
        if (sorted[k] < gm) out[pos[k]] = (int)k;
}

// the reference's calculate_force / calculate_force_sort
template <class T>
__global__ void k_test_force(const typename V4<T>::type* __restrict__ pos, long gm, Grid<T> G, int r,
                             const unsigned int* __restrict__ cs, const int* __restrict__ sorted,
                             const int* __restrict__ dom_sort, int use_sort, const T* __restrict__ p0,
                             T* __restrict__ f0, T* __restrict__ f1, T* __restrict__ f2) {
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < gm; t += (long)gridDim.x * blockDim.x) {
        long p = use_sort ? dom_sort[t] : t;
        typename V4<T>::type xp = ld4(pos, p);
        unsigned int bad = 0;
        int c0 = G.coord(0, xp.x, bad), c1 = G.coord(1, xp.y, bad), c2 = G.coord(2, xp.z, bad);
        T fx = 0, fy = 0, fz = 0;
        for (int dz = -r; dz <= r; ++dz)
            for (int dy = -r; dy <= r; ++dy)
                for (int dx = -r; dx <= r; ++dx) {
                    int x = c0 + dx, y = c1 + dy, z = c2 + dz;
                    if (x < 0 || y < 0 || z < 0 || x >= G.gs[0] || y >= G.gs[1] || z >= G.gs[2]) continue;
                    long c = x + (long)G.gs[0] * (y + (long)G.gs[1] * z);
                    for (unsigned int k = cs[c]; k < cs[c + 1]; ++k) {
                        long q = use_sort ? (long)k : (long)sorted[k];
                        if (q == p) continue;
                        typename V4<T>::type xq = ld4(pos, q);
                        T rx = xq.x - xp.x, ry = xq.y - xp.y, rz = xq.z - xp.z;
                        T nrm = sqrt(rx * rx + ry * ry + rz * rz);
                        if (nrm > T(1e-6)) {
                            T w = p0[q];
                            fx += w * (rx / nrm);
                            fy += w * (ry / nrm);
                            fz += w * (rz / nrm);
                        }
                    }
                }
        f0[p] = fx;
        f1[p] = fy;
        f2[p] = fz;
    }
}

}  // namespace pd

using namespace pd;

extern "C" {

int pd_celllist_create(pd_vd h, double r_cut, int opt, int nn_box, double enlarge_factor, pd_cl* out) {
    if (!h || !out) return PD_EINVAL;
    pd_cl cl = new pd_cl_s();
    cl->opt = opt;
    int r = cl_geometry(cl, h, r_cut, enlarge_factor > 0 ? enlarge_factor : (double)1.013f, nn_box);
    if (r != PD_OK) {
        delete cl;
        return r;
    }
    *out = cl;
    return PD_OK;
}

int pd_celllist_destroy(pd_cl cl) {
    if (!cl) return PD_EINVAL;
    cl->cell_start.release();
    cl->cell_cnt.release();
    cl->sorted.release();
    cl->sorted_tmp.release();
    cl->cell_of.release();
    cl->slot.release();
    cl->dom_sort.release();
    cl->flags.release();
    delete cl;
    return PD_OK;
}

int pd_celllist_update(pd_vd h, pd_cl cl, unsigned long prop_mask, void* stream) {
    if (!h || !cl || cl->owner != h) return PD_EINVAL;
    cudaStream_t st = S(stream);
    long n = h->n_total;
    PD_TRY(cl_build(h, cl, n, nullptr, st));
    // getDomainSortIds: sorted slots holding domain particles
    PD_TRY(cl->flags.ensure(sizeof(unsigned int) * (n + 1)));
    PD_TRY(cl->dom_sort.ensure(sizeof(int) * (n + 1)));
    if (n > 0) {
        unsigned g = grid_for(n, 256);
        pd::launch(k_dom_flags, g, 256, 0, st, cl->sorted.as<int>(), n, h->n_real, cl->flags.as<unsigned int>());
        PD_LAUNCH_CHECK();
        PD_TRY(scan_u32(cl->flags.as<unsigned int>(), cl->slot.as<unsigned int>(), n, nullptr, h->scan_scratch, st));
        pd::launch(k_dom_compact, g, 256, 0, st, cl->sorted.as<int>(), n, h->n_real, cl->slot.as<unsigned int>(),
                                         cl->dom_sort.as<int>());
        PD_LAUNCH_CHECK();
    }
    if (cl->opt & PD_CL_GPU_REORDER) {
        bool wp = (cl->opt & PD_CL_GPU_REORDER_POSITION) != 0;
        unsigned long pm = (cl->opt & PD_CL_GPU_REORDER_PROPERTY) ? prop_mask : 0ul;
        PD_TRY(cl_reorder(h, cl, n, pm, wp, true, st));
        cl->reordered = true;
        cl->reordered_mask = pm;
    } else {
        cl->reordered = false;
    }
    PD_TRY(read_ctrl(h, st));
    if (h->ctrl_h->err & ERR_CELL_RANGE) {
        unsigned int z = 0;
        cudaMemcpy(&h->ctrl->err, &z, sizeof(z), cudaMemcpyHostToDevice);
        set_error("cell list: particles outside the cell grid (clamped to the border cells)");
        h->ctrl_h->err = 0;
    }
    return PD_OK;
}

int pd_restore_order(pd_vd h, pd_cl cl, unsigned long prop_mask, void* stream) {
    if (!h || !cl || cl->owner != h) return PD_EINVAL;
    if (!cl->reordered) {
        set_error("restore_order: the cell list did not reorder the vector");
        return PD_ESTATE;
    }
    cudaStream_t st = S(stream);
    bool wp = (cl->opt & PD_CL_GPU_REORDER_POSITION) != 0;
    // the listed properties (written in cell order) and every property the update
    // reordered return to the original order: the reference swaps its original
    // arrays back, so a reordered property that is not listed keeps its original
    // order (vector_dist.hpp:3042-3049)
    PD_TRY(permute(h, cl->sorted.as<int>(), cl->n_part, prop_mask | cl->reordered_mask, wp, true, true, st));
    cl->reordered = false;
    cl->reordered_mask = 0;
    return PD_OK;
}

int pd_celllist_view(pd_cl cl, pd_cl_view_t* out) {
    if (!cl || !out) return PD_EINVAL;
    memset(out, 0, sizeof(*out));
    out->cell_start = cl->cell_start.as<int>();
    out->sorted_ids = cl->sorted.as<int>();
    out->dom_sort_ids = cl->dom_sort.as<int>();
    out->ncells = cl->ncells;
    for (int d = 0; d < 3; ++d) {
        out->gs[d] = cl->gs[d];
        out->div[d] = cl->div[d];
        out->box_lo[d] = cl->box_lo[d];
        out->spacing[d] = cl->spacing[d];
    }
    out->pad = cl->pad;
    out->nn_box = cl->nn_box;
    out->ghost_marker = cl->ghost_marker;
    out->n_part = cl->n_part;
    return PD_OK;
}

int pd_celllist_get(pd_cl cl, int* cell_start, int* sorted_ids, void* stream) {
    if (!cl) return PD_EINVAL;
    cudaStream_t st = S(stream);
    if (cell_start && cl->cell_start.p)
        PD_CUDA(cudaMemcpyAsync(cell_start, cl->cell_start.p, sizeof(int) * (cl->ncells + 1), cudaMemcpyDeviceToHost, st));
    if (sorted_ids && cl->n_part > 0)
        PD_CUDA(cudaMemcpyAsync(sorted_ids, cl->sorted.p, sizeof(int) * cl->n_part, cudaMemcpyDeviceToHost, st));
    PD_CUDA(cudaStreamSynchronize(st));
    return PD_OK;
}

int pd_test_force(pd_vd h, pd_cl cl, int in_prop, int out_prop, int sorted, void* stream) {
    if (!h || !cl || in_prop < 0 || out_prop < 0 || in_prop >= (int)h->props.size() ||
        out_prop >= (int)h->props.size())
        return PD_EINVAL;
    Prop& A = h->props[in_prop];
    Prop& B = h->props[out_prop];
    int want = h->dtype;
    if (A.type != want || B.type != want || A.ncomp < 1 || B.ncomp < 3) {
        set_error("pd_test_force: in_prop scalar and out_prop 3-vector in the vector's dtype");
        return PD_EINVAL;
    }
    if (sorted && !cl->reordered) {
        set_error("pd_test_force: sorted variant needs a reordered vector");
        return PD_ESTATE;
    }
    cudaStream_t st = S(stream);
    long gm = h->n_real;
    if (gm == 0) return PD_OK;
    unsigned g = grid_for(gm, 128);
    if (h->dtype == PD_F64) {
        double* o = (double*)B.d;
        pd::launch(k_test_force<double>, g, 128, 0, st, (const double4*)h->pos, gm, make_grid<double>(cl), cl->nn_box,
                                                cl->cell_start.as<unsigned int>(), cl->sorted.as<int>(),
                                                cl->dom_sort.as<int>(), sorted, (const double*)A.d, o, o + h->cap,
                                                o + 2 * h->cap);
    } else {
        float* o = (float*)B.d;
        pd::launch(k_test_force<float>, g, 128, 0, st, (const float4*)h->pos, gm, make_grid<float>(cl), cl->nn_box,
                                               cl->cell_start.as<unsigned int>(), cl->sorted.as<int>(),
                                               cl->dom_sort.as<int>(), sorted, (const float*)A.d, o, o + h->cap,
                                               o + 2 * h->cap);
    }
    PD_LAUNCH_CHECK();
    return PD_OK;
}

}  // extern "C"
