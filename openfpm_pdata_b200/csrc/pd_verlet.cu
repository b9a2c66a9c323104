// pd_verlet.cu -- full Verlet list on the GPU (getVerlet / updateVerlet).
//
// The reference builds this list on the CPU only (vector_dist.hpp:1514-1620):
// for every domain particle, all particles (domain + ghost, self included) with
// d2 < r_cut^2, found through a cell list of side r_cut over the domain
// enlarged by the ghost magnified 1.013.  Here:
//   1. the cell list is built by the counting sort of pd_celllist.cu;
//   2. positions are gathered into cell order with the original index in the
//      record's 4th word (pos_cs);
//   3. one CTA per tile of TX cells along x stages the 9 neighbour rows
//      (x-1 .. x+TX for dy, dz in {-1,0,1}; each a contiguous range of pos_cs)
//      in shared memory and every thread scans the 27-cell neighbourhood of its
//      particles from there, in the reference walk order (dz, dy, dx, in-cell
//      order), writing column-major rows nbr[k*stride + i].
// Rows longer than the capacity set ERR_NN_OVERFLOW and record the longest row;
// the host grows the capacity and rebuilds.
//
// Symmetric (half) list, getVerletSym (vector_dist.hpp:1412-1416): each
// interacting pair once.  A domain partner q is kept by p iff q > p; a periodic
// image is kept iff it lies after p in the lexicographic (x, y, z) order.  The
// mirror of a pair (p, image of r) is (r, image of p), shifted by the opposite
// vector, so exactly one of the two is kept; forces or counts accumulated on an
// image are folded onto its source by ghost_put<add_> (vector_dist.hpp:2304).
// The criterion is geometric, not cell-based, so it does not depend on the box
// being a whole number of cells.
#include "pd_device.cuh"
#include "pd_internal.cuh"

namespace pd {

template <class T> struct IdxBits;
template <> struct IdxBits<double> {
    __device__ static double enc(int i) { return __longlong_as_double((long long)i); }
    __device__ static int dec(double w) { return (int)__double_as_longlong(w); }
};
template <> struct IdxBits<float> {
    __device__ static float enc(int i) { return __int_as_float(i); }
    __device__ static int dec(float w) { return __float_as_int(w); }
};

// pos_cs[k] = (pos[sorted[k]].xyz, bits(sorted[k]))
template <class T>
__global__ void k_gather_cs(const typename V4<T>::type* __restrict__ pos, const int* __restrict__ sorted,
                            const unsigned int* __restrict__ cs_end, typename V4<T>::type* __restrict__ out,
                            long n_bound) {
    long n = (long)*cs_end;
    if (n > n_bound) n = n_bound;
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        int i = sorted[k];
        typename V4<T>::type r = ld4(pos, i);
        r.w = IdxBits<T>::enc(i);
        st4(out, k, r);
    }
}

template <class T4> __device__ __forceinline__ bool lex_after(const T4& a, const T4& b) {
    return a.x > b.x || (a.x == b.x && (a.y > b.y || (a.y == b.y && a.z > b.z)));
}

template <class T>
__global__ void __launch_bounds__(128) k_verlet_tile(const typename V4<T>::type* __restrict__ pcs, Grid<T> G, int TX,
                                                     int ntx, const unsigned int* __restrict__ cs, long n_dom, T r2,
                                                     int* __restrict__ nbr, int* __restrict__ nn, long stride,
                                                     int max_nn, int smem_cap, int sym,
                                                     unsigned int* __restrict__ ctrl_err,
                                                     unsigned int* __restrict__ ctrl_nnmax) {
    typedef typename V4<T>::type T4;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T4* sp = reinterpret_cast<T4*>(smem_raw);
    __shared__ unsigned int row_beg[9], row_off[9];
    __shared__ unsigned int cs_sm[9][40];
    __shared__ int use_smem;

    const int gx = G.gs[0];
    const int ny = G.gs[1] - 2 * G.pad, nz = G.gs[2] - 2 * G.pad;
    long t = blockIdx.x;
    int tx = (int)(t % ntx);
    long rest = t / ntx;
    int y = (int)(rest % ny) + G.pad;
    int z = (int)(rest / ny) + G.pad;
    int x0 = G.pad + tx * TX;
    int x1 = min(x0 + TX, gx - G.pad);  // exclusive
    int ncol = x1 - x0 + 3;             // cells x0-1 .. x1 (x1 inclusive) + end marker

    for (int e = threadIdx.x; e < 9 * ncol; e += blockDim.x) {
        int r = e / ncol, j = e % ncol;
        int dz = r / 3 - 1, dy = r % 3 - 1;
        long c = (long)(x0 - 1 + j) + (long)gx * ((y + dy) + (long)G.gs[1] * (z + dz));
        cs_sm[r][j] = cs[c];  // j == ncol-1 reads the start of cell x1+1 = end of cell x1
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int off = 0;
        for (int r = 0; r < 9; ++r) {
            row_beg[r] = cs_sm[r][0];
            row_off[r] = off;
            off += cs_sm[r][ncol - 1] - cs_sm[r][0];
        }
        use_smem = (int)(off <= (unsigned int)smem_cap);
    }
    __syncthreads();
    const bool sm = use_smem != 0;
    if (sm) {
        for (int r = 0; r < 9; ++r) {
            unsigned int b = row_beg[r], len = cs_sm[r][ncol - 1] - b, o = row_off[r];
            for (unsigned int k = threadIdx.x; k < len; k += blockDim.x) sp[o + k] = pcs[b + k];
        }
    }
    __syncthreads();

    // domain particles of the centre row cells x0 .. x1-1 (row index 4: dy = dz = 0)
    unsigned int ib = cs_sm[4][1], ie = cs_sm[4][ncol - 2];
    for (unsigned int k = ib + threadIdx.x; k < ie; k += blockDim.x) {
        T4 xi = pcs[k];
        int i = IdxBits<T>::dec(xi.w);
        if (i >= n_dom) continue;
        // column of k's cell inside the tile: find j with cs_sm[4][j] <= k < cs_sm[4][j+1]
        int j = 1;
        while (j < ncol - 2 && cs_sm[4][j + 1] <= k) ++j;
        int cnt = 0;
#pragma unroll 1
        for (int r = 0; r < 9; ++r) {
            unsigned int a = cs_sm[r][j - 1], e = cs_sm[r][j + 2];
            const T4* base = sm ? (sp + row_off[r] - row_beg[r]) : pcs;
#pragma unroll 4
            for (unsigned int q = a; q < e; ++q) {
                T4 xq = base[q];
                T d2 = dist2(xi.x - xq.x, xi.y - xq.y, xi.z - xq.z);
                if (d2 < r2) {
                    const int qi = IdxBits<T>::dec(xq.w);
                    if (sym && !(qi < n_dom ? qi > i : lex_after(xq, xi))) continue;
                    if (cnt < max_nn) nbr[(long)cnt * stride + i] = qi;
                    cnt++;
                }
            }
        }
        if (cnt > max_nn) {
            atomicOr(ctrl_err, ERR_NN_OVERFLOW);
            atomicMax(ctrl_nnmax, (unsigned int)cnt);
            cnt = max_nn;
        }
        nn[i] = cnt;
    }
}

static int choose_tx(pd_cl cl, long n_all, int& TX) {
    double cells = (double)cl->div[0] * cl->div[1] * cl->div[2];
    double occ = cells > 0 ? (double)n_all / cells : 1.0;
    int tx = (int)(96.0 / (occ > 1e-3 ? occ : 1e-3));
    int nxi = cl->gs[0] - 2 * cl->pad;
    if (tx < 1) tx = 1;
    if (tx > 32) tx = 32;
    if (tx > nxi) tx = nxi;
    TX = tx;
    return PD_OK;
}

// Build the list of domain particles [0, n_dom) over all particles; the
// particle count is h->n_real + *n_img_dev when n_img_dev is given (device
// resident), else h->n_total.
int verlet_build(pd_vd h, pd_vl vl, long n_dom, const unsigned int* n_img_dev, cudaStream_t st, bool check) {
    pd_cl cl = vl->cl;
    long n_all_bound = n_img_dev ? h->cap : h->n_total;
    PD_TRY(cl_build(h, cl, n_all_bound, n_img_dev, st));
    // cell-ordered positions with original indices
    PD_TRY(h->tmp.ensure((size_t)(n_all_bound > 0 ? n_all_bound : 1) * h->pos_bytes));
    const unsigned int* cs_end = cl->cell_start.as<unsigned int>() + cl->ncells;
    unsigned g = grid_for(n_all_bound, 256);
    if (h->dtype == PD_F64)
        pd::launch(k_gather_cs<double>, g, 256, 0, st, (const double4*)h->pos, cl->sorted.as<int>(), cs_end,
                                               h->tmp.as<double4>(), n_all_bound);
    else
        pd::launch(k_gather_cs<float>, g, 256, 0, st, (const float4*)h->pos, cl->sorted.as<int>(), cs_end,
                                              h->tmp.as<float4>(), n_all_bound);
    PD_LAUNCH_CHECK();
    long stride = ((n_dom + 31) / 32) * 32;
    if (stride < 32) stride = 32;
    if (vl->max_nn <= 0) {
        // first build: capacity from the mean density within r (x1.5 + 32), grown on overflow
        double vol = 1.0;
        for (int d = 0; d < 3; ++d) vol *= (h->hi[d] - h->lo[d] + 2 * h->g[d]);
        double dens = (double)(n_img_dev ? h->n_real * 1.3 : h->n_total) / vol;
        double mean = dens * 4.18879 * vl->r_cut * vl->r_cut * vl->r_cut;
        vl->max_nn = (int)(mean * 1.5 + 32);
    }
    for (int attempt = 0; attempt < 3; ++attempt) {
        PD_TRY(vl->nbr.ensure(sizeof(int) * (size_t)stride * vl->max_nn));
        PD_TRY(vl->nn.ensure(sizeof(int) * (n_dom > 0 ? n_dom : 1)));
        vl->stride = stride;
        vl->n_dom = n_dom;
        if (n_dom > 0) {
            int TX;
            choose_tx(cl, h->n_total > 0 ? h->n_total : h->n_real, TX);
            int nxi = cl->gs[0] - 2 * cl->pad;
            int ntx = (nxi + TX - 1) / TX;
            long ntiles = (long)ntx * (cl->gs[1] - 2 * cl->pad) * (cl->gs[2] - 2 * cl->pad);
            int smem_bytes = 64 * 1024;
            int smem_cap = smem_bytes / h->pos_bytes;
            if (h->dtype == PD_F64) {
                static bool attr = false;
                if (!attr) {
                    cudaFuncSetAttribute(k_verlet_tile<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
                    attr = true;
                }
                pd::launch(k_verlet_tile<double>, (unsigned)ntiles, 128, smem_bytes, st, 
                    h->tmp.as<double4>(), [&] {
                        Grid<double> G;
                        for (int d = 0; d < 3; ++d) {
                            G.lo[d] = cl->box_lo[d];
                            G.sp[d] = cl->spacing[d];
                            G.gs[d] = cl->gs[d];
                        }
                        G.pad = cl->pad;
                        return G;
                    }(),
                    TX, ntx, cl->cell_start.as<unsigned int>(), n_dom, (double)(vl->r_cut * vl->r_cut),
                    vl->nbr.as<int>(), vl->nn.as<int>(), stride, vl->max_nn, smem_cap, vl->sym ? 1 : 0,
                    &h->ctrl->err, &h->ctrl->nn_max);
            } else {
                static bool attr = false;
                if (!attr) {
                    cudaFuncSetAttribute(k_verlet_tile<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
                    attr = true;
                }
                float rc = (float)vl->r_cut;
                pd::launch(k_verlet_tile<float>, (unsigned)ntiles, 128, smem_bytes, st, 
                    h->tmp.as<float4>(), [&] {
                        Grid<float> G;
                        for (int d = 0; d < 3; ++d) {
                            G.lo[d] = (float)cl->box_lo[d];
                            G.sp[d] = (float)cl->spacing[d];
                            G.gs[d] = cl->gs[d];
                        }
                        G.pad = cl->pad;
                        return G;
                    }(),
                    TX, ntx, cl->cell_start.as<unsigned int>(), n_dom, rc * rc, vl->nbr.as<int>(), vl->nn.as<int>(),
                    stride, vl->max_nn, smem_cap, vl->sym ? 1 : 0, &h->ctrl->err, &h->ctrl->nn_max);
            }
            PD_LAUNCH_CHECK();
        }
        if (!check) return PD_OK;
        PD_TRY(read_ctrl(h, st));
        if (!(h->ctrl_h->err & ERR_NN_OVERFLOW)) break;
        // grow and rebuild
        vl->max_nn = (int)(h->ctrl_h->nn_max * 1.15 + 8);
        h->ctrl_h->err &= ~ERR_NN_OVERFLOW;
        h->ctrl_h->nn_max = 0;
        PD_CUDA(cudaMemcpyAsync(&h->ctrl->err, &h->ctrl_h->err, sizeof(unsigned int) * 3, cudaMemcpyHostToDevice, st));
    }
    vl->epoch = h->epoch;
    return PD_OK;
}

}  // namespace pd

using namespace pd;

extern "C" {

int pd_verlet_create(pd_vd h, double r_cut, pd_vl* out) {
    if (!h || !out || !(r_cut > 0)) return PD_EINVAL;
    pd_vl vl = new pd_vl_s();
    vl->owner = h;
    vl->r_cut = r_cut;
    vl->cl = new pd_cl_s();
    int r = cl_geometry(vl->cl, h, r_cut, 1.013, 1);
    if (r != PD_OK) {
        delete vl->cl;
        delete vl;
        return r;
    }
    *out = vl;
    return PD_OK;
}

int pd_verlet_create_sym(pd_vd h, double r_cut, pd_vl* out) {
    int r = pd_verlet_create(h, r_cut, out);
    if (r == PD_OK) (*out)->sym = true;
    return r;
}

int pd_verlet_destroy(pd_vl vl) {
    if (!vl) return PD_EINVAL;
    if (vl->cl) pd_celllist_destroy(vl->cl);
    vl->nbr.release();
    vl->nn.release();
    delete vl;
    return PD_OK;
}

int pd_verlet_update(pd_vd h, pd_vl vl, void* stream) {
    if (!h || !vl || vl->owner != h) return PD_EINVAL;
    return verlet_build(h, vl, h->n_real, nullptr, S(stream), true);
}

int pd_verlet_get(pd_vl vl, int* counts, int* idx, long idx_cap, void* stream) {
    if (!vl || !counts) return PD_EINVAL;
    cudaStream_t st = S(stream);
    long n = vl->n_dom;
    if (n == 0) return PD_OK;
    PD_CUDA(cudaMemcpyAsync(counts, vl->nn.p, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
    PD_CUDA(cudaStreamSynchronize(st));
    if (!idx) return PD_OK;
    long tot = 0;
    int mx = 0;
    for (long i = 0; i < n; ++i) {
        tot += counts[i];
        mx = std::max(mx, counts[i]);
    }
    if (tot > idx_cap) {
        set_error("pd_verlet_get: idx_cap %ld < %ld entries", idx_cap, tot);
        return PD_EINVAL;
    }
    std::vector<int> col((size_t)vl->stride * mx);
    if (mx > 0)
        PD_CUDA(cudaMemcpy(col.data(), vl->nbr.p, sizeof(int) * (size_t)vl->stride * mx, cudaMemcpyDeviceToHost));
    long o = 0;
    for (long i = 0; i < n; ++i)
        for (int k = 0; k < counts[i]; ++k) idx[o++] = col[(size_t)k * vl->stride + i];
    return PD_OK;
}

}  // extern "C"
