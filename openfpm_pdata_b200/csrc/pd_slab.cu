// pd_slab.cu -- slab decomposition of one system over ranks: the device half of
// map and ghost_get between sub-domains (Vector/vector_dist_comm.hpp:1957-2014 and
// :1398-1596; the sub-domains of Decomposition/CartDecomposition.hpp reduced to
// slabs along one axis).
//
// Each rank's vector holds its slab.  An exchange is: label (the rows to send and
// their destination ranks, grouped by rank), pack (rows into a caller-owned
// device buffer), the caller's transport between ranks (an all-to-all), unpack.
// Labelling orders the rows of one destination by ascending slot with one flag /
// scan / fill pass per destination group, so the send order is deterministic.
// A packed row holds the position (three values of the vector's type, padded to
// 8 bytes), then the 8-byte property components, then the 4-byte ones.
#include "pd_device.cuh"
#include "pd_internal.cuh"

namespace pd {

static constexpr int SLAB_MAXC = 48;      // columns of a packed row
static constexpr int SLAB_MAXP = 1024;    // slabs (ranks)

// destination rank of every real particle; positions wrapped in place (the split
// axis by the global box when periodic, the other axes by the vector's box)
template <class T>
__global__ void k_slab_owner(typename V4<T>::type* __restrict__ pos, long n, int axis, int per_axis, double glo,
                             double ghi, double w, int P, T lo0, T lo1, T lo2, T hi0, T hi1, T hi2, int per0,
                             int per1, int per2, int* __restrict__ dest) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        typename V4<T>::type r = ld4(pos, i);
        T* c = &r.x;
        const T lo[3] = {lo0, lo1, lo2}, hi[3] = {hi0, hi1, hi2};
        const int per[3] = {per0, per1, per2};
        for (int d = 0; d < 3; ++d) {
            if (d == axis) {
                if (per_axis) c[d] = periodic_l(c[d], (T)ghi, (T)glo);
            } else if (per[d]) {
                c[d] = periodic_l(c[d], hi[d], lo[d]);
            }
        }
        st4(pos, i, r);
        double q = floor(((double)c[axis] - glo) / w);
        int k = (q > 0.0) ? (q < (double)(P - 1) ? (int)q : P - 1) : 0;
        dest[i] = k;
    }
}

__global__ void k_slab_eq(const int* __restrict__ dest, long n, int d, unsigned int* __restrict__ flag) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        flag[i] = dest[i] == d ? 1u : 0u;
}

// halo flags: the slab coordinate below lo_thr (side 0) / at or above hi_thr (side 1)
template <class T>
__global__ void k_slab_side(const typename V4<T>::type* __restrict__ pos, long n, int axis, int side, double thr,
                            unsigned int* __restrict__ flag) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const typename V4<T>::type r = ld4(pos, i);
        const double a = (double)(axis == 0 ? r.x : (axis == 1 ? r.y : r.z));
        flag[i] = (side == 0 ? a < thr : a >= thr) ? 1u : 0u;
    }
}

// rows of group g: slot i at base_g + off[i] where flag[i]; base_g = sum of the
// earlier groups' totals
__global__ void k_slab_fill(const unsigned int* __restrict__ flag, const unsigned int* __restrict__ off, long n,
                            const unsigned int* __restrict__ tot, int g, unsigned char shift,
                            int* __restrict__ idx, unsigned char* __restrict__ shf) {
    __shared__ unsigned long long base;
    if (threadIdx.x == 0) {
        unsigned long long b = 0;
        for (int e = 0; e < g; ++e) b += tot[e];
        base = b;
    }
    __syncthreads();
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        if (flag[i]) {
            const unsigned long long k = base + off[i];
            idx[k] = (int)i;
            if (shf) shf[k] = shift;
        }
}

// column table of a packed row
struct SlabCols {
    int nc;
    int row_bytes;
    int axis_col;  // the column of the split-axis coordinate (shifted in halo rows)
    unsigned char* base[SLAB_MAXC];
    long stride[SLAB_MAXC];  // bytes between particles in the vector
    int esize[SLAB_MAXC];
    int off[SLAB_MAXC];  // byte offset in the row
};

__device__ __forceinline__ void copy_elem(void* d, const void* s, int esize) {
    if (esize == 8) *(unsigned long long*)d = *(const unsigned long long*)s;
    else *(unsigned int*)d = *(const unsigned int*)s;
}

template <class T>
__global__ void k_slab_pack(SlabCols C, long rows, const int* __restrict__ idx, const unsigned char* __restrict__ shf,
                            T L, unsigned char* __restrict__ out) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < rows; k += (long)gridDim.x * blockDim.x) {
        const long i = idx[k];
        unsigned char* row = out + k * (long)C.row_bytes;
        for (int c = 0; c < C.nc; ++c) {
            const unsigned char* src = C.base[c] + i * C.stride[c];
            if (c == C.axis_col && shf && shf[k]) {
                T v = *(const T*)src;
                v = shf[k] == 1 ? v + L : v - L;
                *(T*)(row + C.off[c]) = v;
            } else {
                copy_elem(row + C.off[c], src, C.esize[c]);
            }
        }
    }
}

template <class T>
__global__ void k_slab_unpack(SlabCols C, long rows, long first, const unsigned char* __restrict__ in,
                              int* __restrict__ gid, int ids) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < rows; k += (long)gridDim.x * blockDim.x) {
        const long i = first + k;
        const unsigned char* row = in + k * (long)C.row_bytes;
        for (int c = 0; c < C.nc; ++c) copy_elem(C.base[c] + i * C.stride[c], row + C.off[c], C.esize[c]);
        *(T*)(C.base[0] + i * C.stride[0] + 3 * sizeof(T)) = T(0);  // the record's unused fourth value
        gid[i] = ids ? (int)k : -1;
    }
}

// columns of the vector for the properties in mask: positions (x, y, z), then the
// 8-byte property components, then the 4-byte ones
static int slab_cols(pd_vd h, unsigned long mask, SlabCols& C) {
    memset(&C, 0, sizeof(C));
    const int es = h->dtype == PD_F64 ? 8 : 4;
    int off = 0, nc = 0;
    for (int k = 0; k < 3; ++k) {
        C.base[nc] = (unsigned char*)h->pos + k * es;
        C.stride[nc] = h->pos_bytes;
        C.esize[nc] = es;
        C.off[nc] = off;
        off += es;
        ++nc;
    }
    off = (off + 7) & ~7;
    for (int pass = 0; pass < 2; ++pass) {
        const int want = pass == 0 ? 8 : 4;
        for (size_t p = 0; p < h->props.size(); ++p) {
            if (!((mask >> p) & 1ul)) continue;
            const Prop& P = h->props[p];
            if (P.esize != want) continue;
            for (int c = 0; c < P.ncomp; ++c) {
                if (nc == SLAB_MAXC) {
                    set_error("slab: more than %d columns in a row", SLAB_MAXC);
                    return PD_EINVAL;
                }
                C.base[nc] = (unsigned char*)P.d + (size_t)c * h->cap * P.esize;
                C.stride[nc] = P.esize;
                C.esize[nc] = P.esize;
                C.off[nc] = off;
                off += P.esize;
                ++nc;
            }
        }
    }
    C.nc = nc;
    C.row_bytes = (off + 7) & ~7;
    C.axis_col = h->slab_axis;
    return PD_OK;
}

static int slab_check(pd_vd h, const pd_slab_t* s) {
    if (!h || !s || s->axis < 0 || s->axis > 2 || s->nslabs < 1 || s->nslabs > SLAB_MAXP || !(s->hi > s->lo) ||
        !(s->ghost >= 0)) {
        set_error("slab: invalid decomposition");
        return PD_EINVAL;
    }
    if (s->nslabs > 1 && s->ghost > (s->hi - s->lo) / s->nslabs) {
        set_error("slab: the ghost %.6g is wider than a slab", s->ghost);
        return PD_EINVAL;
    }
    return PD_OK;
}

// groups (flag sets over n slots) in send order -> h->slab_idx / slab_shift, totals on the host
struct SlabGroup {
    int dest;
    unsigned char shift;
};

static int slab_scratch(pd_vd h, long n, long groups) {
    PD_TRY(h->slab_flag.ensure(sizeof(unsigned int) * (size_t)(n > 0 ? n : 1)));
    PD_TRY(h->slab_off.ensure(sizeof(unsigned int) * (size_t)(n > 0 ? n : 1)));
    PD_TRY(h->slab_tot.ensure(sizeof(unsigned int) * (size_t)(groups > 0 ? groups : 1)));
    PD_TRY(h->slab_idx.ensure(sizeof(int) * (size_t)(2 * n > 0 ? 2 * n : 1)));
    PD_TRY(h->slab_shift.ensure((size_t)(2 * n > 0 ? 2 * n : 1)));
    return PD_OK;
}

}  // namespace pd

using namespace pd;

extern "C" {

int pd_slab_map_label(pd_vd h, const pd_slab_t* s, long* send_counts, void* stream) {
    PD_TRY(slab_check(h, s));
    if (!send_counts) return PD_EINVAL;
    cudaStream_t st = S(stream);
    const long n = h->n_real;
    const int P = s->nslabs;
    for (int d = 0; d < P; ++d) send_counts[d] = 0;
    h->n_total = h->n_real;  // the ghost is dropped (vector_dist_comm.hpp:1969-1970)
    h->img_valid = false;
    h->slab_kind = 1;
    h->slab_rows = 0;
    h->slab_axis = s->axis;
    h->epoch++;
    if (n == 0) return PD_OK;
    PD_TRY(slab_scratch(h, n, P));
    PD_TRY(h->tmp2.ensure(sizeof(int) * (size_t)n));
    int* dest = h->tmp2.as<int>();
    const unsigned g = grid_for(n, 256);
    const double w = (s->hi - s->lo) / P;
    const int pa = s->periodic ? 1 : 0;
    const int p0 = h->bc[0] == PD_PERIODIC, p1 = h->bc[1] == PD_PERIODIC, p2 = h->bc[2] == PD_PERIODIC;
    if (h->dtype == PD_F64)
        pd::launch(k_slab_owner<double>, g, 256, 0, st, (double4*)h->pos, n, s->axis, pa, s->lo, s->hi, w, P, h->lo[0],
                   h->lo[1], h->lo[2], h->hi[0], h->hi[1], h->hi[2], p0, p1, p2, dest);
    else
        pd::launch(k_slab_owner<float>, g, 256, 0, st, (float4*)h->pos, n, s->axis, pa, s->lo, s->hi, w, P,
                   (float)h->lo[0], (float)h->lo[1], (float)h->lo[2], (float)h->hi[0], (float)h->hi[1],
                   (float)h->hi[2], p0, p1, p2, dest);
    PD_LAUNCH_CHECK();
    unsigned int* flag = h->slab_flag.as<unsigned int>();
    unsigned int* off = h->slab_off.as<unsigned int>();
    unsigned int* tot = h->slab_tot.as<unsigned int>();
    for (int d = 0; d < P; ++d) {
        pd::launch(k_slab_eq, g, 256, 0, st, (const int*)dest, n, d, flag);
        PD_TRY(scan_u32(flag, off, n, tot + d, h->scan_scratch, st));
        pd::launch(k_slab_fill, g, 256, 0, st, (const unsigned int*)flag, (const unsigned int*)off, n,
                   (const unsigned int*)tot, d, (unsigned char)0, h->slab_idx.as<int>(), (unsigned char*)nullptr);
        PD_LAUNCH_CHECK();
    }
    std::vector<unsigned int> t(P);
    PD_CUDA(cudaMemcpyAsync(t.data(), tot, sizeof(unsigned int) * P, cudaMemcpyDeviceToHost, st));
    PD_CUDA(cudaStreamSynchronize(st));
    long rows = 0;
    for (int d = 0; d < P; ++d) {
        send_counts[d] = t[d];
        rows += t[d];
    }
    h->slab_rows = rows;
    return PD_OK;
}

int pd_slab_halo_label(pd_vd h, const pd_slab_t* s, int rank, long* send_counts, void* stream) {
    PD_TRY(slab_check(h, s));
    const int P = s->nslabs;
    if (!send_counts || rank < 0 || rank >= P) return PD_EINVAL;
    for (int d = 0; d < P; ++d) send_counts[d] = 0;
    cudaStream_t st = S(stream);
    // local particles and periodic images: not a halo received before
    const long n = (h->halo_epoch == h->epoch) ? h->halo_base : h->n_total;
    h->slab_kind = 2;
    h->slab_rows = 0;
    h->slab_axis = s->axis;
    h->slab_L = s->hi - s->lo;
    if (P == 1 || n == 0) return PD_OK;
    const double w = (s->hi - s->lo) / P;
    const double e0 = s->lo + w * rank, e1 = (rank == P - 1) ? s->hi : s->lo + w * (rank + 1);
    // the two sides in order of their destination ranks (lower side first on a tie)
    struct Side {
        int dest;
        unsigned char shift;  // 0 none, 1 +L, 2 -L
        double thr;
        int side;
    };
    std::vector<Side> sides;
    if (rank > 0) sides.push_back({rank - 1, 0, e0 + s->ghost, 0});
    else if (s->periodic) sides.push_back({P - 1, 1, e0 + s->ghost, 0});
    if (rank < P - 1) sides.push_back({rank + 1, 0, e1 - s->ghost, 1});
    else if (s->periodic) sides.push_back({0, 2, e1 - s->ghost, 1});
    if (sides.size() == 2 && sides[1].dest < sides[0].dest) std::swap(sides[0], sides[1]);
    PD_TRY(slab_scratch(h, n, 2));
    unsigned int* flag = h->slab_flag.as<unsigned int>();
    unsigned int* off = h->slab_off.as<unsigned int>();
    unsigned int* tot = h->slab_tot.as<unsigned int>();
    const unsigned g = grid_for(n, 256);
    for (size_t k = 0; k < sides.size(); ++k) {
        if (h->dtype == PD_F64)
            pd::launch(k_slab_side<double>, g, 256, 0, st, (const double4*)h->pos, n, s->axis, sides[k].side,
                       sides[k].thr, flag);
        else
            pd::launch(k_slab_side<float>, g, 256, 0, st, (const float4*)h->pos, n, s->axis, sides[k].side,
                       sides[k].thr, flag);
        PD_TRY(scan_u32(flag, off, n, tot + k, h->scan_scratch, st));
        pd::launch(k_slab_fill, g, 256, 0, st, (const unsigned int*)flag, (const unsigned int*)off, n,
                   (const unsigned int*)tot, (int)k, sides[k].shift, h->slab_idx.as<int>(),
                   h->slab_shift.as<unsigned char>());
        PD_LAUNCH_CHECK();
    }
    unsigned int t[2] = {0, 0};
    PD_CUDA(cudaMemcpyAsync(t, tot, sizeof(unsigned int) * sides.size(), cudaMemcpyDeviceToHost, st));
    PD_CUDA(cudaStreamSynchronize(st));
    long rows = 0;
    for (size_t k = 0; k < sides.size(); ++k) {
        send_counts[sides[k].dest] += t[k];
        rows += t[k];
    }
    h->slab_rows = rows;
    return PD_OK;
}

int pd_slab_row_bytes(pd_vd h, unsigned long prop_mask, long* bytes) {
    if (!h || !bytes) return PD_EINVAL;
    SlabCols C;
    PD_TRY(slab_cols(h, prop_mask, C));
    *bytes = C.row_bytes;
    return PD_OK;
}

int pd_slab_pack(pd_vd h, unsigned long prop_mask, void* send, long cap_rows, void* stream) {
    if (!h || cap_rows < 0) return PD_EINVAL;
    if (h->slab_kind == 0) {
        set_error("slab_pack: no labelling to pack (call pd_slab_map_label or pd_slab_halo_label)");
        return PD_ESTATE;
    }
    if (h->slab_rows > cap_rows) {
        set_error("slab_pack: %ld rows, room for %ld", h->slab_rows, cap_rows);
        return PD_EOVERFLOW;
    }
    if (h->slab_rows == 0) return PD_OK;
    PD_TRY(check_device_ptr(send, "pd_slab_pack", "the send buffer"));
    SlabCols C;
    PD_TRY(slab_cols(h, prop_mask, C));
    cudaStream_t st = S(stream);
    const unsigned char* shf = h->slab_kind == 2 ? h->slab_shift.as<unsigned char>() : nullptr;
    const unsigned g = grid_for(h->slab_rows, 256);
    if (h->dtype == PD_F64)
        pd::launch(k_slab_pack<double>, g, 256, 0, st, C, h->slab_rows, (const int*)h->slab_idx.as<int>(), shf,
                   h->slab_L, (unsigned char*)send);
    else
        pd::launch(k_slab_pack<float>, g, 256, 0, st, C, h->slab_rows, (const int*)h->slab_idx.as<int>(), shf,
                   (float)h->slab_L, (unsigned char*)send);
    PD_LAUNCH_CHECK();
    return PD_OK;
}

int pd_slab_map_unpack(pd_vd h, unsigned long prop_mask, const void* recv, long n_recv, void* stream) {
    if (!h || n_recv < 0 || (n_recv > 0 && !recv) || n_recv >= (1L << 31)) return PD_EINVAL;
    if (n_recv > 0) PD_TRY(check_device_ptr(recv, "pd_slab_map_unpack", "the receive buffer"));
    cudaStream_t st = S(stream);
    PD_TRY(ensure_capacity(h, n_recv + 1, st));
    for (size_t p = 0; p < h->props.size(); ++p)
        if (!((prop_mask >> p) & 1ul) && n_recv > 0)
            for (int c = 0; c < h->props[p].ncomp; ++c)
                PD_CUDA(cudaMemsetAsync(h->props[p].d + (size_t)c * h->cap * h->props[p].esize, 0,
                                        (size_t)n_recv * h->props[p].esize, st));
    if (n_recv > 0) {
        SlabCols C;
        PD_TRY(slab_cols(h, prop_mask, C));
        const unsigned g = grid_for(n_recv, 256);
        if (h->dtype == PD_F64)
            pd::launch(k_slab_unpack<double>, g, 256, 0, st, C, n_recv, 0L, (const unsigned char*)recv, h->gid, 1);
        else
            pd::launch(k_slab_unpack<float>, g, 256, 0, st, C, n_recv, 0L, (const unsigned char*)recv, h->gid, 1);
        PD_LAUNCH_CHECK();
    }
    h->n_real = h->n_total = n_recv;
    h->n_img = 0;
    h->img_valid = false;
    h->slab_kind = 0;
    h->epoch++;
    return PD_OK;
}

int pd_slab_halo_unpack(pd_vd h, unsigned long prop_mask, const void* recv, long n_recv, void* stream) {
    if (!h || n_recv < 0 || (n_recv > 0 && !recv) || n_recv >= (1L << 31)) return PD_EINVAL;
    if (n_recv > 0) PD_TRY(check_device_ptr(recv, "pd_slab_halo_unpack", "the receive buffer"));
    cudaStream_t st = S(stream);
    const long base = (h->halo_epoch == h->epoch) ? h->halo_base : h->n_total;
    PD_TRY(ensure_capacity(h, base + n_recv + 1, st));
    if (n_recv > 0) {
        SlabCols C;
        PD_TRY(slab_cols(h, prop_mask, C));
        const unsigned g = grid_for(n_recv, 256);
        if (h->dtype == PD_F64)
            pd::launch(k_slab_unpack<double>, g, 256, 0, st, C, n_recv, base, (const unsigned char*)recv, h->gid, 0);
        else
            pd::launch(k_slab_unpack<float>, g, 256, 0, st, C, n_recv, base, (const unsigned char*)recv, h->gid, 0);
        PD_LAUNCH_CHECK();
    }
    h->n_total = base + n_recv;
    h->slab_kind = 0;
    h->epoch++;
    h->halo_base = base;
    h->halo_epoch = h->epoch;
    return PD_OK;
}

}  // extern "C"
