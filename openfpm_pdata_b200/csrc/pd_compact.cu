// Stream compaction of the domain particles: remove_marked and get_indexes_by_type
// (Vector/cuda/vector_dist_cuda_funcs.cuh:313-481).
//
// remove_marked<prp>: the mark property is flipped in place (x -> x == 0, the
// reference's destructive step, flip_one_to_zero :313-321) while each tile counts
// its kept particles, the tile counts are scanned, and every kept particle (mark
// 0 before the flip) is scattered, in order, with its position, global id and all
// properties (copy_new_to_old_by_scan :295-311), its rank within the tile from
// warp ballots.  The ghosts are dropped: the vector then holds the kept particles
// only (setGhostMarker(kept), :406).  When nothing is marked the vector keeps its
// particles and the flipped mark (:366-372).
//
// The scatter writes all columns of one particle in one thread (a column table
// passed by value) straight into new storage of the same capacity, which replaces
// the old; the vector's epoch moves on, so views taken before are stale.
//
// get_indexes_by_type<prp, functor>: flag p < end whose property satisfies the
// comparison (mark_indexes :414-423), scan, and write p at its scan offset
// (fill_indexes :425-438): the indexes come out ascending.
#include <mutex>

#include "pd_device.cuh"
#include "pd_internal.cuh"

namespace pd {

static constexpr int CMAXC = 24;  // columns per scatter launch

struct ColSet {
    int nc;
    const unsigned char* src[CMAXC];
    unsigned char* dst[CMAXC];
    int wsize[CMAXC];  // bytes per element: 4, 8, 16 or 32
};

// compaction tiles: CT_BLOCK threads, CT_ITEMS passes of CT_BLOCK consecutive particles
static constexpr int CT_BLOCK = 512;
static constexpr int CT_ITEMS = 8;
static constexpr long CT_TILE = (long)CT_BLOCK * CT_ITEMS;

// the mark flipped in place (x -> x == 0), a keep byte per particle and the
// tile's count of kept particles
template <class E>
__global__ void __launch_bounds__(CT_BLOCK) k_flip_mark(E* __restrict__ m, long n, unsigned char* __restrict__ keep,
                                                        unsigned int* __restrict__ part) {
    const long base = (long)blockIdx.x * CT_TILE;
    unsigned int cnt = 0;
    for (int k = 0; k < CT_ITEMS; ++k) {
        const long i = base + (long)k * CT_BLOCK + threadIdx.x;
        if (i < n) {
            const bool kp = (m[i] == E(0));
            m[i] = kp ? E(1) : E(0);
            keep[i] = kp ? 1 : 0;
            cnt += kp ? 1u : 0u;
        }
    }
    cnt = block_sum<unsigned int, CT_BLOCK>(cnt);
    if (threadIdx.x == 0) part[blockIdx.x] = cnt;
}

// every kept particle of the tile to its slot: the tile's base from the scanned
// counts, the rank within the tile from warp ballots (kept particles keep their
// order).  The ballots of all CT_ITEMS passes are taken first and their counts
// scanned once over (pass, warp), so the tile needs two barriers, not three a pass.
__global__ void __launch_bounds__(CT_BLOCK) k_compact_scatter(ColSet C, long n, const unsigned char* __restrict__ keep,
                                                              const unsigned int* __restrict__ part) {
    constexpr int NW = CT_BLOCK / 32, NC = CT_ITEMS * NW;  // counts in (pass, warp) order
    __shared__ unsigned int cnt[NC];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long base = (long)blockIdx.x * CT_TILE;
    unsigned int bal[CT_ITEMS];
#pragma unroll
    for (int k = 0; k < CT_ITEMS; ++k) {
        const long i = base + (long)k * CT_BLOCK + threadIdx.x;
        bal[k] = __ballot_sync(0xffffffffu, i < n && keep[i]);
        if (lane == 0) cnt[k * NW + w] = __popc(bal[k]);
    }
    __syncthreads();
    // exclusive scan of the NC counts by warp 0 (NC / 32 per lane, then the lanes')
    if (w == 0) {
        constexpr int PER = NC / 32;
        unsigned int v[PER], s = 0;
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            v[j] = cnt[lane * PER + j];
            s += v[j];
        }
        unsigned int incl = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        unsigned int run = part[blockIdx.x] + incl - s;
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            cnt[lane * PER + j] = run;
            run += v[j];
        }
    }
    __syncthreads();
    unsigned int d[CT_ITEMS];  // (n < 2^32)
    unsigned int kept = 0;
#pragma unroll
    for (int k = 0; k < CT_ITEMS; ++k) {
        kept |= (bal[k] >> lane & 1u) << k;
        d[k] = cnt[k * NW + w] + __popc(bal[k] & ((1u << lane) - 1u));
    }
    // one particle at a time, column by column: at 32 registers four CTAs of 512 fit
    // an SM, which keeps more loads in flight than fewer threads holding several each
    for (int k = 0; k < CT_ITEMS; ++k) {
        if (!(kept >> k & 1u)) continue;
        const long i = base + (long)k * CT_BLOCK + threadIdx.x;
        for (int c = 0; c < C.nc; ++c) {
            switch (C.wsize[c]) {
                case 4: ((unsigned int*)C.dst[c])[d[k]] = ((const unsigned int*)C.src[c])[i]; break;
                case 8: ((unsigned long long*)C.dst[c])[d[k]] = ((const unsigned long long*)C.src[c])[i]; break;
                case 16: ((uint4*)C.dst[c])[d[k]] = ((const uint4*)C.src[c])[i]; break;
                default: {
                    const uint4* s4 = (const uint4*)C.src[c] + 2 * i;
                    uint4* t4 = (uint4*)C.dst[c] + 2 * (long)d[k];
                    t4[0] = s4[0];
                    t4[1] = s4[1];
                }
            }
        }
    }
}

template <class E>
__device__ __forceinline__ bool cmp_ok(E v, E ref, int cmp) {
    switch (cmp) {
        case PD_CMP_EQ: return v == ref;
        case PD_CMP_NE: return v != ref;
        case PD_CMP_LT: return v < ref;
        case PD_CMP_LE: return v <= ref;
        case PD_CMP_GT: return v > ref;
        default: return v >= ref;
    }
}

template <class E>
__global__ void k_mark_indexes(const E* __restrict__ a, long n, E ref, int cmp, unsigned int* __restrict__ flag) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        flag[i] = cmp_ok(a[i], ref, cmp) ? 1u : 0u;
}

__global__ void k_fill_indexes(const unsigned int* __restrict__ flag, const unsigned int* __restrict__ off, long n,
                               unsigned int* __restrict__ ids) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        if (flag[i]) ids[off[i]] = (unsigned int)i;
}

// halo flags of a slab: x[i][axis] below the lower threshold, at or above the upper
__global__ void k_slab_mark(const double* __restrict__ x, long n, int axis, double lo_thr, double hi_thr,
                            unsigned int* __restrict__ f0, unsigned int* __restrict__ f1) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double a = x[3 * i + axis];
        f0[i] = a < lo_thr ? 1u : 0u;
        f1[i] = a >= hi_thr ? 1u : 0u;
    }
}

}  // namespace pd

using namespace pd;

extern "C" {

int pd_remove_marked(pd_vd h, int prop, void* stream) {
    if (!h || prop < 0 || prop >= (int)h->props.size()) return PD_EINVAL;
    const Prop& M = h->props[prop];
    cudaStream_t st = S(stream);
    const long n = h->n_real;
    if (n == 0) return PD_OK;
    if (n >= (1L << 32)) return PD_EINVAL;
    // keep bytes and the per-tile counts (scanned in place); the total to n_keep
    const long nt = (n + CT_TILE - 1) / CT_TILE;
    PD_TRY(h->tmp2.ensure((size_t)n + sizeof(unsigned int) * (size_t)nt + 16));
    unsigned char* keep = h->tmp2.as<unsigned char>();
    unsigned int* part = reinterpret_cast<unsigned int*>(keep + (((size_t)n + 15) & ~(size_t)15));
    const unsigned g = (unsigned)nt;
    // the kept particles go straight into new storage of the same capacity, which
    // then replaces the old (the reference swaps its compacted vectors in,
    // vector_dist_cuda_funcs.cuh:405-418); after the first call the storage comes
    // from the library's block cache.  It is taken before the first launch: taking
    // a block freed since the last synchronisation synchronises the device, which
    // between the launches would stall them.  The scatter needs no count on the
    // host, so flip, scan and scatter run back to back and the call synchronises once.
    void* np = nullptr;
    int* ng = nullptr;
    std::vector<char*> nprops;
    PD_TRY(alloc_storage(h, h->cap, &np, &ng, nprops));
    switch (M.type) {
        case PD_F64: pd::launch(k_flip_mark<double>, g, CT_BLOCK, 0, st, (double*)M.d, n, keep, part); break;
        case PD_F32: pd::launch(k_flip_mark<float>, g, CT_BLOCK, 0, st, (float*)M.d, n, keep, part); break;
        case PD_I32: pd::launch(k_flip_mark<int>, g, CT_BLOCK, 0, st, (int*)M.d, n, keep, part); break;
        case PD_U32: pd::launch(k_flip_mark<unsigned int>, g, CT_BLOCK, 0, st, (unsigned int*)M.d, n, keep, part); break;
        case PD_I64: pd::launch(k_flip_mark<long long>, g, CT_BLOCK, 0, st, (long long*)M.d, n, keep, part); break;
        default:
            free_storage(np, ng, nprops);
            return PD_EINVAL;
    }
    if (cudaGetLastError() != cudaSuccess || scan_partials(part, nt, &h->ctrl->n_keep, st) != PD_OK) {
        cudaStreamSynchronize(st);
        free_storage(np, ng, nprops);
        set_error("remove_marked: the compaction kernels failed");
        return PD_ECUDA;
    }
    struct Col {
        const unsigned char* s;
        unsigned char* d;
        int w;
    };
    std::vector<Col> cols;
    cols.push_back({(const unsigned char*)h->pos, (unsigned char*)np, h->pos_bytes});
    cols.push_back({(const unsigned char*)h->gid, (unsigned char*)ng, (int)sizeof(int)});
    for (size_t p = 0; p < h->props.size(); ++p) {
        const Prop& P = h->props[p];
        for (int c = 0; c < P.ncomp; ++c) {
            const size_t o = (size_t)c * h->cap * P.esize;
            cols.push_back({(const unsigned char*)P.d + o, (unsigned char*)nprops[p] + o, P.esize});
        }
    }
    int rc = PD_OK;
    for (size_t c0 = 0; c0 < cols.size() && rc == PD_OK; c0 += CMAXC) {
        const size_t c1 = std::min(cols.size(), c0 + (size_t)CMAXC);
        ColSet C;
        memset(&C, 0, sizeof(C));
        C.nc = (int)(c1 - c0);
        for (size_t c = c0; c < c1; ++c) {
            C.src[c - c0] = cols[c].s;
            C.dst[c - c0] = cols[c].d;
            C.wsize[c - c0] = cols[c].w;
        }
        pd::launch(k_compact_scatter, g, CT_BLOCK, 0, st, C, n, (const unsigned char*)keep, (const unsigned int*)part);
        if (cudaGetLastError() != cudaSuccess) rc = PD_ECUDA;
    }
    if (rc == PD_OK && cudaMemcpyAsync(&h->ctrl_h->n_keep, &h->ctrl->n_keep, sizeof(unsigned int),
                                       cudaMemcpyDeviceToHost, st) != cudaSuccess)
        rc = PD_ECUDA;
    // the old storage returns to the cache only after the scatter has read it
    if (cudaStreamSynchronize(st) != cudaSuccess) rc = PD_ECUDA;
    if (rc != PD_OK) {
        free_storage(np, ng, nprops);
        set_error("remove_marked: the compaction kernels failed");
        return rc;
    }
    const long k = h->ctrl_h->n_keep;
    if (k == n) {  // nothing marked: the particles stay, the mark stays flipped
        free_storage(np, ng, nprops);
        return PD_OK;
    }
    std::vector<char*> old;
    for (auto& P : h->props) old.push_back(P.d);
    free_storage(h->pos, h->gid, old);
    h->pos = np;
    h->gid = ng;
    for (size_t p = 0; p < h->props.size(); ++p) h->props[p].d = nprops[p];
    h->n_real = h->n_total = k;
    h->n_img = 0;
    h->img_valid = false;
    h->epoch++;
    return PD_OK;
}

int pd_get_indexes_by_type(pd_vd h, int prop, int cmp, long long value, long end, unsigned int* ids, long cap,
                           long* n_out, void* stream) {
    if (!h || !n_out || prop < 0 || prop >= (int)h->props.size() || cmp < PD_CMP_EQ || cmp > PD_CMP_GE || cap < 0)
        return PD_EINVAL;
    const Prop& P = h->props[prop];
    cudaStream_t st = S(stream);
    long n = end < 0 ? h->n_real : std::min(end, h->n_total);
    *n_out = 0;
    if (n <= 0) return PD_OK;
    if (n >= (1L << 32)) return PD_EINVAL;
    PD_TRY(h->tmp2.ensure(sizeof(unsigned int) * 3 * (size_t)n));
    unsigned int* flag = h->tmp2.as<unsigned int>();
    unsigned int* off = flag + n;
    unsigned int* out = off + n;
    const unsigned g = grid_for(n, 256);
    switch (P.type) {
        case PD_F64: pd::launch(k_mark_indexes<double>, g, 256, 0, st, (const double*)P.d, n, (double)value, cmp, flag); break;
        case PD_F32: pd::launch(k_mark_indexes<float>, g, 256, 0, st, (const float*)P.d, n, (float)value, cmp, flag); break;
        case PD_I32: pd::launch(k_mark_indexes<int>, g, 256, 0, st, (const int*)P.d, n, (int)value, cmp, flag); break;
        case PD_U32:
            pd::launch(k_mark_indexes<unsigned int>, g, 256, 0, st, (const unsigned int*)P.d, n, (unsigned int)value,
                       cmp, flag);
            break;
        case PD_I64: pd::launch(k_mark_indexes<long long>, g, 256, 0, st, (const long long*)P.d, n, value, cmp, flag); break;
        default: return PD_EINVAL;
    }
    PD_LAUNCH_CHECK();
    PD_TRY(scan_u32(flag, off, n, &h->ctrl->n_keep, h->scan_scratch, st));
    pd::launch(k_fill_indexes, g, 256, 0, st, (const unsigned int*)flag, (const unsigned int*)off, n, out);
    PD_LAUNCH_CHECK();
    PD_CUDA(cudaMemcpyAsync(&h->ctrl_h->n_keep, &h->ctrl->n_keep, sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
    PD_CUDA(cudaStreamSynchronize(st));
    const long m = h->ctrl_h->n_keep;
    *n_out = m;
    if (m > cap) {
        set_error("get_indexes_by_type: %ld indexes, room for %ld", m, cap);
        return PD_EOVERFLOW;
    }
    if (m > 0) {
        if (!ids) return PD_EINVAL;
        // ids may be device or host memory (unified addressing)
        PD_CUDA(cudaMemcpyAsync(ids, out, sizeof(unsigned int) * m, cudaMemcpyDefault, st));
        PD_CUDA(cudaStreamSynchronize(st));
    }
    return PD_OK;
}

int pd_slab_halo(const double* x, long n, int axis, double lo_thr, double hi_thr, int* idx_lo, int* idx_hi,
                 long* n_lo, long* n_hi, void* stream) {
    if (!x || n < 0 || axis < 0 || axis > 2 || !n_lo || !n_hi) return PD_EINVAL;
    *n_lo = 0;
    *n_hi = 0;
    if (n == 0) return PD_OK;
    if (n >= (1L << 31)) return PD_EINVAL;
    PD_TRY(check_device_ptr(x, "pd_slab_halo", "the positions"));
    int dev = 0;
    PD_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return PD_EINVAL;
    cudaStream_t st = S(stream);
    // scratch of the calls on each device (one call at a time): flags, offsets,
    // index lists, totals
    static std::mutex mu;
    static Buf work_dev[64], scratch_dev[64];
    std::lock_guard<std::mutex> lk(mu);
    Buf& work = work_dev[dev];
    Buf& scratch = scratch_dev[dev];
    PD_TRY(work.ensure(sizeof(unsigned int) * (6 * (size_t)n + 2)));
    unsigned int* f0 = work.as<unsigned int>();
    unsigned int *f1 = f0 + n, *o0 = f1 + n, *o1 = o0 + n, *l0 = o1 + n, *l1 = l0 + n, *tot = l1 + n;
    const unsigned g = grid_for(n, 256);
    pd::launch(k_slab_mark, g, 256, 0, st, x, n, axis, lo_thr, hi_thr, f0, f1);
    PD_LAUNCH_CHECK();
    PD_TRY(scan_u32(f0, o0, n, tot, scratch, st));
    PD_TRY(scan_u32(f1, o1, n, tot + 1, scratch, st));
    pd::launch(k_fill_indexes, g, 256, 0, st, (const unsigned int*)f0, (const unsigned int*)o0, n, l0);
    pd::launch(k_fill_indexes, g, 256, 0, st, (const unsigned int*)f1, (const unsigned int*)o1, n, l1);
    PD_LAUNCH_CHECK();
    unsigned int m[2] = {0, 0};
    PD_CUDA(cudaMemcpyAsync(m, tot, sizeof(m), cudaMemcpyDeviceToHost, st));
    PD_CUDA(cudaStreamSynchronize(st));
    *n_lo = m[0];
    *n_hi = m[1];
    if ((m[0] && !idx_lo) || (m[1] && !idx_hi)) return PD_EINVAL;
    // the lists may go to device or host memory (unified addressing)
    if (m[0]) PD_CUDA(cudaMemcpyAsync(idx_lo, l0, sizeof(int) * m[0], cudaMemcpyDefault, st));
    if (m[1]) PD_CUDA(cudaMemcpyAsync(idx_hi, l1, sizeof(int) * m[1], cudaMemcpyDefault, st));
    PD_CUDA(cudaStreamSynchronize(st));
    return PD_OK;
}

}  // extern "C"
