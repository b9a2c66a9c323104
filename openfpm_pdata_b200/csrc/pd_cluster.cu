// pd_cluster.cu -- velocity-Verlet LJ steps of a small system with the cell list
// rebuilt every step, all steps of a run in one launch of one thread-block cluster.
//
// The cell-list step (kick-drift, wrap, periodic images, cell list of particles and
// images, 27-cell force walk, kick, energies) is a dozen dependent phases over a
// few thousand particles: as separate kernels (even replayed from a CUDA graph)
// the launch gaps dominate.  Here one cluster of 16 CTAs (16 SMs; 8 where the GPU
// cannot place a cluster of 16) runs every phase of every step, with the cluster barrier (barrier.cluster, a hardware
// barrier that every thread of the cluster reaches the same number of times: the
// control flow around it is uniform) between dependent phases; the scans run on
// the cluster's first CTA.  Data stay in global memory (a few hundred KB, L2
// resident).  The phases restate the separate kernels' operations (k_kick_drift,
// k_wrap, k_ghost_count / k_ghost_write, the counting sort with its stabilising
// rank pass, k_lj_cell, k_kick) in the same arithmetic order per particle; only
// the order of the energy sums differs.
#include <cooperative_groups.h>
#include <cstring>

#include "pd_device.cuh"
#include "pd_ghost_dev.cuh"
#include "pd_internal.cuh"
#include "pd_lj.cuh"
#include "pd_md.cuh"

namespace cg = cooperative_groups;

namespace pd {

static constexpr int CL_CTAS = 16;       // CTAs of the cluster (non-portable size; 8 where 16 cannot be placed)
static constexpr int CL_THREADS = 1024;  // threads per CTA
static constexpr long CL_MAXN = 65536;   // real particles handled by the cluster path
static constexpr unsigned int CL_SORT_CAP = 256;  // shared ints per warp for ordering a crowded cell

template <class T> struct ClArgs {
    typename V4<T>::type* pos;  // real [0, n), images [n, n + img_cap)
    int* gid;
    int* img_src;
    unsigned char* img_shift;
    T* v;
    T* f;
    long cap, n, img_cap;
    T lo[3], hi[3];
    int per[3];
    const BoxSet<T>* boxes;
    const T* shifts;
    Grid<T> G;
    long ncells;
    unsigned int *cnt, *cstart, *cell_of, *slot, *img_cnt, *img_start, *tot;
    int *sorted_tmp, *sorted;
    typename V4<T>::type* pcs;  // cell-ordered copy of positions and images, w = index bits
    int q;                      // lanes per particle in the force walk (a power of two <= 32)
    LJP<T> P;
    T half, dt;
    double mass;
    double* part;  // [CTAs][3]: potential energy, virial, kinetic energy
    double* E;     // [steps][4]
    int steps;
    unsigned int* err;
};

// coherent loads of position records (data written earlier in the same launch by
// other CTAs of the cluster: not through the read-only cache)
__device__ __forceinline__ double4 ldc4(const double4* p, long i) {
    const double2* q = reinterpret_cast<const double2*>(p + i);
    const double2 a = q[0], b = q[1];
    return make_double4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ float4 ldc4(const float4* p, long i) { return p[i]; }

template <class T> __device__ __forceinline__ T idx_bits(int i);
template <> __device__ __forceinline__ double idx_bits<double>(int i) { return __longlong_as_double((long long)i); }
template <> __device__ __forceinline__ float idx_bits<float>(int i) { return __int_as_float(i); }
template <class T> __device__ __forceinline__ int idx_of(T w);
template <> __device__ __forceinline__ int idx_of<double>(double w) { return (int)__double_as_longlong(w); }
template <> __device__ __forceinline__ int idx_of<float>(float w) { return __float_as_int(w); }

// exclusive scan of a[0, n) into out (out may alias a), total to *total; one CTA
__device__ void cta_scan(const unsigned int* a, unsigned int* out, long n, unsigned int* total, unsigned int* wsum) {
    const long C = (n + CL_THREADS - 1) / CL_THREADS;
    const long b = (long)threadIdx.x * C;
    unsigned int loc = 0;
    for (long j = 0; j < C; ++j)
        if (b + j < n) loc += a[b + j];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned int inc = loc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) wsum[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const unsigned int y = wsum[lane];
        unsigned int z = y;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned int t = __shfl_up_sync(0xffffffffu, z, o);
            if (lane >= o) z += t;
        }
        wsum[lane] = z - y;
    }
    __syncthreads();
    unsigned int run = wsum[warp] + inc - loc;
    for (long j = 0; j < C; ++j)
        if (b + j < n) {
            const unsigned int v = a[b + j];
            out[b + j] = run;
            run += v;
        }
    if (threadIdx.x == CL_THREADS - 1) *total = run;
    __syncthreads();
}

template <class T>
__global__ void __launch_bounds__(CL_THREADS, 1) k_md_cluster(ClArgs<T> A) {
    typedef typename V4<T>::type T4;
    cg::cluster_group cluster = cg::this_cluster();
    __shared__ BoxSet<T> B;
    __shared__ unsigned int wsum[32];
    __shared__ int cell_sort_buf[32][CL_SORT_CAP];  // per warp: in-cell ordering of crowded cells
    for (int i = threadIdx.x; i < (int)(sizeof(BoxSet<T>) / 4); i += blockDim.x)
        reinterpret_cast<int*>(&B)[i] = reinterpret_cast<const int*>(A.boxes)[i];
    __syncthreads();
    const unsigned int rank = cluster.block_rank();
    const long gt = (long)rank * CL_THREADS + threadIdx.x;
    const int nct = (int)cluster.num_blocks();
    const long GT = (long)nct * CL_THREADS;
    const long n = A.n;
    unsigned int bad = 0, ovf = 0;
    for (int s = 0; s < A.steps; ++s) {
        // 1. v += h f; x += dt v; periodic wrap.  Cell counts cleared.
        for (long i = gt; i < n; i += GT) {
            T4 x = ldc4(A.pos, i);
            const T vx = A.v[i] + A.half * A.f[i];
            const T vy = A.v[A.cap + i] + A.half * A.f[A.cap + i];
            const T vz = A.v[2 * A.cap + i] + A.half * A.f[2 * A.cap + i];
            x.x += A.dt * vx;
            x.y += A.dt * vy;
            x.z += A.dt * vz;
            A.v[i] = vx;
            A.v[A.cap + i] = vy;
            A.v[2 * A.cap + i] = vz;
            if (A.per[0]) x.x = periodic_l(x.x, A.hi[0], A.lo[0]);
            if (A.per[1]) x.y = periodic_l(x.y, A.hi[1], A.lo[1]);
            if (A.per[2]) x.z = periodic_l(x.z, A.hi[2], A.lo[2]);
            st4(A.pos, i, x);
        }
        for (long c = gt; c <= A.ncells; c += GT) A.cnt[c] = 0u;
        cluster.sync();
        // 2. images per particle: distinct shift ids of the ghost boxes holding it
        for (long i = gt; i < n; i += GT) {
            const T4 r = ldc4(A.pos, i);
            unsigned int c = 0;
            int old = -1;
            for (int b = 0; b < B.nb; ++b) {
                const int sv = B.sv[b];
                if (inside_np(B, b, r.x, r.y, r.z) && sv != old) {
                    old = sv;
                    ++c;
                }
            }
            A.img_cnt[i] = c;
        }
        cluster.sync();
        // 3. image offsets (first CTA)
        if (rank == 0) cta_scan(A.img_cnt, A.img_start, n, A.tot, wsum);
        cluster.sync();
        // 4. the images, particle-major, shift ids ascending
        for (long i = gt; i < n; i += GT) {
            const T4 r = ldc4(A.pos, i);
            long m = A.img_start[i];
            int old = -1;
            for (int b = 0; b < B.nb; ++b) {
                const int sv = B.sv[b];
                if (inside_np(B, b, r.x, r.y, r.z) && sv != old) {
                    old = sv;
                    if (m < A.img_cap && n + m < A.cap) {
                        T4 q;
                        q.x = r.x - A.shifts[3 * sv];
                        q.y = r.y - A.shifts[3 * sv + 1];
                        q.z = r.z - A.shifts[3 * sv + 2];
                        q.w = r.w;
                        st4(A.pos, n + m, q);
                        A.gid[n + m] = A.gid[i];
                        A.img_src[m] = (int)i;
                        A.img_shift[m] = (unsigned char)sv;
                    } else {
                        ovf = 1u;
                    }
                    ++m;
                }
            }
        }
        cluster.sync();
        // 5. cell of every particle and image, slot from the cell's counter
        const long m_img = min((long)*A.tot, A.img_cap);
        const long nt = n + m_img;
        for (long k = gt; k < nt; k += GT) {
            const T4 r = ldc4(A.pos, k);
            const unsigned int c = (unsigned int)A.G.cell(r.x, r.y, r.z, bad);
            A.cell_of[k] = c;
            A.slot[k] = atomicAdd(&A.cnt[c], 1u);
        }
        cluster.sync();
        // 6. cell starts (first CTA)
        if (rank == 0) cta_scan(A.cnt, A.cstart, A.ncells + 1, A.tot + 1, wsum);
        cluster.sync();
        // 7. scatter to the unordered slot
        for (long k = gt; k < nt; k += GT) A.sorted_tmp[A.cstart[A.cell_of[k]] + A.slot[k]] = (int)k;
        cluster.sync();
        // 8. in-cell order by index (one warp per cell), then the cell-ordered position copy
        {
            const long warp = gt >> 5, nw = GT >> 5;
            const int lane = threadIdx.x & 31;
            for (long c = warp; c < A.ncells; c += nw) {
                const unsigned int b0 = A.cstart[c], e0 = A.cstart[c + 1], cn = e0 - b0;
                warp_cell_order(A.sorted_tmp + b0, A.sorted + b0, cn, cell_sort_buf[threadIdx.x >> 5], CL_SORT_CAP);
                __syncwarp();
                for (unsigned int a = lane; a < cn; a += 32) {
                    const int v = A.sorted[b0 + a];
                    T4 r = ldc4(A.pos, v);
                    r.w = idx_bits<T>(v);
                    st4(A.pcs, b0 + a, r);
                }
            }
        }
        cluster.sync();
        // 9. forces: q lanes per particle walk the 27 cells through the cell-ordered
        // copy (three cells of a row are one contiguous range), their sums meet by
        // shuffles; then v += h f and the energies
        double pe = 0, vir = 0, ke = 0;
        {
            const int q = A.q;
            const long per = GT / q;
            const long iters = (n + per - 1) / per;  // the same for every thread (whole warps shuffle)
            const int sub = (int)(gt % q);
            for (long it = 0; it < iters; ++it) {
                const long i = gt / q + it * per;
                const bool active = i < n;
                const T4 xi = ldc4(A.pos, active ? i : 0);
                const int c = active ? (int)A.cell_of[i] : 0;
                const int c0 = c % A.G.gs[0], c1 = (c / A.G.gs[0]) % A.G.gs[1], c2 = c / (A.G.gs[0] * A.G.gs[1]);
                T fx = 0, fy = 0, fz = 0, e = 0, w = 0;
                for (int r9 = 0; r9 < 9 && active; ++r9) {
                    const int y = c1 + r9 % 3 - 1, z = c2 + r9 / 3 - 1;
                    if (y < 0 || z < 0 || y >= A.G.gs[1] || z >= A.G.gs[2]) continue;
                    const int xa = max(c0 - 1, 0), xb = min(c0 + 1, A.G.gs[0] - 1);
                    const long rb = (long)A.G.gs[0] * (y + (long)A.G.gs[1] * z);
                    const unsigned int ka = A.cstart[rb + xa], kb = A.cstart[rb + xb + 1];
#pragma unroll 2
                    for (unsigned int k = ka + sub; k < kb; k += q) {
                        const T4 xq = ldc4(A.pcs, k);
                        if (idx_of<T>(xq.w) == (int)i) continue;
                        const T dx = xi.x - xq.x, dy2 = xi.y - xq.y, dz2 = xi.z - xq.z;
                        const T r2 = dist2(dx, dy2, dz2);
                        if (r2 < A.P.rc2) lj_acc(A.P, r2, dx, dy2, dz2, fx, fy, fz, e, w);
                    }
                }
                for (int o = 1; o < q; o <<= 1) {
                    fx += __shfl_xor_sync(0xffffffffu, fx, o);
                    fy += __shfl_xor_sync(0xffffffffu, fy, o);
                    fz += __shfl_xor_sync(0xffffffffu, fz, o);
                    e += __shfl_xor_sync(0xffffffffu, e, o);
                    w += __shfl_xor_sync(0xffffffffu, w, o);
                }
                if (active && sub == 0) {
                    A.f[i] = fx;
                    A.f[A.cap + i] = fy;
                    A.f[2 * A.cap + i] = fz;
                    pe += 0.5 * (double)e;
                    vir += 0.5 * (double)w;
                    const T vx = A.v[i] + A.half * fx;
                    const T vy = A.v[A.cap + i] + A.half * fy;
                    const T vz = A.v[2 * A.cap + i] + A.half * fz;
                    A.v[i] = vx;
                    A.v[A.cap + i] = vy;
                    A.v[2 * A.cap + i] = vz;
                    ke += 0.5 * A.mass * ((double)vx * vx + (double)vy * vy + (double)vz * vz);
                }
            }
        }
        pe = block_sum<double, CL_THREADS>(pe);
        vir = block_sum<double, CL_THREADS>(vir);
        ke = block_sum<double, CL_THREADS>(ke);
        if (threadIdx.x == 0) {
            A.part[3 * rank] = pe;
            A.part[3 * rank + 1] = vir;
            A.part[3 * rank + 2] = ke;
        }
        cluster.sync();
        // 10. the step's energies, CTA partials in a fixed order
        if (rank == 0 && threadIdx.x == 0) {
            double a = 0, b = 0, c = 0;
            for (int r = 0; r < nct; ++r) {
                a += A.part[3 * r + 2];
                b += A.part[3 * r];
                c += A.part[3 * r + 1];
            }
            double* Es = A.E + 4 * (long)s;
            Es[0] = a;
            Es[1] = b;
            Es[2] = c;
            Es[3] = 1.0;
        }
        // the next step rewrites part only after several cluster barriers
    }
    if (bad) atomicOr(A.err, ERR_CELL_RANGE);
    if (ovf) atomicOr(A.err, ERR_IMG_OVERFLOW);
}

template <class T> static int md_run_cluster_t(pd_md md, int steps, cudaStream_t st, double* E) {
    pd_vd h = md->h;
    pd_cl cl = md->cl;
    const long n = h->n_real;
    Prop& V = h->props[md->mp.vel_prop];
    Prop& F = h->props[md->mp.force_prop];
    // image room: the last count with a margin
    const long img_cap = h->n_img + h->n_img / 2 + 1024;
    PD_TRY(ensure_capacity(h, n + img_cap + 1, st));
    const long nt = n + img_cap;
    const long nc = cl->ncells;
    PD_TRY(cl->cell_cnt.ensure(sizeof(unsigned int) * (nc + 1)));
    PD_TRY(cl->cell_start.ensure(sizeof(unsigned int) * (nc + 1)));
    PD_TRY(cl->cell_of.ensure(sizeof(unsigned int) * nt));
    PD_TRY(cl->slot.ensure(sizeof(unsigned int) * nt));
    PD_TRY(cl->sorted.ensure(sizeof(int) * nt));
    PD_TRY(cl->sorted_tmp.ensure(sizeof(int) * nt));
    PD_TRY(h->img_cnt.ensure(sizeof(unsigned int) * (n + 1)));
    PD_TRY(h->img_start.ensure(sizeof(unsigned int) * (n + 1)));
    PD_TRY(h->img_src.ensure(sizeof(int) * img_cap));
    PD_TRY(h->img_shift.ensure(img_cap));
    PD_TRY(md->kpart.ensure(sizeof(double) * 3 * CL_CTAS + sizeof(unsigned int) * 4));
    PD_TRY(md->E.ensure(sizeof(double) * 4 * (steps + 1)));
    if (h->nbox == 0) PD_TRY(ghost_boxes_upload(h, st));
    ClArgs<T> A;
    memset(&A, 0, sizeof(A));
    A.pos = (typename V4<T>::type*)h->pos;
    A.gid = h->gid;
    A.img_src = h->img_src.as<int>();
    A.img_shift = h->img_shift.as<unsigned char>();
    A.v = (T*)V.d;
    A.f = (T*)F.d;
    A.cap = h->cap;
    A.n = n;
    A.img_cap = img_cap;
    for (int d = 0; d < 3; ++d) {
        A.lo[d] = (T)h->lo[d];
        A.hi[d] = (T)h->hi[d];
        A.per[d] = h->bc[d] == PD_PERIODIC;
        A.G.lo[d] = (T)cl->box_lo[d];
        A.G.sp[d] = (T)cl->spacing[d];
        A.G.gs[d] = cl->gs[d];
    }
    A.G.pad = cl->pad;
    A.boxes = h->boxes.as<BoxSet<T>>();
    A.shifts = h->shifts.as<T>();
    A.ncells = nc;
    A.cnt = cl->cell_cnt.as<unsigned int>();
    A.cstart = cl->cell_start.as<unsigned int>();
    A.cell_of = cl->cell_of.as<unsigned int>();
    A.slot = cl->slot.as<unsigned int>();
    A.img_cnt = h->img_cnt.as<unsigned int>();
    A.img_start = h->img_start.as<unsigned int>();
    A.sorted = cl->sorted.as<int>();
    A.sorted_tmp = cl->sorted_tmp.as<int>();
    PD_TRY(h->tmp.ensure((size_t)nt * h->pos_bytes));
    A.pcs = h->tmp.as<typename V4<T>::type>();

    A.P.eps24 = (T)(24.0 * md->lj.eps);
    A.P.eps4 = (T)(4.0 * md->lj.eps);
    A.P.sig2 = (T)(md->lj.sigma * md->lj.sigma);
    const T rc = (T)md->lj.r_cut;
    A.P.rc2 = rc * rc;
    A.half = (T)(0.5 * md->mp.dt / md->mp.mass);
    A.dt = (T)md->mp.dt;
    A.mass = md->mp.mass;
    A.part = md->kpart.as<double>();
    A.tot = reinterpret_cast<unsigned int*>(A.part + 3 * CL_CTAS);
    A.E = md->E.as<double>();
    A.steps = steps;
    A.err = &h->ctrl->err;
    // one cluster of 16 CTAs (one per SM) where the GPU can place it, else 8
    static int nct = 0;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1] = {};
    cfg.blockDim = dim3(CL_THREADS, 1, 1);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    if (nct == 0) {
        nct = 8;
        if (cudaFuncSetAttribute(k_md_cluster<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
            cfg.gridDim = dim3(CL_CTAS, 1, 1);
            attr[0].val.clusterDim.x = CL_CTAS;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            int nclusters = 0;
            if (cudaOccupancyMaxActiveClusters(&nclusters, k_md_cluster<T>, &cfg) == cudaSuccess && nclusters >= 1)
                nct = CL_CTAS;
        }
        cudaGetLastError();
    }
    {
        const long GT = (long)nct * CL_THREADS;
        int q = 1;
        while (q < 32 && (long)(2 * q) * n <= GT) q <<= 1;
        A.q = q;
    }
    cfg.gridDim = dim3(nct, 1, 1);
    attr[0].val.clusterDim.x = nct;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    PD_CUDA(cudaLaunchKernelEx(&cfg, k_md_cluster<T>, A));
    __atomic_fetch_add(&g_launches, 1ull, __ATOMIC_RELAXED);
    md->cluster_ctas = nct;
    unsigned int tot = 0;
    PD_CUDA(cudaMemcpyAsync(&tot, A.tot, sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
    if (E && steps > 0) PD_CUDA(cudaMemcpyAsync(E, md->E.p, sizeof(double) * 4 * steps, cudaMemcpyDeviceToHost, st));
    PD_TRY(read_ctrl(h, st));  // synchronises the stream
    if (h->ctrl_h->err & (ERR_IMG_OVERFLOW | ERR_CELL_RANGE)) {
        set_error("pd_md_run: cluster step overflow or particle outside the cell grid (err=0x%x)", h->ctrl_h->err);
        return PD_EOVERFLOW;
    }
    // the vector holds the last step's images (generation order) with their records;
    // their properties are refreshed from the sources
    h->n_img = tot;
    h->n_total = n + tot;
    h->img_valid = true;
    h->img_gen_order = true;
    PD_TRY(ghost_replay(h, ~0ul, false, nullptr, h->n_img, st));
    md->steps += steps;
    md->builds += steps;
    h->epoch++;
    return PD_OK;
}

bool md_cluster_eligible(pd_md md) {
    pd_vd h = md->h;
    return md->mp.use_cell_list && md->physics == 0 && !md->mixed && !md->timing && md->cl && h->n_real > 0 &&
           h->n_real <= CL_MAXN && md->cl->pad == 1 && md->cl->ncells <= 4L * CL_MAXN;
}

int md_run_cluster(pd_md md, int steps, cudaStream_t st, double* E) {
    if (!md->ready) {
        PD_TRY(md_rebuild(md, st));
        PD_TRY(md_forces(md, st));
        md->ready = true;
        PD_TRY(read_ctrl(md->h, st));
        md->h->n_img = md->h->ctrl_h->n_img;
    }
    if (steps == 0) return PD_OK;
    return md->h->dtype == PD_F64 ? md_run_cluster_t<double>(md, steps, st, E)
                                  : md_run_cluster_t<float>(md, steps, st, E);
}

}  // namespace pd
