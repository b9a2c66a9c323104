// pd_serve.cu -- serving loop: many independent LJ systems (precision form)
// resident on one GPU, stepped together by persistent batched kernels.
//
// The reference's only many-systems idiom is a test kernel reading an array of
// vector_dist / cell-list views (Vector/cuda/vector_dist_gpu_MP_tests.cu:427-781).
// Here that array is a device table of system descriptors (SysDesc) and one
// velocity-Verlet step of every active system is ONE CUDA graph of persistent
// kernels over the work of all systems:
//   kick-drift   256-particle chunks of every system; largest displacement per system
//   decide       one block: rebuild flag per system (displacement > skin/2) and the
//                compacted work lists of the flagged systems
//   rebuild      flagged systems only, every phase batched over them: offsets ->
//                FP64 positions + wrap + cell hash, per-system scans, stable
//                counting sort, reorder, periodic images (count, scan, write),
//                image cell sort, FP32 staging copies and offsets, tiled Verlet
//                rows (TMA-staged tiles, the single-system build's row code)
//   replay       image offsets of the systems that did not rebuild
//   forces       tiles of every system from an atomic work queue (load balance over
//                uneven systems); the tile body is the single-system mixed kernel's
//   kick         chunks, kinetic energy per chunk
//   energies     one block per system, fixed-order sums -> E[step]
// The host synchronises once per step (the graph's end) to read the rebuild
// flags and error bits and to retire finished systems.  Partials are indexed by
// (system, work item), never by CTA, and every rebuild phase reproduces the
// single-system build's arithmetic and orders, so a system's results do not
// depend on the other systems in the batch and equal the single-system driver's.
//
// Slots: a system runs in a slot whose device containers (vector, integrator,
// build scratch) are kept after the system retires and reused by the next one
// (buffers only grow), so admission and retirement allocate nothing in steady
// state.  Admission: FIFO; a request is admitted when a slot is free and its
// memory estimate fits the server's HBM budget, which is reserved in the server's
// memory pool at creation (capped by the free memory then);
// its first build and forces run through the single-system path, with the slot's
// image capacity reserved beforehand with a margin for the batched rebuilds.
// Autotuner: per size bucket (floor(log2 N)), the first admitted system times the
// force kernel for several tile widths on a throw-away copy; the best is kept.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <deque>
#include <map>
#include <memory>
#include <condition_variable>
#include <mutex>
#include <system_error>
#include <thread>
#include <vector>

#include "pd_device.cuh"
#include "pd_ghost_dev.cuh"
#include "pd_internal.cuh"
#include "pd_lj.cuh"
#include "pd_md.cuh"
#include "pd_mixed.cuh"
#include "pd_mixed_dev.cuh"
#include "pd_tile.cuh"
#include "pd_tile_dev.cuh"

namespace pd {

static constexpr int SRV_SMEM = 48 * 1024;            // staging bytes per tile CTA (fixed: graph-invariant)
static constexpr unsigned SRV_CAP = SRV_SMEM / 16;    // staged FP32 records per tile
static constexpr int SRV_BSMEM = 24 * 1024;           // staging bytes per CTA of the batched list build (one z-layer)
static constexpr unsigned SRV_BCAP = SRV_BSMEM / 16;
static constexpr int SRV_BIG = 192 * 1024;            // staging of the overflow kernels (tiles beyond SRV_CAP)
static constexpr unsigned SRV_BIG_CAP = SRV_BIG / 16;
static constexpr int CHUNK = 256;                     // threads per block of the chunked kernels
static constexpr int SCH = 1024;                      // elements per scan chunk
static constexpr int MAXS = 1024;                     // slots at most

// rebuild work kinds (items per system)
// K_P  particle chunks of 256          K_C  cell chunks of 256 (ncell + 1 counters)
// K_Q  cell scan chunks of 1024        K_QP particle scan chunks of 1024
// K_I  image chunks of 256 (capacity)  K_A  particle + image chunks of 256 (capacity)
// K_T  tiles                           K_W  cells, 8 per block (one warp each)
enum { K_P, K_C, K_Q, K_QP, K_I, K_A, K_T, K_W, NK };

struct SysDesc {
    // state (slot containers)
    float4* off;
    float4* offb;
    float4* offK;
    double4* pos;
    int* gid;
    int* img_src;
    unsigned char* img_shift;
    float* v;
    float* f;
    long cap, n_real, img_cap, ncell;
    unsigned int* n_img;  // device image count of the last build
    // cell grid (side r_cut + skin) and tiles
    Grid<double> G;
    CellGeom C;
    double L;
    TileGeom tg;
    unsigned int* csR;
    unsigned int* csI;
    unsigned int* nbr;
    int* nn;
    long tstride;
    int max_nn;
    float sx, sy, sz;
    float lo_thr, hi_thr;
    double r2;
    int lanes, block;  // the force kernel's lanes per particle and CTA size for this system (tuned per size)
    const BoxSet<double>* boxes;
    const double* shifts;
    // build scratch
    unsigned int* cntR;
    unsigned int* cntI;
    unsigned int* cell_of;
    unsigned int* rank;
    unsigned int* img_cnt;
    unsigned int* img_start;
    unsigned int* spart;
    int* sorted;
    int* sorted_tmp;
    double4* scr_pos;
    int* scr_gid;
    float* scr_v;
    int* scr_src;
    unsigned char* scr_shf;
    float4* pos32;
    // step work decomposition (prefixes over the active systems)
    long tile_base, ntiles;
    long chunk_base, nchunk;
    long img_base, nimg_chunk;
    long tpart_base, kpart_base;
    long cnt[NK];  // rebuild work items per kind
    unsigned int* err;
    double* E;
    int* step;
    double mass;
    int slot;
};

// the force kernel's launch shapes: lanes per particle 1, 2, 4 x CTAs of FBLOCK_T, FBLOCK_T / 2
static constexpr int NSHAPE = 6;
__host__ __device__ constexpr int shape_group(int lanes, int block) {
    return (lanes == 1 ? 0 : (lanes == 2 ? 1 : 2)) + (block == FBLOCK_T ? 0 : 3);
}

struct BatchHdr {
    int nsys;
    int pad0;
    long tot_tiles, tot_chunks, tot_img;
    unsigned int ovf_force;  // tiles deferred to the large-staging kernels
    unsigned int ovf_build;
    // force-kernel groups (shape_group: lanes per particle x CTA size): the
    // descriptors list the groups in order, group k's tiles are [grp[k], grp[k+1])
    long grp[NSHAPE + 1];
    unsigned int grp_ctr[NSHAPE];  // work queue of each group's persistent kernel
};

// compacted work of the systems flagged for a rebuild this step
struct RbWork {
    int nflag;
    int pad;
    long tot[NK];
    int sys[MAXS];
    long base[NK][MAXS + 1];
};

__device__ __forceinline__ int find_sys(const SysDesc* __restrict__ D, int nsys, long g, int which) {
    int lo = 0, hi = nsys - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        long b = which == 0 ? D[mid].tile_base : (which == 1 ? D[mid].chunk_base : D[mid].img_base);
        if (b <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// flagged-system index k owning item g of kind K (bases ascending, empty systems skipped)
__device__ __forceinline__ int find_flagged(const RbWork* __restrict__ W, int K, long g) {
    int lo = 0, hi = W->nflag - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (W->base[K][mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// grid-stride loop over the items of kind K of the flagged systems; the body sees
// the system `d` and the item index `c` inside it (block-uniform)
#define RB_LOOP(K)                                                                                  \
    for (long g_ = blockIdx.x; g_ < W->tot[K]; g_ += gridDim.x) {                                   \
        const int k_ = find_flagged(W, K, g_);                                                      \
        const SysDesc& d = D[W->sys[k_]];                                                           \
        const long c = g_ - W->base[K][k_];

#define RB_END }

// exclusive scan over a block of 256 threads (valid in every thread); total in `tot`
__device__ __forceinline__ unsigned int block_scan256(unsigned int v, unsigned int& tot) {
    __shared__ unsigned int ws[8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    if (w == 0) {
        unsigned int t = lane < 8 ? ws[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            unsigned int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < 8) ws[lane] = t;
    }
    __syncthreads();
    const unsigned int r = x - v + (w ? ws[w - 1] : 0u);
    tot = ws[7];
    __syncthreads();
    return r;
}

// exclusive scan of longs over a block of 1024 threads
__device__ __forceinline__ long block_scan1024(long v, long& tot) {
    __shared__ long ws[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    if (w == 0) {
        long t = ws[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            long y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        ws[lane] = t;
    }
    __syncthreads();
    const long r = x - v + (w ? ws[w - 1] : 0L);
    tot = ws[31];
    __syncthreads();
    return r;
}

// ---------------------------------------------------------------------------
// step kernels

__global__ void __launch_bounds__(CHUNK) k_b_kick_drift(const SysDesc* __restrict__ D, const BatchHdr* __restrict__ B,
                                                        float half, float dt, unsigned long long* __restrict__ maxd2,
                                                        const unsigned int* __restrict__ phase) {
    const int nsys = B->nsys;
    const long tot = B->tot_chunks;
    for (long g = blockIdx.x; g < tot; g += gridDim.x) {
        const int s = find_sys(D, nsys, g, 1);
        const SysDesc& d = D[s];
        if (phase[d.slot] == 0) continue;  // first build pending: no step yet
        const long i = (g - d.chunk_base) * CHUNK + threadIdx.x;
        double mx = 0;
        if (i < d.n_real) {
            float4 o = d.off[i];
            const long cap = d.cap;
            float vx = d.v[i] + half * d.f[i];
            float vy = d.v[cap + i] + half * d.f[cap + i];
            float vz = d.v[2 * cap + i] + half * d.f[2 * cap + i];
            o.x = d.C.qf(o.x + dt * vx);
            o.y = d.C.qf(o.y + dt * vy);
            o.z = d.C.qf(o.z + dt * vz);
            d.v[i] = vx;
            d.v[cap + i] = vy;
            d.v[2 * cap + i] = vz;
            d.off[i] = o;
            float4 b = d.offb[i];
            mx = (double)dist2(o.x - b.x, o.y - b.y, o.z - b.z);
        }
        mx = warp_max(mx);
        if ((threadIdx.x & 31) == 0 && mx > 0) atomic_max_nonneg(maxd2 + d.slot, mx);
    }
}

// rebuild flags (first build, or displacement beyond skin/2) and the compacted work
// of the flagged systems (one block of 1024)
__global__ void __launch_bounds__(1024) k_b_decide(const SysDesc* __restrict__ D, const BatchHdr* __restrict__ B,
                                                   const unsigned long long* __restrict__ maxd2, double lim2,
                                                   int always, unsigned int* __restrict__ flag,
                                                   const unsigned int* __restrict__ phase, RbWork* __restrict__ W) {
    const int nsys = B->nsys;
    const int s = threadIdx.x;
    int fl = 0;
    if (s < nsys) {
        const double d2 = __longlong_as_double((long long)maxd2[D[s].slot]);
        fl = (always || phase[D[s].slot] == 0 || d2 > lim2) ? 1 : 0;
        flag[D[s].slot] = (unsigned int)fl;
    }
    long nf = 0;
    const long k = block_scan1024(fl, nf);
    if (fl) W->sys[k] = s;
    if (threadIdx.x == 0) W->nflag = (int)nf;
    for (int K = 0; K < NK; ++K) {
        long tot = 0;
        const long b = block_scan1024(fl ? D[s].cnt[K] : 0L, tot);
        if (fl) W->base[K][k] = b;
        if (threadIdx.x == 0) W->tot[K] = tot;
    }
}

__global__ void __launch_bounds__(CHUNK) k_b_replay(const SysDesc* __restrict__ D, const BatchHdr* __restrict__ B,
                                                    const unsigned int* __restrict__ flag) {
    const int nsys = B->nsys;
    const long tot = B->tot_img;
    for (long g = blockIdx.x; g < tot; g += gridDim.x) {
        const int s = find_sys(D, nsys, g, 2);
        const SysDesc& d = D[s];
        if (flag[d.slot]) continue;
        const long k = (g - d.img_base) * CHUNK + threadIdx.x;
        if (k < (long)*d.n_img) {
            float4 o = d.off[d.img_src[k]], q = d.offK[k];
            float4 r = d.off[d.n_real + k];
            r.x = o.x + q.x;
            r.y = o.y + q.y;
            r.z = o.z + q.z;
            d.off[d.n_real + k] = r;
        }
    }
}

// one tile of system d with its tuned lanes per particle (the overflow kernels)
template <int BLOCK>
__device__ __forceinline__ void b_force_tile_any(const SysDesc& d, long t, unsigned int cap, const LJP<float>& Pr,
                                                 float4* sm, TileShM& S, unsigned long long* bar, unsigned int& uses,
                                                 double& pe, double& vir) {
    if (d.lanes == 1)
        mixed_tile<1, BLOCK>(t, d.off, d.n_real, d.tg, d.csR, d.csI, cap, d.nbr, d.nn, d.tstride, d.sx, d.sy, d.sz, Pr,
                             d.f, d.cap, d.err, sm, S, bar, uses, pe, vir);
    else if (d.lanes == 4)
        mixed_tile<4, BLOCK>(t, d.off, d.n_real, d.tg, d.csR, d.csI, cap, d.nbr, d.nn, d.tstride, d.sx, d.sy, d.sz, Pr,
                             d.f, d.cap, d.err, sm, S, bar, uses, pe, vir);
    else
        mixed_tile<2, BLOCK>(t, d.off, d.n_real, d.tg, d.csR, d.csI, cap, d.nbr, d.nn, d.tstride, d.sx, d.sy, d.sz, Pr,
                             d.f, d.cap, d.err, sm, S, bar, uses, pe, vir);
}

// Persistent force kernel of one shape group (LANES lanes per particle, CTAs of
// BLOCK threads): the tiles [grp[k], grp[k+1]) of the systems of that shape.
template <int LANES, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_b_force(const SysDesc* __restrict__ D, BatchHdr* __restrict__ B,
                                                   LJP<float> Pr, double* __restrict__ tpart,
                                                   long* __restrict__ ovf) {
    extern __shared__ __align__(128) unsigned char tile_raw[];
    float4* sm = reinterpret_cast<float4*>(tile_raw);
    __shared__ TileShM S;
    __shared__ unsigned long long bar;
    __shared__ long cur;
    constexpr int G = shape_group(LANES, BLOCK);
    const long first = B->grp[G], tot = B->grp[G + 1];
    if (first >= tot) return;  // no system of this shape in the batch
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    unsigned int uses = 0;
    const int nsys = B->nsys;
    for (;;) {
        // generic-proxy accesses of the previous tile are ordered before the next bulk copies
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) cur = first + (long)atomicAdd(&B->grp_ctr[G], 1u);
        __syncthreads();
        const long g = cur;
        if (g >= tot) break;
        const int s = find_sys(D, nsys, g, 0);
        const SysDesc& d = D[s];
        double pe = 0, vir = 0;
        if (mixed_tile<LANES, BLOCK>(g - d.tile_base, d.off, d.n_real, d.tg, d.csR, d.csI, SRV_CAP, d.nbr, d.nn,
                                     d.tstride, d.sx, d.sy, d.sz, Pr, d.f, d.cap, d.err, sm, S, &bar, uses, pe, vir,
                                     &B->ovf_force, ovf, g))
            continue;  // deferred to k_b_force_ovf
        pe = block_sum<double, BLOCK>(pe);
        vir = block_sum<double, BLOCK>(vir);
        if (threadIdx.x == 0) {
            const long slot = d.tpart_base + (g - d.tile_base);
            tpart[2 * slot] = pe;
            tpart[2 * slot + 1] = vir;
        }
    }
}

// tiles whose staging exceeds SRV_CAP, with SRV_BIG of shared memory (each CTA size
// takes the tiles of its systems)
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_b_force_ovf(const SysDesc* __restrict__ D, const BatchHdr* __restrict__ B,
                                                       LJP<float> Pr, double* __restrict__ tpart,
                                                       const long* __restrict__ ovf) {
    extern __shared__ __align__(128) unsigned char tile_raw[];
    float4* sm = reinterpret_cast<float4*>(tile_raw);
    __shared__ TileShM S;
    __shared__ unsigned long long bar;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    unsigned int uses = 0;
    const int nsys = B->nsys;
    const long tot = B->ovf_force;
    for (long q = blockIdx.x; q < tot; q += gridDim.x) {
        const long g = ovf[q];
        const int s = find_sys(D, nsys, g, 0);
        const SysDesc& d = D[s];
        if (d.block != BLOCK) continue;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        double pe = 0, vir = 0;
        b_force_tile_any<BLOCK>(d, g - d.tile_base, SRV_BIG_CAP, Pr, sm, S, &bar, uses, pe, vir);
        pe = block_sum<double, BLOCK>(pe);
        vir = block_sum<double, BLOCK>(vir);
        if (threadIdx.x == 0) {
            const long slot = d.tpart_base + (g - d.tile_base);
            tpart[2 * slot] = pe;
            tpart[2 * slot + 1] = vir;
        }
    }
}

__global__ void __launch_bounds__(CHUNK) k_b_kick(const SysDesc* __restrict__ D, const BatchHdr* __restrict__ B,
                                                  float half, double* __restrict__ kpart,
                                                  const unsigned int* __restrict__ phase) {
    const int nsys = B->nsys;
    const long tot = B->tot_chunks;
    for (long g = blockIdx.x; g < tot; g += gridDim.x) {
        const int s = find_sys(D, nsys, g, 1);
        const SysDesc& d = D[s];
        if (phase[d.slot] == 0) continue;
        const long c = g - d.chunk_base;
        const long i = c * CHUNK + threadIdx.x;
        double ke = 0;
        if (i < d.n_real) {
            const long cap = d.cap;
            float vx = d.v[i] + half * d.f[i];
            float vy = d.v[cap + i] + half * d.f[cap + i];
            float vz = d.v[2 * cap + i] + half * d.f[2 * cap + i];
            d.v[i] = vx;
            d.v[cap + i] = vy;
            d.v[2 * cap + i] = vz;
            ke = 0.5 * d.mass * ((double)vx * vx + (double)vy * vy + (double)vz * vz);
        }
        ke = block_sum<double, CHUNK>(ke);
        if (threadIdx.x == 0) kpart[d.kpart_base + c] = ke;
    }
}

// one block per system: E[step] = (KE, PE, virial, rebuilt) in a fixed order; a
// system whose first build and forces ran in this graph records nothing and steps
// from the next one
__global__ void __launch_bounds__(256) k_b_energy(const SysDesc* __restrict__ D, const BatchHdr* __restrict__ B,
                                                  const double* __restrict__ tpart, const double* __restrict__ kpart,
                                                  const unsigned int* __restrict__ flag,
                                                  unsigned int* __restrict__ phase) {
    const int s = blockIdx.x;
    if (s >= B->nsys) return;
    const SysDesc& d = D[s];
    if (phase[d.slot] == 0) {
        __syncthreads();
        if (threadIdx.x == 0) phase[d.slot] = 1;
        return;
    }
    double ke = 0, pe = 0, w = 0;
    for (long c = threadIdx.x; c < d.nchunk; c += 256) ke += kpart[d.kpart_base + c];
    for (long t = threadIdx.x; t < d.ntiles; t += 256) {
        pe += tpart[2 * (d.tpart_base + t)];
        w += tpart[2 * (d.tpart_base + t) + 1];
    }
    ke = block_sum<double, 256>(ke);
    pe = block_sum<double, 256>(pe);
    w = block_sum<double, 256>(w);
    if (threadIdx.x == 0) {
        const int st = *d.step;
        d.E[4 * st] = ke;
        d.E[4 * st + 1] = pe;
        d.E[4 * st + 2] = w;
        d.E[4 * st + 3] = (double)flag[d.slot];
        *d.step = st + 1;
    }
}

// ---------------------------------------------------------------------------
// batched rebuild of the flagged systems.  Each phase restates the arithmetic and
// the orders of the single-system path (mixed_to_positions + wrap_positions,
// cl_build + cl_reorder, ghost_generate, md_tiles, mixed_from_positions).

__global__ void __launch_bounds__(CHUNK) k_rb_zero(const SysDesc* __restrict__ D, const RbWork* __restrict__ W) {
    RB_LOOP(K_C)
    const long i = c * CHUNK + threadIdx.x;
    if (i <= d.ncell) {
        d.cntR[i] = 0;
        d.cntI[i] = 0;
    }
    RB_END
}

// offsets -> FP64 positions (first build: the submitted positions), periodic wrap,
// cell hash with warp-aggregated counts
__global__ void __launch_bounds__(CHUNK) k_rb_unpack(const SysDesc* __restrict__ D, const RbWork* __restrict__ W,
                                                     const unsigned int* __restrict__ phase) {
    RB_LOOP(K_P)
    const long i = c * CHUNK + threadIdx.x;
    const bool ok = i < d.n_real;
    const unsigned int act = __ballot_sync(0xffffffffu, ok);
    unsigned int bad = 0;
    if (ok) {
        double4 r;
        if (phase[d.slot] == 0) {
            r = ld4(d.pos, i);
        } else {
            float4 o = d.off[i];
            double cx, cy, cz;
            d.C.centre(__float_as_uint(o.w), cx, cy, cz);
            r = make_double4(cx + (double)o.x, cy + (double)o.y, cz + (double)o.z, 0.0);
        }
        r.x = periodic_l(r.x, d.L, 0.0);
        r.y = periodic_l(r.y, d.L, 0.0);
        r.z = periodic_l(r.z, d.L, 0.0);
        st4(d.pos, i, r);
        unsigned int cc = (unsigned int)d.G.cell(r.x, r.y, r.z, bad);
        d.cell_of[i] = cc;
        d.rank[i] = warp_agg_inc(d.cntR, cc, act);
    }
    if (bad) atomicOr(d.err, ERR_CELL_RANGE);
    RB_END
}

// per-system exclusive scans: 0 cntR -> csR (ncell + 1), 1 img_cnt -> img_start (n,
// total = image count), 2 cntI -> csI (ncell + 1)
template <int WHICH> struct ScanSel {
    static __device__ __forceinline__ const unsigned int* in(const SysDesc& d) {
        return WHICH == 0 ? d.cntR : (WHICH == 1 ? d.img_cnt : d.cntI);
    }
    static __device__ __forceinline__ unsigned int* out(const SysDesc& d) {
        return WHICH == 0 ? d.csR : (WHICH == 1 ? d.img_start : d.csI);
    }
    static __device__ __forceinline__ long len(const SysDesc& d) { return WHICH == 1 ? d.n_real : d.ncell + 1; }
    static constexpr int kind = WHICH == 1 ? K_QP : K_Q;
};

template <int WHICH>
__global__ void __launch_bounds__(CHUNK) k_rb_scan_sum(const SysDesc* __restrict__ D, const RbWork* __restrict__ W) {
    typedef ScanSel<WHICH> Sel;
    RB_LOOP(Sel::kind)
    const unsigned int* a = Sel::in(d);
    const long len = Sel::len(d);
    const long b = c * SCH + 4L * threadIdx.x;
    unsigned int v = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j)
        if (b + j < len) v += a[b + j];
    v = block_sum<unsigned int, CHUNK>(v);
    if (threadIdx.x == 0) d.spart[c] = v;
    RB_END
}

template <int WHICH>
__global__ void __launch_bounds__(CHUNK) k_rb_scan_mid(const SysDesc* __restrict__ D, const RbWork* __restrict__ W) {
    typedef ScanSel<WHICH> Sel;
    if ((int)blockIdx.x >= W->nflag) return;
    const SysDesc& d = D[W->sys[blockIdx.x]];
    const long len = Sel::len(d);
    const long np = (len + SCH - 1) / SCH;
    unsigned int carry = 0;
    for (long b = 0; b < np; b += CHUNK) {
        const long i = b + threadIdx.x;
        const unsigned int v = i < np ? d.spart[i] : 0u;
        unsigned int tot = 0;
        const unsigned int e = block_scan256(v, tot);
        if (i < np) d.spart[i] = carry + e;
        carry += tot;
    }
    if (WHICH == 1 && threadIdx.x == 0) {
        long m = carry;
        if (m > d.img_cap || d.n_real + m > d.cap) {
            atomicOr(d.err, ERR_IMG_OVERFLOW);
            m = min(d.img_cap, d.cap - d.n_real);
        }
        *d.n_img = (unsigned int)m;
    }
}

template <int WHICH>
__global__ void __launch_bounds__(CHUNK) k_rb_scan_apply(const SysDesc* __restrict__ D, const RbWork* __restrict__ W) {
    typedef ScanSel<WHICH> Sel;
    RB_LOOP(Sel::kind)
    const unsigned int* a = Sel::in(d);
    unsigned int* o = Sel::out(d);
    const long len = Sel::len(d);
    const long b = c * SCH + 4L * threadIdx.x;
    unsigned int e[4], sum = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        e[j] = b + j < len ? a[b + j] : 0u;
        sum += e[j];
    }
    unsigned int tot = 0;
    unsigned int run = d.spart[c] + block_scan256(sum, tot);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (b + j < len) o[b + j] = run;
        run += e[j];
    }
    RB_END
}

// slot inside the cell (unordered)
template <int IMG>
__global__ void __launch_bounds__(CHUNK) k_rb_scatter(const SysDesc* __restrict__ D, const RbWork* __restrict__ W) {
    RB_LOOP(IMG ? K_I : K_P)
    const long i = c * CHUNK + threadIdx.x;
    const long n = IMG ? (long)*d.n_img : d.n_real;
    const unsigned int* st = IMG ? d.csI : d.csR;
    if (i < n) d.sorted_tmp[st[d.cell_of[i]] + d.rank[i]] = (int)i;
    RB_END
}

// stable order inside every cell: one warp per cell orders its members by index
template <int IMG>
__global__ void __launch_bounds__(CHUNK) k_rb_stabilise(const SysDesc* __restrict__ D, const RbWork* __restrict__ W) {
    __shared__ int cell_sort_buf[CHUNK / 32][CELL_SORT_SMEM];
    RB_LOOP(K_W)
    const long cell = c * 8 + (threadIdx.x >> 5);
    if (cell < d.ncell) {
        const unsigned int* start = IMG ? d.csI : d.csR;
        const int* in = d.sorted_tmp;
        int* out = d.sorted;
        const unsigned int s0 = start[cell], e0 = start[cell + 1];
        warp_cell_order(in + s0, out + s0, e0 - s0, cell_sort_buf[threadIdx.x >> 5]);
    }
    RB_END
}

// reorder of the real particles into cell order: positions, ids, velocities
__global__ void __launch_bounds__(CHUNK) k_rb_gather(const SysDesc* __restrict__ D, const RbWork* __restrict__ W) {
    RB_LOOP(K_P)
    const long k = c * CHUNK + threadIdx.x;
    const long n = d.n_real;
    if (k < n) {
        const int j = d.sorted[k];
        d.scr_pos[k] = ld4(d.pos, j);
        d.scr_gid[k] = d.gid[j];
        d.scr_v[k] = d.v[j];
        d.scr_v[n + k] = d.v[d.cap + j];
        d.scr_v[2 * n + k] = d.v[2 * d.cap + j];
    }
    RB_END
}

// write back + periodic image count per particle (num_shift_ghost_each_part)
__global__ void __launch_bounds__(CHUNK) k_rb_put_count(const SysDesc* __restrict__ D, const RbWork* __restrict__ W) {
    __shared__ BoxSet<double> Bx;
    RB_LOOP(K_P)
    __syncthreads();
    for (int i = threadIdx.x; i < (int)(sizeof(BoxSet<double>) / 4); i += blockDim.x)
        reinterpret_cast<int*>(&Bx)[i] = reinterpret_cast<const int*>(d.boxes)[i];
    __syncthreads();
    const long k = c * CHUNK + threadIdx.x;
    const long n = d.n_real;
    if (k < n) {
        const double4 r = d.scr_pos[k];
        st4(d.pos, k, r);
        d.gid[k] = d.scr_gid[k];
        d.v[k] = d.scr_v[k];
        d.v[d.cap + k] = d.scr_v[n + k];
        d.v[2 * d.cap + k] = d.scr_v[2 * n + k];
        unsigned int cnt = 0;
        int old = -1;
        for (int i = 0; i < Bx.nb; ++i) {
            int s = Bx.sv[i];
            if (inside_np(Bx, i, r.x, r.y, r.z) && s != old) {
                old = s;
                cnt++;
            }
        }
        d.img_cnt[k] = cnt;
    }
    RB_END
}

// shift_ghost_each_part: image j of particle p goes to slot n + start[p] + j
__global__ void __launch_bounds__(CHUNK) k_rb_ghost_write(const SysDesc* __restrict__ D,
                                                          const RbWork* __restrict__ W) {
    __shared__ BoxSet<double> Bx;
    RB_LOOP(K_P)
    __syncthreads();
    for (int i = threadIdx.x; i < (int)(sizeof(BoxSet<double>) / 4); i += blockDim.x)
        reinterpret_cast<int*>(&Bx)[i] = reinterpret_cast<const int*>(d.boxes)[i];
    __syncthreads();
    const long p = c * CHUNK + threadIdx.x;
    const long n = d.n_real;
    if (p < n) {
        const double4 r = ld4(d.pos, p);
        long m = d.img_start[p];
        int old = -1;
        bool over = false;
        for (int i = 0; i < Bx.nb; ++i) {
            int s = Bx.sv[i];
            if (inside_np(Bx, i, r.x, r.y, r.z) && s != old) {
                old = s;
                if (m < d.img_cap && n + m < d.cap) {
                    double4 q;
                    q.x = r.x - d.shifts[3 * s];
                    q.y = r.y - d.shifts[3 * s + 1];
                    q.z = r.z - d.shifts[3 * s + 2];
                    q.w = r.w;
                    st4(d.pos, n + m, q);
                    d.gid[n + m] = d.gid[p];
                    d.img_src[m] = (int)p;
                    d.img_shift[m] = (unsigned char)s;
                } else {
                    over = true;
                }
                m++;
            }
        }
        if (over) atomicOr(d.err, ERR_IMG_OVERFLOW);
    }
    RB_END
}

// cell hash of the images
__global__ void __launch_bounds__(CHUNK) k_rb_hash_img(const SysDesc* __restrict__ D, const RbWork* __restrict__ W) {
    RB_LOOP(K_I)
    const long k = c * CHUNK + threadIdx.x;
    const bool ok = k < (long)*d.n_img;
    const unsigned int act = __ballot_sync(0xffffffffu, ok);
    unsigned int bad = 0;
    if (ok) {
        const double4 r = ld4(d.pos, d.n_real + k);
        unsigned int cc = (unsigned int)d.G.cell(r.x, r.y, r.z, bad);
        d.cell_of[k] = cc;
        d.rank[k] = warp_agg_inc(d.cntI, cc, act);
    }
    if (bad) atomicOr(d.err, ERR_CELL_RANGE);
    RB_END
}

__global__ void __launch_bounds__(CHUNK) k_rb_gather_img(const SysDesc* __restrict__ D,
                                                         const RbWork* __restrict__ W) {
    RB_LOOP(K_I)
    const long k = c * CHUNK + threadIdx.x;
    if (k < (long)*d.n_img) {
        const int j = d.sorted[k];
        d.scr_pos[k] = ld4(d.pos, d.n_real + j);
        d.scr_gid[k] = d.gid[d.n_real + j];
        d.scr_src[k] = d.img_src[j];
        d.scr_shf[k] = d.img_shift[j];
    }
    RB_END
}

__global__ void __launch_bounds__(CHUNK) k_rb_put_img(const SysDesc* __restrict__ D, const RbWork* __restrict__ W) {
    RB_LOOP(K_I)
    const long k = c * CHUNK + threadIdx.x;
    if (k < (long)*d.n_img) {
        st4(d.pos, d.n_real + k, d.scr_pos[k]);
        d.gid[d.n_real + k] = d.scr_gid[k];
        d.img_src[k] = d.scr_src[k];
        d.img_shift[k] = d.scr_shf[k];
    }
    RB_END
}

// FP32 staging copies of the list build and FP32 offsets of every particle
__global__ void __launch_bounds__(CHUNK) k_rb_offsets(const SysDesc* __restrict__ D, const RbWork* __restrict__ W) {
    RB_LOOP(K_A)
    const long k = c * CHUNK + threadIdx.x;
    unsigned int bad = 0;
    if (k < d.n_real + (long)*d.n_img) {
        const double4 r = ld4(d.pos, k);
        d.pos32[k] = make_float4((float)r.x, (float)r.y, (float)r.z, __int_as_float((int)k));
        unsigned int cc = (unsigned int)d.G.cell(r.x, r.y, r.z, bad);
        double cx, cy, cz;
        d.C.centre(cc, cx, cy, cz);
        d.off[k] = make_float4(d.C.qd(r.x - cx), d.C.qd(r.y - cy), d.C.qd(r.z - cz), __uint_as_float(cc));
    }
    if (bad) atomicOr(d.err, ERR_CELL_RANGE);
    RB_END
}

// offsets at the build (real) and the constant parts of the image offsets
__global__ void __launch_bounds__(CHUNK) k_rb_image_k(const SysDesc* __restrict__ D, const RbWork* __restrict__ W) {
    RB_LOOP(K_A)
    const long k = c * CHUNK + threadIdx.x;
    const long n = d.n_real;
    if (k < n) {
        d.offb[k] = d.off[k];
    } else if (k - n < (long)*d.n_img) {
        const long m = k - n;
        const int s = d.img_src[m];
        double4 xi = ld4(d.pos, n + m), xs = ld4(d.pos, s);
        double ci[3], cs[3];
        d.C.centre(__float_as_uint(d.off[n + m].w), ci[0], ci[1], ci[2]);
        d.C.centre(__float_as_uint(d.off[s].w), cs[0], cs[1], cs[2]);
        d.offK[m] = make_float4(d.C.qd((xi.x - ci[0]) - (xs.x - cs[0])), d.C.qd((xi.y - ci[1]) - (xs.y - cs[1])),
                                d.C.qd((xi.z - ci[2]) - (xs.z - cs[2])), 0.f);
    }
    RB_END
}

// tiled Verlet rows of the flagged systems (persistent CTAs, one mbarrier each).
// BIG = 0: every flagged tile, built one z-layer at a time in SRV_BSMEM; tiles
// with a layer beyond it (or more than 2 x TBLOCK domain particles) are appended
// to the overflow list; BIG = 1: the overflow list, whole tiles in SRV_BIG.
template <int BIG>
__global__ void __launch_bounds__(TBLOCK) k_rb_build(const SysDesc* __restrict__ D, const RbWork* __restrict__ W,
                                                     BatchHdr* __restrict__ B, long* __restrict__ ovf,
                                                     unsigned int* __restrict__ nn_max) {
    extern __shared__ __align__(128) unsigned char tile_raw[];
    float4* sm = reinterpret_cast<float4*>(tile_raw);
    __shared__ TileSh S;
    __shared__ unsigned int segb[18][TXMAX + 3];
    __shared__ unsigned long long bar;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    unsigned int parity = 0;
    const unsigned int cap = BIG ? SRV_BIG_CAP : SRV_BCAP;
    const long tot = BIG ? (long)B->ovf_build : W->tot[K_T];
    for (long q = blockIdx.x; q < tot; q += gridDim.x) {
        // generic-proxy reads of the previous tile are ordered before the next bulk copies
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        const long g = BIG ? ovf[q] : q;
        const int k = find_flagged(W, K_T, g);
        const SysDesc& d = D[W->sys[k]];
        const long c = g - W->base[K_T][k];
        tile_layout(d.tg, c, d.csR, d.csI, S);
        const unsigned int ib = S.cR[4][1], ie = S.cR[4][S.ncol - 2];
        if (ib == ie) continue;
        tile_segb(S, segb);
        if (!BIG) {
            unsigned int lmax = S.total - S.oR[6];
            lmax = max(lmax, S.oR[3] - S.oR[0]);
            lmax = max(lmax, S.oR[6] - S.oR[3]);
            if (lmax > cap || ie - ib > 2u * TBLOCK) {
                if (threadIdx.x == 0) ovf[atomicAdd(&B->ovf_build, 1u)] = g;
                continue;
            }
            if (!tile_rows_layers<double>(S, segb, d.pos32, d.pos32 + d.n_real, sm, cap, d.pos, d.r2, d.lo_thr,
                                          d.hi_thr, d.nbr, d.nn, d.tstride, d.max_nn, d.err, nn_max, &bar, parity))
                break;  // a bounded wait gave up (error bit set): the barrier phase is unknown
            continue;
        }
        const int st = tile_stage_bar<float>(d.pos32, d.pos32 + d.n_real, S, sm, cap, d.err, &bar, parity);
        if (st > 0) parity ^= 1u;
        if (st < 0) {
            // the tile does not fit (error bit set; the next tile may), or the bounded
            // wait gave up: its barrier phase cannot be tracked further, so stop
            if (S.total <= cap) break;
            continue;
        }
        tile_rows<double>(S, segb, sm, d.pos, d.r2, d.lo_thr, d.hi_thr, d.nbr, d.nn, d.tstride, d.max_nn, d.err,
                          nn_max);
    }
}

__global__ void k_srv_iota(int* __restrict__ g, long n) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        g[i] = (int)i;
}

}  // namespace pd

using namespace pd;

// ---------------------------------------------------------------------------
// launch shape of a system's force kernel: tile width (cells along x), lanes per
// particle, threads per CTA
struct SrvShape {
    int tx, lanes, block;
};

struct SrvSlot {
    pd_vd h = nullptr;
    pd_md md = nullptr;
    int vp = -1, fp = -1;
    long img_cap = 0;
    Buf cntI, cell_of, rank, sorted, sorted_tmp, spart, scr_pos, scr_gid, scr_v, scr_src, scr_shf, Edev, step;
    void release() {
        Buf* b[] = {&cntI, &cell_of, &rank, &sorted, &sorted_tmp, &spart, &scr_pos,
                    &scr_gid, &scr_v, &scr_src, &scr_shf, &Edev, &step};
        for (Buf* x : b) x->release();
        if (md) pd_md_destroy(md);
        if (h) pd_destroy(h);
        md = nullptr;
        h = nullptr;
    }
};

// A ring of pinned host memory (mapped for the device) whose regions are taken
// in order and freed at the front: a region freed out of order is kept until all
// older ones are freed.  take() returns nullptr when the ring has no room; the
// caller then falls back to host vectors.
struct PinnedFifo {
    struct Region {
        long ticket;
        size_t lo, hi;
        cudaEvent_t ev;  // work that reads the region (none: free once marked)
        bool done;
    };
    char* base = nullptr;
    const char* dev = nullptr;
    size_t bytes = 0;
    std::deque<Region> q;

    int create(size_t b) {
        bytes = b;
        void* d = nullptr;
        if (cudaMallocHost((void**)&base, b) != cudaSuccess || cudaHostGetDevicePointer(&d, base, 0) != cudaSuccess) {
            cudaGetLastError();
            return PD_ENOMEM;
        }
        dev = static_cast<const char*>(d);
        return PD_OK;
    }
    void destroy() {
        for (auto& g : q)
            if (g.ev) cudaEventDestroy(g.ev);
        q.clear();
        if (base) cudaFreeHost(base);
        base = nullptr;
    }
    // free the regions at the front that are marked and whose work has finished
    void trim(std::vector<cudaEvent_t>& ev_free) {
        while (!q.empty()) {
            Region& f = q.front();
            if (!f.done) break;
            if (f.ev && cudaEventQuery(f.ev) != cudaSuccess) {
                cudaGetLastError();  // cudaErrorNotReady
                break;
            }
            if (f.ev) ev_free.push_back(f.ev);
            q.pop_front();
        }
    }
    // a region of `need` bytes after the newest one (wrapping to the start), or
    // nullptr when it would reach the oldest region still held
    char* take(long ticket, size_t need, long& lo_out, std::vector<cudaEvent_t>& ev_free) {
        need = (need + 255) & ~(size_t)255;
        trim(ev_free);
        size_t lo = 0;
        if (!q.empty()) {
            const size_t T = q.front().lo, H = q.back().hi;
            const bool wrapped = q.back().lo < T;
            if (!wrapped && H + need <= bytes) lo = H;
            else if (!wrapped && need <= T) lo = 0;
            else if (wrapped && H + need <= T) lo = H;
            else return nullptr;
        } else if (need > bytes) {
            return nullptr;
        }
        q.push_back({ticket, lo, lo + need, nullptr, false});
        lo_out = (long)lo;
        return base + lo;
    }
    Region* find(long ticket) {
        for (auto& g : q)
            if (g.ticket == ticket) return &g;
        return nullptr;
    }
};

struct SrvReq {
    long ticket = 0;
    long n = 0;
    double L = 0;
    int steps = 0;
    int state = 0;  // 0 queued, 1 running, 2 done, 3 failed
    std::vector<double> x, v, xo, E;  // x, v: the submitted state when it is not in the inbox
    long in_lo = -1;                   // offset of the submitted state in the pinned inbox, or -1
    long out_lo = -1;                  // offset of the result in the pinned outbox, or -1 (xo, E)
    double t_submit = 0, t_admit = 0, t_done = 0;
    size_t bytes = 0;
    int slot = -1;
    int bucket = 0;
    int done_steps = 0;
    bool first = true;  // the next step graph runs its first build and forces
};

// Copies of the submitted arrays into pinned memory: one core copies at about
// 6 GB/s, so a submission of a megabyte or more is cut into pieces of at least
// 512 KB that the caller and up to three workers (no more than the cores beside
// the caller's) copy.  The workers start at the first such submission and live
// as long as the server; if they cannot be started the caller copies everything.
struct CopyJob {
    char* dst;
    const char* src;
    size_t bytes;
};

struct CopyPool {
    std::vector<std::thread> workers;
    std::mutex mu;
    std::condition_variable wake, done;
    std::vector<CopyJob> pieces;
    size_t next = 0, left = 0;
    bool stop = false, tried = false;

    ~CopyPool() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        wake.notify_all();
        for (auto& t : workers) t.join();
    }
    // take and copy pieces until none is left
    void drain() {
        for (;;) {
            CopyJob c;
            {
                std::lock_guard<std::mutex> lk(mu);
                if (next >= pieces.size()) return;
                c = pieces[next++];
            }
            memcpy(c.dst, c.src, c.bytes);
            std::lock_guard<std::mutex> lk(mu);
            if (--left == 0) done.notify_all();
        }
    }
    void worker() {
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu);
                wake.wait(lk, [this] { return stop || next < pieces.size(); });
                if (stop) return;
            }
            drain();
        }
    }
    void copy(const CopyJob* jobs, int nj) {
        size_t total = 0;
        for (int j = 0; j < nj; ++j) total += jobs[j].bytes;
        if (total < ((size_t)1 << 20)) {
            for (int j = 0; j < nj; ++j) memcpy(jobs[j].dst, jobs[j].src, jobs[j].bytes);
            return;
        }
        if (!tried) {
            tried = true;
            try {
                const unsigned hw = std::thread::hardware_concurrency();
                const int nw = hw == 0 ? 3 : (int)std::min(3u, hw > 1 ? hw - 1 : 0u);
                for (int k = 0; k < nw; ++k) workers.emplace_back([this] { worker(); });
            } catch (const std::system_error&) {
            }
        }
        const size_t T = std::min<size_t>(workers.size() + 1, std::max<size_t>(1, total / ((size_t)512 << 10)));
        const size_t want = (total + T - 1) / T;
        {
            std::lock_guard<std::mutex> lk(mu);
            pieces.clear();
            for (int j = 0; j < nj; ++j)
                for (size_t a = 0; a < jobs[j].bytes; a += want)
                    pieces.push_back({jobs[j].dst + a, jobs[j].src + a, std::min(want, jobs[j].bytes - a)});
            next = 0;
            left = pieces.size();
        }
        wake.notify_all();
        drain();
        std::unique_lock<std::mutex> lk(mu);
        done.wait(lk, [this] { return left == 0; });
    }
};

struct pd_srv_s {
    long budget = 0;
    int max_slots = 0;
    pd_lj_params_t lj;
    double dt = 0.005, skin = 0.3;
    std::chrono::steady_clock::time_point t0;
    long next_ticket = 1;
    std::map<long, std::unique_ptr<SrvReq>> reqs;
    std::deque<long> queue;
    std::vector<SrvReq*> active;
    std::vector<std::pair<SrvReq*, bool>> finished;  // (system, failed), retired by the next tick
    std::vector<long> completed;                      // tickets finished since the last poll
    std::vector<SrvSlot> slots;
    size_t used = 0;
    // device tables (fixed capacity: graph-invariant pointers)
    Buf desc, hdr, maxd2, errs, flags, phase, work, nnmax, tpart, kpart, ovf_f, ovf_b;
    long tpart_cap = 0, kpart_cap = 0;
    std::vector<SysDesc> hdesc;
    BatchHdr hhdr;
    unsigned int* flags_h = nullptr;  // pinned: rebuild flag and error bits per slot after each step
    unsigned int* errs_h = nullptr;
    cudaStream_t st = nullptr;     // step graphs
    cudaStream_t as = nullptr;     // admission and retirement, overlapping the running step graph
    cudaMemPool_t pool = nullptr;  // device memory of the slots (stream-ordered on `as`)
    cudaEvent_t ev_adm = nullptr;  // end of the last admissions on `as`
    // pinned staging: a ring for the admissions' uploads (a region is reused once
    // the event recorded after its copies has completed) and a buffer for downloads,
    // both 1/64 of the budget within [8 MB, 256 MB]
    char* up = nullptr;
    size_t up_bytes = 0, up_head = 0;
    struct UpUse {
        size_t lo, hi;
        cudaEvent_t ev;
    };
    std::deque<UpUse> up_use;
    std::vector<cudaEvent_t> ev_free;
    char* down = nullptr;
    size_t down_bytes = 0;
    // pinned inbox: a submitted state is copied here once when there is room and
    // read by the admission's upload kernel; regions are taken in submission order
    // and freed in admission order, the same FIFO order
    PinnedFifo inbox;
    // pinned outbox: a finished system's positions and energies are copied here by
    // the GPU and read by pd_srv_result; regions are freed at pd_srv_release
    PinnedFifo outbox;
    std::unique_ptr<CopyPool> copier;  // submissions' copies into the inbox
    bool adm_pending = false;
    cudaGraphExec_t gstep[4] = {nullptr, nullptr, nullptr, nullptr};  // 1, 2, 4, 8 steps per launch
    bool dirty = true;
    // autotuner: size bucket -> tile width, lanes per particle, CTA size of the force kernel
    bool autotune = true;
    SrvShape fixed{0, 2, pd::FBLOCK_T};
    std::map<int, SrvShape> tuned;
    // statistics
    long particle_steps = 0, systems_done = 0, steps_run = 0, rebuilds = 0;
    double tune_ms = 0;
    double ms[4] = {0, 0, 0, 0};  // admit, of which slot reset, step, retire
};

namespace pd {

static double now_s(pd_srv s) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - s->t0).count();
}

static size_t estimate_bytes(long n) {
    // positions (FP64 record + FP32 offsets + staging copies), images (~30% for
    // mid-size boxes), FP32 velocity / force, rows of ~100 16-bit entries, scratch
    return (size_t)n * 700 + ((size_t)8 << 20);
}

// periodic images expected for n particles spread over a cubic box of side L, ghost g
static long image_estimate(long n, double L, double g) {
    double r = ((L + 2 * g) * (L + 2 * g) * (L + 2 * g)) / (L * L * L) - 1.0;
    return (long)(n * r);
}

static void fill_desc(pd_srv s, SrvReq* r, SysDesc& d) {
    SrvSlot& sl = s->slots[r->slot];
    pd_vd h = sl.h;
    pd_md md = sl.md;
    pd_cl cl = md->vl->cl;
    memset(&d, 0, sizeof(d));
    d.off = md->off.as<float4>();
    d.offb = md->offb.as<float4>();
    d.offK = md->offK.as<float4>();
    d.pos = (double4*)h->pos;
    d.gid = h->gid;
    d.img_src = h->img_src.as<int>();
    d.img_shift = h->img_shift.as<unsigned char>();
    d.v = (float*)h->props[sl.vp].d;
    d.f = (float*)h->props[sl.fp].d;
    d.cap = h->cap;
    d.n_real = h->n_real;
    d.img_cap = sl.img_cap;
    d.ncell = cl->ncells;
    d.n_img = &h->ctrl->n_img;
    for (int k = 0; k < 3; ++k) {
        d.G.lo[k] = cl->box_lo[k];
        d.G.sp[k] = cl->spacing[k];
        d.G.gs[k] = cl->gs[k];
    }
    d.G.pad = cl->pad;
    d.C = mixed_cell_geom(cl);
    d.L = r->L;
    d.tg = md->tg;
    d.csR = md->csR.as<unsigned int>();
    d.csI = md->csI.as<unsigned int>();
    d.nbr = md->tnbr.as<unsigned int>();
    d.nn = md->tnn.as<int>();
    d.tstride = md->tstride;
    d.max_nn = md->tmax_nn;
    d.lanes = md->tile_p;
    d.block = md->tile_block;
    d.sx = (float)d.C.sp[0];  // exact: multiples of the quantum
    d.sy = (float)d.C.sp[1];
    d.sz = (float)d.C.sp[2];
    const double rl = md->vl->r_cut;
    const double band = fp32_band(h, rl);
    d.lo_thr = (float)(rl * rl - band);
    d.hi_thr = (float)(rl * rl + band);
    d.r2 = rl * rl;
    d.boxes = h->boxes.as<BoxSet<double>>();
    d.shifts = h->shifts.as<double>();
    d.cntR = cl->cell_cnt.as<unsigned int>();
    d.cntI = sl.cntI.as<unsigned int>();
    d.cell_of = sl.cell_of.as<unsigned int>();
    d.rank = sl.rank.as<unsigned int>();
    d.img_cnt = h->img_cnt.as<unsigned int>();
    d.img_start = h->img_start.as<unsigned int>();
    d.spart = sl.spart.as<unsigned int>();
    d.sorted = sl.sorted.as<int>();
    d.sorted_tmp = sl.sorted_tmp.as<int>();
    d.scr_pos = sl.scr_pos.as<double4>();
    d.scr_gid = sl.scr_gid.as<int>();
    d.scr_v = sl.scr_v.as<float>();
    d.scr_src = sl.scr_src.as<int>();
    d.scr_shf = sl.scr_shf.as<unsigned char>();
    d.pos32 = md->pos32.as<float4>();
    d.ntiles = md->ntiles;
    d.nchunk = (h->n_real + CHUNK - 1) / CHUNK;
    d.nimg_chunk = (sl.img_cap + CHUNK - 1) / CHUNK;
    const long n = h->n_real, nc = cl->ncells;
    d.cnt[K_P] = (n + CHUNK - 1) / CHUNK;
    d.cnt[K_C] = (nc + 1 + CHUNK - 1) / CHUNK;
    d.cnt[K_Q] = (nc + 1 + SCH - 1) / SCH;
    d.cnt[K_QP] = (n + SCH - 1) / SCH;
    d.cnt[K_I] = (sl.img_cap + CHUNK - 1) / CHUNK;
    d.cnt[K_A] = (n + sl.img_cap + CHUNK - 1) / CHUNK;
    d.cnt[K_T] = md->ntiles;
    d.cnt[K_W] = (nc + 7) / 8;
    d.err = s->errs.as<unsigned int>() + r->slot;
    d.E = sl.Edev.as<double>();
    d.step = sl.step.as<int>();
    d.mass = md->mp.mass;
    d.slot = r->slot;
}

// rebuild the descriptor table, prefixes and partial-buffer layout
static int upload_tables(pd_srv s) {
    int ns = (int)s->active.size();
    s->hdesc.resize(ns);
    long tb = 0, cb = 0, ib = 0, tp = 0, kp = 0;
    // the systems in order of their force kernel's shape group (each group's tiles
    // contiguous), in admission order within a group
    std::vector<SrvReq*> order;
    for (int grp = 0; grp < NSHAPE; ++grp)
        for (SrvReq* r : s->active) {
            const pd_md m = s->slots[r->slot].md;
            if (shape_group(m->tile_p, m->tile_block) == grp) order.push_back(r);
        }
    for (int grp = 0; grp <= NSHAPE; ++grp) s->hhdr.grp[grp] = 0;
    for (int k = 0; k < ns; ++k) {
        SysDesc& d = s->hdesc[k];
        fill_desc(s, order[k], d);
        for (int grp = shape_group(d.lanes, d.block) + 1; grp <= NSHAPE; ++grp) s->hhdr.grp[grp] = tb + d.ntiles;
        d.tile_base = tb;
        d.chunk_base = cb;
        d.img_base = ib;
        d.tpart_base = tp;
        d.kpart_base = kp;
        tb += d.ntiles;
        cb += d.nchunk;
        ib += d.nimg_chunk;
        tp += d.ntiles;
        kp += d.nchunk;
    }
    if (tp > s->tpart_cap || kp > s->kpart_cap) {
        set_error("serving: partial buffers too small (%ld tiles, %ld chunks)", tp, kp);
        return PD_EOVERFLOW;
    }
    s->hhdr.nsys = ns;
    s->hhdr.tot_tiles = tb;
    s->hhdr.tot_chunks = cb;
    s->hhdr.tot_img = ib;
    for (int grp = 0; grp < NSHAPE; ++grp) s->hhdr.grp_ctr[grp] = 0;
    if (ns) PD_CUDA(cudaMemcpyAsync(s->desc.p, s->hdesc.data(), sizeof(SysDesc) * ns, cudaMemcpyHostToDevice, s->st));
    PD_CUDA(cudaMemcpyAsync(s->hdr.p, &s->hhdr, sizeof(BatchHdr), cudaMemcpyHostToDevice, s->st));
    PD_CUDA(cudaStreamSynchronize(s->st));  // host staging vectors are reused
    s->dirty = false;
    return PD_OK;
}

static constexpr int GRAPH_KERNELS = 38;  // kernel nodes per step of the step graphs

// the step graphs: 2^lk velocity-Verlet steps of every active system per launch
static int capture_graph(pd_srv s, int lk) {
    float half = (float)(0.5 * s->dt / 1.0), dt = (float)s->dt;
    LJP<float> P{};
    P.eps24 = (float)(24.0 * s->lj.eps);
    P.eps4 = (float)(4.0 * s->lj.eps);
    P.sig2 = (float)(s->lj.sigma * s->lj.sigma);
    mixed_cutoff(s->lj, P);
#define PD_SRV_FORCE_ATTR(L, BL) \
    PD_CUDA(cudaFuncSetAttribute(k_b_force<L, BL>, cudaFuncAttributeMaxDynamicSharedMemorySize, SRV_SMEM));
    PD_SRV_FORCE_ATTR(1, FBLOCK_T)
    PD_SRV_FORCE_ATTR(2, FBLOCK_T)
    PD_SRV_FORCE_ATTR(4, FBLOCK_T)
    PD_SRV_FORCE_ATTR(1, FBLOCK_T / 2)
    PD_SRV_FORCE_ATTR(2, FBLOCK_T / 2)
    PD_SRV_FORCE_ATTR(4, FBLOCK_T / 2)
#undef PD_SRV_FORCE_ATTR
    PD_CUDA(cudaFuncSetAttribute(k_rb_build<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, SRV_BSMEM));
    PD_CUDA(cudaFuncSetAttribute(k_b_force_ovf<FBLOCK_T>, cudaFuncAttributeMaxDynamicSharedMemorySize, SRV_BIG));
    PD_CUDA(cudaFuncSetAttribute(k_b_force_ovf<FBLOCK_T / 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, SRV_BIG));
    PD_CUDA(cudaFuncSetAttribute(k_rb_build<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, SRV_BIG));
    int sms = 148, dev = 0, per = 1, per2 = 1, perb = 1;
    PD_CUDA(cudaGetDevice(&dev));
    PD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    PD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_b_force<2, FBLOCK_T>, FBLOCK_T, SRV_SMEM));
    PD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per2, k_b_force<2, FBLOCK_T / 2>, FBLOCK_T / 2, SRV_SMEM));
    PD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perb, k_rb_build<0>, TBLOCK, SRV_BSMEM));
    const int gf = sms * std::max(per, 1), gf2 = sms * std::max(per2, 1), gb = sms * std::max(perb, 1), gc = sms * 8;
    const SysDesc* D = s->desc.as<SysDesc>();
    BatchHdr* B = s->hdr.as<BatchHdr>();
    RbWork* W = s->work.as<RbWork>();
    unsigned long long* md2 = s->maxd2.as<unsigned long long>();
    unsigned int* fl = s->flags.as<unsigned int>();
    const double lim2 = 0.25 * s->skin * s->skin;
    const int always = s->skin <= 0 ? 1 : 0;
    const int M = s->max_slots;
    cudaGraph_t g = nullptr;
    cudaStream_t st = s->st;
    PD_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    for (int step = 0; step < (1 << lk); ++step) {
    cudaMemsetAsync(md2, 0, sizeof(unsigned long long) * M, st);
    cudaMemsetAsync(&B->ovf_force, 0, 2 * sizeof(unsigned int), st);  // ovf_force, ovf_build
    cudaMemsetAsync(B->grp_ctr, 0, sizeof(B->grp_ctr), st);
    unsigned int* ph = s->phase.as<unsigned int>();
    k_b_kick_drift<<<gc, CHUNK, 0, st>>>(D, B, half, dt, md2, ph);
    k_b_decide<<<1, 1024, 0, st>>>(D, B, md2, lim2, always, fl, ph, W);
    // batched rebuild of the flagged systems
    k_rb_zero<<<gc, CHUNK, 0, st>>>(D, W);
    k_rb_unpack<<<gc, CHUNK, 0, st>>>(D, W, ph);
    k_rb_scan_sum<0><<<gc, CHUNK, 0, st>>>(D, W);
    k_rb_scan_mid<0><<<M, CHUNK, 0, st>>>(D, W);
    k_rb_scan_apply<0><<<gc, CHUNK, 0, st>>>(D, W);
    k_rb_scatter<0><<<gc, CHUNK, 0, st>>>(D, W);
    k_rb_stabilise<0><<<gc, CHUNK, 0, st>>>(D, W);
    k_rb_gather<<<gc, CHUNK, 0, st>>>(D, W);
    k_rb_put_count<<<gc, CHUNK, 0, st>>>(D, W);
    k_rb_scan_sum<1><<<gc, CHUNK, 0, st>>>(D, W);
    k_rb_scan_mid<1><<<M, CHUNK, 0, st>>>(D, W);
    k_rb_scan_apply<1><<<gc, CHUNK, 0, st>>>(D, W);
    k_rb_ghost_write<<<gc, CHUNK, 0, st>>>(D, W);
    k_rb_hash_img<<<gc, CHUNK, 0, st>>>(D, W);
    k_rb_scan_sum<2><<<gc, CHUNK, 0, st>>>(D, W);
    k_rb_scan_mid<2><<<M, CHUNK, 0, st>>>(D, W);
    k_rb_scan_apply<2><<<gc, CHUNK, 0, st>>>(D, W);
    k_rb_scatter<1><<<gc, CHUNK, 0, st>>>(D, W);
    k_rb_stabilise<1><<<gc, CHUNK, 0, st>>>(D, W);
    k_rb_gather_img<<<gc, CHUNK, 0, st>>>(D, W);
    k_rb_put_img<<<gc, CHUNK, 0, st>>>(D, W);
    k_rb_offsets<<<gc, CHUNK, 0, st>>>(D, W);
    k_rb_image_k<<<gc, CHUNK, 0, st>>>(D, W);
    k_rb_build<0><<<gb, TBLOCK, SRV_BSMEM, st>>>(D, W, B, s->ovf_b.as<long>(), s->nnmax.as<unsigned int>());
    k_rb_build<1><<<sms, TBLOCK, SRV_BIG, st>>>(D, W, B, s->ovf_b.as<long>(), s->nnmax.as<unsigned int>());
    // step of every system
    k_b_replay<<<gc, CHUNK, 0, st>>>(D, B, fl);
    // one persistent force kernel per shape group (a group without systems returns at once)
    k_b_force<1, FBLOCK_T><<<gf, FBLOCK_T, SRV_SMEM, st>>>(D, B, P, s->tpart.as<double>(), s->ovf_f.as<long>());
    k_b_force<2, FBLOCK_T><<<gf, FBLOCK_T, SRV_SMEM, st>>>(D, B, P, s->tpart.as<double>(), s->ovf_f.as<long>());
    k_b_force<4, FBLOCK_T><<<gf, FBLOCK_T, SRV_SMEM, st>>>(D, B, P, s->tpart.as<double>(), s->ovf_f.as<long>());
    k_b_force<1, FBLOCK_T / 2><<<gf2, FBLOCK_T / 2, SRV_SMEM, st>>>(D, B, P, s->tpart.as<double>(), s->ovf_f.as<long>());
    k_b_force<2, FBLOCK_T / 2><<<gf2, FBLOCK_T / 2, SRV_SMEM, st>>>(D, B, P, s->tpart.as<double>(), s->ovf_f.as<long>());
    k_b_force<4, FBLOCK_T / 2><<<gf2, FBLOCK_T / 2, SRV_SMEM, st>>>(D, B, P, s->tpart.as<double>(), s->ovf_f.as<long>());
    k_b_force_ovf<FBLOCK_T><<<sms, FBLOCK_T, SRV_BIG, st>>>(D, B, P, s->tpart.as<double>(), s->ovf_f.as<long>());
    k_b_force_ovf<FBLOCK_T / 2><<<sms, FBLOCK_T / 2, SRV_BIG, st>>>(D, B, P, s->tpart.as<double>(),
                                                                   s->ovf_f.as<long>());
    k_b_kick<<<gc, CHUNK, 0, st>>>(D, B, half, s->kpart.as<double>(), ph);
    k_b_energy<<<M, 256, 0, st>>>(D, B, s->tpart.as<double>(), s->kpart.as<double>(), fl, ph);
    }
    cudaMemcpyAsync(s->flags_h, fl, sizeof(unsigned int) * M, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(s->errs_h, s->errs.p, sizeof(unsigned int) * M, cudaMemcpyDeviceToHost, st);
    cudaError_t ce = cudaStreamEndCapture(st, &g);
    if (ce != cudaSuccess) {
        set_error("serving: graph capture failed: %s", cudaGetErrorString(ce));
        return PD_ECUDA;
    }
    ce = cudaGraphInstantiate(&s->gstep[lk], g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) {
        set_error("serving: graph instantiation failed: %s", cudaGetErrorString(ce));
        return PD_ECUDA;
    }
    return PD_OK;
}

// grow a slot vector's particle capacity without keeping its contents (a new
// system is loaded next): stream-ordered frees and allocations, no host wait
static int slot_capacity(pd_vd h, long need) {
    if (need <= h->cap) return PD_OK;
    long ncap = need + need / 4 + 1024;
    dev_free(h->pos);
    dev_free(h->gid);
    h->pos = nullptr;
    h->gid = nullptr;
    for (Prop& P : h->props) {
        dev_free(P.d);
        P.d = nullptr;
    }
    h->cap = 0;
    PD_CUDA(dev_alloc(&h->pos, (size_t)ncap * h->pos_bytes));
    PD_CUDA(dev_alloc((void**)&h->gid, sizeof(int) * ncap));
    for (Prop& P : h->props) PD_CUDA(dev_alloc((void**)&P.d, (size_t)P.esize * P.ncomp * ncap));
    h->cap = ncap;
    h->epoch++;
    return PD_OK;
}

// (re)initialise a slot's containers for a system of n particles in a box of side L
static int slot_reset(pd_srv s, SrvSlot& sl, SrvReq* r, const SrvShape& shape) {
    const double rl = s->lj.r_cut + s->skin;
    if (!sl.h) {
        double lo[3] = {0, 0, 0}, hi[3] = {r->L, r->L, r->L};
        int bc[3] = {PD_PERIODIC, PD_PERIODIC, PD_PERIODIC};
        double g[3] = {rl, rl, rl};
        PD_TRY(pd_create(3, PD_F64, 0, lo, hi, bc, g, 0, &sl.h));  // sized below, on the server's stream
        PD_TRY(pd_add_prop(sl.h, PD_F32, 3, &sl.vp));
        PD_TRY(pd_add_prop(sl.h, PD_F32, 3, &sl.fp));
        pd_md_params_t mp;
        memset(&mp, 0, sizeof(mp));
        mp.dt = s->dt;
        mp.mass = 1.0;
        mp.skin = s->skin;
        mp.vel_prop = sl.vp;
        mp.force_prop = sl.fp;
        mp.precision = PD_PREC_MIXED;
        PD_TRY(pd_md_create(sl.h, &s->lj, &mp, &sl.md));
        sl.md->swap_reorder = false;  // the slot tables keep the vector's device pointers
    } else {
        pd_vd h = sl.h;
        pd_md md = sl.md;
        for (int d = 0; d < 3; ++d) {
            h->lo[d] = 0.0;
            h->hi[d] = r->L;
        }
        h->nbox = 0;  // the ghost boxes of the new box are uploaded by the first build
        h->n_img = 0;
        PD_CUDA(cudaMemsetAsync(h->ctrl, 0, sizeof(Ctrl), s->as));
        memset(h->ctrl_h, 0, sizeof(Ctrl));
        PD_TRY(cl_geometry(md->vl->cl, h, rl, 1.013, 1));
        mixed_set_quantum(md->vl->cl, s->skin);
        md->ready = false;
        md->steps = 0;
        md->builds = 0;
        md->off_valid = false;
        md->tiles_active = false;
        md->tmax_nn = 0;
        md->nblk = force_blocks(r->n);
        PD_TRY(md->fpart.ensure(sizeof(double) * 2 * md->nblk));
        PD_TRY(md->kpart.ensure(sizeof(double) * md->nblk));
        PD_TRY(md->xb.ensure((size_t)r->n * h->pos_bytes));
    }
    sl.md->tile_tx = shape.tx;
    sl.md->tile_p = shape.lanes;
    sl.md->tile_block = shape.block;
    // capacities for the batched rebuilds, reserved before the first build so that
    // the buffers it fills are not reallocated afterwards
    sl.img_cap = (long)(1.3 * image_estimate(r->n, r->L, rl)) + 2048;
    pd_vd h = sl.h;
    pd_md md = sl.md;
    PD_TRY(slot_capacity(h, r->n + sl.img_cap + 1));
    h->n_real = h->n_total = r->n;
    h->img_valid = false;
    h->epoch++;
    pd::launch(k_srv_iota, grid_for(r->n, CHUNK), CHUNK, 0, s->as, h->gid, r->n);
    PD_LAUNCH_CHECK();
    PD_TRY(md->off.ensure(sizeof(float4) * (size_t)h->cap));
    PD_TRY(md->offK.ensure(sizeof(float4) * (size_t)sl.img_cap));
    PD_TRY(md->pos32.ensure(sizeof(float4) * (size_t)h->cap));
    PD_TRY(h->img_src.ensure(sizeof(int) * (size_t)sl.img_cap));
    PD_TRY(h->img_shift.ensure((size_t)sl.img_cap));
    return PD_OK;
}

// scratch of the batched rebuild, from the slot's geometry after the first build
static int slot_scratch(pd_srv s, SrvSlot& sl, SrvReq* r) {
    pd_vd h = sl.h;
    pd_md md = sl.md;
    pd_cl cl = md->vl->cl;
    const long n = r->n, nc = cl->ncells, m = std::max(n, sl.img_cap);
    PD_TRY(cl->cell_cnt.ensure(sizeof(unsigned int) * (nc + 1)));
    PD_TRY(sl.cntI.ensure(sizeof(unsigned int) * (nc + 1)));
    PD_TRY(sl.cell_of.ensure(sizeof(unsigned int) * m));
    PD_TRY(sl.rank.ensure(sizeof(unsigned int) * m));
    PD_TRY(sl.sorted.ensure(sizeof(int) * m));
    PD_TRY(sl.sorted_tmp.ensure(sizeof(int) * m));
    PD_TRY(sl.spart.ensure(sizeof(unsigned int) * (std::max(nc + 1, n) / SCH + 2)));
    PD_TRY(sl.scr_pos.ensure(sizeof(double4) * m));
    PD_TRY(sl.scr_gid.ensure(sizeof(int) * m));
    PD_TRY(sl.scr_v.ensure(sizeof(float) * 3 * n));
    PD_TRY(sl.scr_src.ensure(sizeof(int) * sl.img_cap));
    PD_TRY(sl.scr_shf.ensure((size_t)sl.img_cap));
    PD_TRY(h->img_cnt.ensure(sizeof(unsigned int) * (n + 1)));
    PD_TRY(h->img_start.ensure(sizeof(unsigned int) * (n + 1)));
    PD_TRY(sl.Edev.ensure(sizeof(double) * 4 * (r->steps > 0 ? r->steps : 1)));
    PD_TRY(sl.step.ensure(sizeof(int)));
    PD_CUDA(cudaMemsetAsync(sl.step.p, 0, sizeof(int), s->as));
    PD_CUDA(cudaMemsetAsync(s->errs.as<unsigned int>() + r->slot, 0, sizeof(unsigned int), s->as));
    return PD_OK;
}

// the admission of `r` has launched everything that reads its inbox region: the
// region is freed once the work queued so far on the admission stream is done
static void inbox_release(pd_srv s, SrvReq* r) {
    if (r->in_lo < 0) return;
    if (PinnedFifo::Region* g = s->inbox.find(r->ticket)) {
        cudaEvent_t ev = nullptr;
        if (!s->ev_free.empty()) {
            ev = s->ev_free.back();
            s->ev_free.pop_back();
        } else if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
            ev = nullptr;
        }
        if (ev && cudaEventRecord(ev, s->as) != cudaSuccess) {
            s->ev_free.push_back(ev);
            ev = nullptr;
        }
        if (!ev) cudaStreamSynchronize(s->as);  // no event: wait here instead
        cudaGetLastError();
        g->ev = ev;
        g->done = true;
    }
    r->in_lo = -1;
}

// a region of `need` bytes of the upload ring, after the copies that last used it
static char* ring_take(pd_srv s, size_t need, size_t& lo_out) {
    need = (need + 255) & ~(size_t)255;
    if (need > s->up_bytes) return nullptr;
    if (s->up_head + need > s->up_bytes) s->up_head = 0;
    const size_t lo = s->up_head, hi = lo + need;
    for (auto it = s->up_use.begin(); it != s->up_use.end();) {
        const bool overlap = it->lo < hi && lo < it->hi;
        if (overlap || cudaEventQuery(it->ev) == cudaSuccess) {
            if (overlap) cudaEventSynchronize(it->ev);
            s->ev_free.push_back(it->ev);
            it = s->up_use.erase(it);
        } else {
            ++it;
        }
    }
    cudaGetLastError();  // a query of an unfinished event reports cudaErrorNotReady
    s->up_head = hi;
    lo_out = lo;
    return s->up + lo;
}

static int ring_mark(pd_srv s, size_t lo, size_t need) {
    need = (need + 255) & ~(size_t)255;
    cudaEvent_t ev = nullptr;
    if (!s->ev_free.empty()) {
        ev = s->ev_free.back();
        s->ev_free.pop_back();
    } else {
        PD_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    }
    PD_CUDA(cudaEventRecord(ev, s->as));
    s->up_use.push_back({lo, lo + need, ev});
    return PD_OK;
}

// staging layout: ghost boxes, shift vectors, positions and velocities as submitted
static size_t stage_off_shifts() { return (sizeof(BoxSet<double>) + 63) & ~(size_t)63; }
static size_t stage_off_pos() { return (stage_off_shifts() + 81 * sizeof(double) + 63) & ~(size_t)63; }

// the submitted state read from pinned host memory (x, v: n x,y,z triples) into
// the slot: FP64 position records and FP32 velocity components (stride cap);
// each block stages its 256 triples through shared memory so the host reads
// are contiguous
__global__ void __launch_bounds__(256) k_srv_unpack(const double* __restrict__ x, const double* __restrict__ v, long n,
                                                    double4* __restrict__ pos, float* __restrict__ V, long cap) {
    __shared__ double sx[3 * 256], sv[3 * 256];
    for (long base = (long)blockIdx.x * 256; base < n; base += (long)gridDim.x * 256) {
        const int m = (int)min(256L, n - base);
        for (int j = threadIdx.x; j < 3 * m; j += 256) {
            sx[j] = x[3 * base + j];
            sv[j] = v[3 * base + j];
        }
        __syncthreads();
        const int t = threadIdx.x;
        if (t < m) {
            pos[base + t] = make_double4(sx[3 * t], sx[3 * t + 1], sx[3 * t + 2], 0.0);
            V[base + t] = (float)sv[3 * t];
            V[cap + base + t] = (float)sv[3 * t + 1];
            V[2 * cap + base + t] = (float)sv[3 * t + 2];
        }
        __syncthreads();
    }
}

// upload the submitted state and the ghost boxes of the box, stream-ordered on the
// admission stream from the pinned upload ring (the host does not wait): the host
// copies the submitted arrays as they are, a kernel forms the slot's layout
static int load_state(pd_srv s, SrvSlot& sl, SrvReq* r) {
    pd_vd h = sl.h;
    const long n = r->n;
    const bool inbox = r->in_lo >= 0;  // the state is in the inbox: only the boxes go through the ring
    const size_t ox = stage_off_pos(), ov = ox + ((sizeof(double) * 3 * n + 63) & ~(size_t)63);
    const size_t need = inbox ? ox : ov + sizeof(double) * 3 * n;
    size_t lo = 0;
    char* st = ring_take(s, need, lo);
    char* tmp = nullptr;
    if (!st) {  // larger than the ring: pinned staging of its own, waited for below
        if (cudaMallocHost((void**)&tmp, need) != cudaSuccess) {
            cudaGetLastError();
            set_error("serving: pinned staging of %zu bytes failed", need);
            return PD_ENOMEM;
        }
        st = tmp;
    }
    BoxSet<double>* B = reinterpret_cast<BoxSet<double>*>(st);
    double* sh = reinterpret_cast<double*>(st + stage_off_shifts());
    int rc = ghost_boxes_host(h, B, sh);
    if (rc == PD_OK) rc = h->boxes.ensure(sizeof(BoxSet<double>));
    if (rc == PD_OK) rc = h->shifts.ensure(sizeof(double) * 81);
    void* dst = nullptr;
    if (rc == PD_OK) {
        h->nbox = B->nb;
        if (!inbox) {
            memcpy(st + ox, r->x.data(), sizeof(double) * 3 * n);
            memcpy(st + ov, r->v.data(), sizeof(double) * 3 * n);
        }
        cudaError_t ce = cudaMemcpyAsync(h->boxes.p, B, sizeof(BoxSet<double>), cudaMemcpyHostToDevice, s->as);
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync(h->shifts.p, sh, sizeof(double) * 81, cudaMemcpyHostToDevice, s->as);
        const char* xs = nullptr;  // device view of the submitted positions; velocities follow
        if (ce == cudaSuccess && !inbox) {
            ce = cudaHostGetDevicePointer(&dst, st, 0);
            xs = static_cast<const char*>(dst) + ox;
        } else if (ce == cudaSuccess) {
            xs = s->inbox.dev + r->in_lo;  // the inbox region: positions, then velocities at the same distance
        }
        if (ce == cudaSuccess && n > 0) {
            pd::launch(k_srv_unpack, (unsigned)std::min((n + 255) / 256, 148L * 8), 256, 0, s->as,
                       reinterpret_cast<const double*>(xs), reinterpret_cast<const double*>(xs + (ov - ox)), n,
                       (double4*)h->pos, (float*)h->props[sl.vp].d, h->cap);
            ce = cudaGetLastError();
        }
        if (ce != cudaSuccess) {
            set_error("serving: upload failed: %s", cudaGetErrorString(ce));
            rc = PD_ECUDA;
        }
    }
    if (!tmp) return rc == PD_OK ? ring_mark(s, lo, need) : rc;
    cudaStreamSynchronize(s->as);
    cudaFreeHost(tmp);
    return rc;
}

static int autotune_tx_on(pd_srv s, SrvSlot& sl, SrvReq* r);

// time the single-system force for candidate shapes (tile width x lanes per particle
// x CTA size) on a throw-away copy of the system (so the admitted system starts from
// the submitted state); keep the fastest
static int autotune_tx(pd_srv s, SrvReq* r) {
    AllocScope scope(s->as, s->pool);
    SrvSlot tmp;
    int rc = slot_reset(s, tmp, r, SrvShape{0, 2, FBLOCK_T});
    if (rc == PD_OK) rc = load_state(s, tmp, r);
    if (rc == PD_OK) rc = autotune_tx_on(s, tmp, r);
    cudaStreamSynchronize(s->as);
    tmp.release();
    return rc;
}

// the force time of the slot's system for its current shape (three launches after a warm one)
static int time_forces(pd_srv s, SrvSlot& sl, cudaEvent_t a, cudaEvent_t b, float& ms) {
    PD_TRY(md_forces(sl.md, s->as));
    PD_CUDA(cudaEventRecord(a, s->as));
    for (int k = 0; k < 3; ++k) PD_TRY(md_forces(sl.md, s->as));
    PD_CUDA(cudaEventRecord(b, s->as));
    PD_CUDA(cudaEventSynchronize(b));
    PD_CUDA(cudaEventElapsedTime(&ms, a, b));
    return PD_OK;
}

// two stages: the tile width with 2 lanes and CTAs of FBLOCK_T, then lanes per
// particle x CTA size at that width (systems of at least two tiles per SM)
static int autotune_shape(pd_srv s, SrvSlot& sl, SrvReq* r, cudaEvent_t a, cudaEvent_t b) {
    static const int cand_tx[] = {5, 7, 9, 12};
    static const int cand_lanes[] = {1, 2, 4};
    static const int cand_block[] = {FBLOCK_T, FBLOCK_T / 2};
    SrvShape best{0, 2, FBLOCK_T};
    float best_ms = 1e30f, ms = 0;
    sl.md->tile_p = 2;
    sl.md->tile_block = FBLOCK_T;
    for (int tx : cand_tx) {
        sl.md->tile_tx = tx;
        if (md_rebuild(sl.md, s->as) != PD_OK || !sl.md->tiles_active || sl.md->tcap > SRV_BIG_CAP) continue;
        PD_TRY(time_forces(s, sl, a, b, ms));
        if (ms < best_ms) {
            best_ms = ms;
            best.tx = tx;
        }
    }
    if (best.tx == 0) {
        set_error("serving: no tile width fits the batched kernel's shared memory");
        return PD_EOVERFLOW;
    }
    sl.md->tile_tx = best.tx;
    PD_TRY(md_rebuild(sl.md, s->as));
    // Lanes and CTA size only for systems of at least two tiles per SM: the timing
    // of a smaller system's single launch measures its latency, not the throughput
    // it gets among the batch's tiles.  Another shape must beat the default by 10 %.
    int sms = 148, dev = 0;
    PD_CUDA(cudaGetDevice(&dev));
    PD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (sl.md->ntiles >= 2L * sms) {
        const float base_ms = best_ms;
        for (int lanes : cand_lanes)
            for (int block : cand_block) {
                if (lanes == 2 && block == FBLOCK_T) continue;  // timed in the first stage
                sl.md->tile_p = lanes;
                sl.md->tile_block = block;
                PD_TRY(time_forces(s, sl, a, b, ms));
                if (ms < best_ms && ms < 0.9f * base_ms) {
                    best_ms = ms;
                    best.lanes = lanes;
                    best.block = block;
                }
            }
    }
    s->tuned[r->bucket] = best;
    return PD_OK;
}

static int autotune_tx_on(pd_srv s, SrvSlot& sl, SrvReq* r) {
    cudaEvent_t a, b;
    PD_CUDA(cudaEventCreate(&a));
    PD_CUDA(cudaEventCreate(&b));
    const double t0 = now_s(s);
    const int rc = autotune_shape(s, sl, r, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    s->tune_ms += 1000.0 * (now_s(s) - t0);
    return rc;
}

// Admission is host-side setup only: geometry, tile plan and capacities of the
// slot, the submitted state uploaded; the first build and forces run inside the
// next step graph (phase 0), restating the single-system first build.
static int admit_one(pd_srv s, SrvReq* r, int slot) {
    r->slot = slot;
    r->bucket = (int)std::floor(std::log2((double)std::max(r->n, 1L)));
    // the bucket's shape: set by the caller or tuned before, else tuned now, else the fixed one
    if (s->autotune && !s->tuned.count(r->bucket)) PD_TRY(autotune_tx(s, r));
    const auto it = s->tuned.find(r->bucket);
    const SrvShape shape = it != s->tuned.end() ? it->second : s->fixed;
    SrvSlot& sl = s->slots[slot];
    const double t0 = now_s(s);
    PD_TRY(slot_reset(s, sl, r, shape));
    s->ms[1] += 1e3 * (now_s(s) - t0);
    pd_md md = sl.md;
    pd_cl cl = md->vl->cl;
    const long n = r->n;
    PD_TRY(tile_plan(cl, n, md->tile_tx, md->tg, md->ntiles));
    // row capacity of the tiled build (tile_build's first estimate)
    md->tstride = std::max(32L, ((n + 31) / 32) * 32);
    const double rl = md->vl->r_cut;
    const double vol = r->L * r->L * r->L;
    md->tmax_nn = (((int)((double)n / vol * 4.18879 * rl * rl * rl * 1.5 + 32)) + 1) & ~1;
    PD_TRY(md->tnbr.ensure(sizeof(unsigned short) * (size_t)md->tstride * md->tmax_nn));
    PD_TRY(md->tnn.ensure(sizeof(int) * (size_t)md->tstride));
    PD_TRY(md->csR.ensure(sizeof(unsigned int) * (cl->ncells + 1)));
    PD_TRY(md->csI.ensure(sizeof(unsigned int) * (cl->ncells + 1)));
    PD_TRY(md->offb.ensure(sizeof(float4) * (size_t)n));
    md->tcap = SRV_CAP;
    md->tiles_active = true;
    md->off_valid = true;
    md->ready = true;
    PD_TRY(slot_scratch(s, sl, r));
    PD_TRY(load_state(s, sl, r));
    PD_CUDA(cudaMemsetAsync(s->phase.as<unsigned int>() + slot, 0, sizeof(unsigned int), s->as));
    r->x.clear();
    r->x.shrink_to_fit();
    r->v.clear();
    r->v.shrink_to_fit();
    r->state = 1;
    r->done_steps = 0;
    r->first = true;
    r->t_admit = now_s(s);
    return PD_OK;
}

// download bytes of one finished system: positions in id order, energies
static size_t retire_bytes(const SrvReq* r) {
    return (sizeof(double) * 3 * r->n + sizeof(double) * 4 * r->steps + 127) & ~(size_t)63;
}

// retire the finished systems: each system's final positions are formed in
// FP64 and written in id order on the GPU, then copied with its energies to the
// pinned outbox, where pd_srv_result reads them; when the outbox has no room, to
// the download buffer and from there to host vectors, in groups that fit that
// buffer, one wait per group
static int retire_all(pd_srv s, std::vector<std::pair<SrvReq*, bool>>& fin) {
    std::vector<char*> dst(fin.size(), nullptr);
    size_t k0 = 0;
    while (k0 < fin.size()) {
        size_t k1 = k0, used = 0;
        for (; k1 < fin.size(); ++k1) {
            if (fin[k1].second) continue;
            SrvReq* r = fin[k1].first;
            const size_t b = retire_bytes(r);
            if ((dst[k1] = s->outbox.take(r->ticket, b, r->out_lo, s->ev_free))) continue;
            if (b > s->down_bytes) {  // larger than the download buffer: alone in a group, buffer grown
                if (used > 0) break;
                if (s->down) cudaFreeHost(s->down);
                s->down = nullptr;
                s->down_bytes = 0;
                if (cudaMallocHost((void**)&s->down, b) != cudaSuccess) {
                    cudaGetLastError();
                    s->down = nullptr;
                    set_error("serving: pinned download buffer of %zu bytes failed", b);
                    return PD_ENOMEM;
                }
                s->down_bytes = b;
            }
            if (used + b > s->down_bytes) break;
            dst[k1] = s->down + used;
            used += b;
        }
        bool any = false;
        for (size_t k = k0; k < k1; ++k) {
            if (fin[k].second) continue;
            SrvReq* r = fin[k].first;
            SrvSlot& sl = s->slots[r->slot];
            pd_vd h = sl.h;
            const long n = r->n;
            double* xo = reinterpret_cast<double*>(h->pos);  // 24 n bytes of the 32 n held
            PD_TRY(mixed_to_positions_by_id(h, sl.md->vl->cl, sl.md->off, xo, s->as));
            const size_t ox = sizeof(double) * 3 * n, oe = (ox + 63) & ~(size_t)63;
            PD_CUDA(cudaMemcpyAsync(dst[k], xo, ox, cudaMemcpyDeviceToHost, s->as));
            PD_CUDA(cudaMemcpyAsync(dst[k] + oe, sl.Edev.p, sizeof(double) * 4 * r->steps, cudaMemcpyDeviceToHost,
                                    s->as));
            any = true;
        }
        if (any) PD_CUDA(cudaStreamSynchronize(s->as));
        for (size_t k = k0; k < k1; ++k) {
            SrvReq* r = fin[k].first;
            if (!fin[k].second) {
                const long n = r->n;
                const size_t ox = sizeof(double) * 3 * n, oe = (ox + 63) & ~(size_t)63;
                const double* E = reinterpret_cast<const double*>(dst[k] + oe);
                if (r->out_lo < 0) {
                    const double* X = reinterpret_cast<const double*>(dst[k]);
                    r->xo.assign(X, X + 3 * (size_t)n);
                    r->E.assign(E, E + 4 * (size_t)r->steps);
                }
                for (int j = 0; j < r->steps; ++j) s->rebuilds += E[4 * j + 3] != 0.0 ? 1 : 0;
            }
            r->state = fin[k].second ? 3 : 2;
            r->t_done = now_s(s);
            s->used -= r->bytes;
            s->systems_done++;
            s->completed.push_back(r->ticket);
        }
        k0 = k1;
    }
    fin.clear();
    return PD_OK;
}

}  // namespace pd

extern "C" {

int pd_srv_create(long hbm_budget_bytes, int max_slots, const pd_lj_params_t* lj, double dt, double skin,
                  pd_srv* out) {
    if (!out || !lj || max_slots < 1 || max_slots > MAXS || hbm_budget_bytes <= 0 || !(dt > 0) || skin < 0)
        return PD_EINVAL;
    pd_srv s = new pd_srv_s();
    s->budget = hbm_budget_bytes;
    s->max_slots = max_slots;
    s->lj = *lj;
    s->dt = dt;
    s->skin = skin;
    s->t0 = std::chrono::steady_clock::now();
    s->slots.resize(max_slots);
    memset(&s->hhdr, 0, sizeof(s->hhdr));
    int r = PD_OK;
    // partial buffers sized from the budget: at most budget/700 particles in flight
    long pmax = hbm_budget_bytes / 700 + 4096L * max_slots;
    s->kpart_cap = pmax / CHUNK + 2L * max_slots;
    s->tpart_cap = pmax / 4 + 4096L * max_slots;  // small boxes have about one tile per 7 particles
    {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaMemPoolProps pp;
        memset(&pp, 0, sizeof(pp));
        pp.allocType = cudaMemAllocationTypePinned;
        pp.location.type = cudaMemLocationTypeDevice;
        pp.location.id = dev;
        if (cudaMemPoolCreate(&s->pool, &pp) != cudaSuccess) {
            cudaGetLastError();
            s->pool = nullptr;
            delete s;
            set_error("pd_srv_create: memory pool creation failed");
            return PD_ECUDA;
        }
        unsigned long long keep = ~0ull;  // freed slot memory stays in the pool for reuse
        cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->as, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev_adm, cudaEventDisableTiming) != cudaSuccess ||
        (r = s->desc.ensure(sizeof(SysDesc) * max_slots)) != PD_OK || (r = s->hdr.ensure(sizeof(BatchHdr))) != PD_OK ||
        (r = s->maxd2.ensure(sizeof(unsigned long long) * max_slots)) != PD_OK ||
        (r = s->errs.ensure(sizeof(unsigned int) * max_slots)) != PD_OK ||
        (r = s->flags.ensure(sizeof(unsigned int) * max_slots)) != PD_OK ||
        (r = s->phase.ensure(sizeof(unsigned int) * max_slots)) != PD_OK ||
        (r = s->work.ensure(sizeof(RbWork))) != PD_OK || (r = s->nnmax.ensure(sizeof(unsigned int))) != PD_OK ||
        (r = s->tpart.ensure(sizeof(double) * 2 * s->tpart_cap)) != PD_OK ||
        (r = s->kpart.ensure(sizeof(double) * s->kpart_cap)) != PD_OK ||
        (r = s->ovf_f.ensure(sizeof(long) * s->tpart_cap)) != PD_OK ||
        (r = s->ovf_b.ensure(sizeof(long) * s->tpart_cap)) != PD_OK ||
        cudaMallocHost(&s->flags_h, sizeof(unsigned int) * max_slots) != cudaSuccess ||
        cudaMallocHost((void**)&s->up, (s->up_bytes = std::min((size_t)256 << 20,
                                                               std::max((size_t)8 << 20,
                                                                        (size_t)hbm_budget_bytes / 64)))) !=
            cudaSuccess ||
        cudaMallocHost((void**)&s->down, (s->down_bytes = s->up_bytes)) != cudaSuccess ||
        s->inbox.create(std::min((size_t)1 << 30, std::max((size_t)8 << 20, (size_t)hbm_budget_bytes / 32))) !=
            PD_OK ||
        s->outbox.create(std::min((size_t)1 << 30, std::max((size_t)8 << 20, (size_t)hbm_budget_bytes / 32))) !=
            PD_OK ||
        cudaMallocHost(&s->errs_h, sizeof(unsigned int) * max_slots) != cudaSuccess) {
        cudaGetLastError();
        pd_srv_destroy(s);
        set_error("pd_srv_create: allocation failed");
        return r != PD_OK ? r : PD_ENOMEM;
    }
    cudaMemset(s->hdr.p, 0, sizeof(BatchHdr));
    cudaMemset(s->errs.p, 0, sizeof(unsigned int) * max_slots);
    cudaMemset(s->flags.p, 0, sizeof(unsigned int) * max_slots);
    cudaMemset(s->phase.p, 0, sizeof(unsigned int) * max_slots);
    cudaMemset(s->work.p, 0, sizeof(RbWork));
    cudaDeviceSynchronize();
    {
        // reserve the budget in the pool once (one physical allocation instead of
        // one per slot buffer; the pool keeps freed memory)
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        size_t want = std::min((size_t)hbm_budget_bytes, fr > ((size_t)2 << 30) ? fr - ((size_t)2 << 30) : 0);
        void* p = nullptr;
        if (want > 0 && cudaMallocFromPoolAsync(&p, want, s->pool, s->as) == cudaSuccess) {
            cudaFreeAsync(p, s->as);
            cudaStreamSynchronize(s->as);
        }
        cudaGetLastError();
        // admission counts against the budget capped by the free memory at creation
        // (held by the pool when the reservation above succeeded): no free-memory query
        // per step (cudaMemGetInfo took 10-100 ms at times on a shared node)
        s->budget = (long)std::min((size_t)s->budget, want);
    }
    for (int lk = 0; lk < 4 && r == PD_OK; ++lk) r = capture_graph(s, lk);
    if (r != PD_OK) {
        pd_srv_destroy(s);
        return r;
    }
    *out = s;
    return PD_OK;
}

int pd_srv_destroy(pd_srv s) {
    if (!s) return PD_EINVAL;
    if (s->st) cudaStreamSynchronize(s->st);
    if (s->as) cudaStreamSynchronize(s->as);
    if (s->pool && s->as) {
        AllocScope scope(s->as, s->pool);
        for (SrvSlot& sl : s->slots) sl.release();
        cudaStreamSynchronize(s->as);
    }
    for (auto& u : s->up_use) cudaEventDestroy(u.ev);
    for (cudaEvent_t e : s->ev_free) cudaEventDestroy(e);
    if (s->up) cudaFreeHost(s->up);
    if (s->down) cudaFreeHost(s->down);
    s->inbox.destroy();
    s->outbox.destroy();
    s->slots.clear();
    for (auto& ge : s->gstep)
        if (ge) cudaGraphExecDestroy(ge);
    Buf* bufs[] = {&s->desc, &s->hdr,   &s->maxd2, &s->errs, &s->flags, &s->phase,
                   &s->work, &s->nnmax, &s->tpart, &s->kpart, &s->ovf_f, &s->ovf_b};
    for (Buf* b : bufs) b->release();
    if (s->flags_h) cudaFreeHost(s->flags_h);
    if (s->errs_h) cudaFreeHost(s->errs_h);
    if (s->st) cudaStreamDestroy(s->st);
    if (s->as) cudaStreamDestroy(s->as);
    if (s->ev_adm) cudaEventDestroy(s->ev_adm);
    if (s->pool) cudaMemPoolDestroy(s->pool);
    delete s;
    return PD_OK;
}

int pd_srv_set_tuning(pd_srv s, int autotune, int tx, int lanes, int block) {
    if (!s || tx < 0 || tx > TXMAX || (lanes != 1 && lanes != 2 && lanes != 4) ||
        (block != FBLOCK_T && block != FBLOCK_T / 2))
        return PD_EINVAL;
    s->autotune = autotune != 0;
    s->fixed = SrvShape{tx, lanes, block};
    return PD_OK;
}

int pd_srv_set_shape(pd_srv s, int bucket, int tx, int lanes, int block) {
    if (!s || bucket < 0 || tx < 1 || tx > TXMAX || (lanes != 1 && lanes != 2 && lanes != 4) ||
        (block != FBLOCK_T && block != FBLOCK_T / 2))
        return PD_EINVAL;
    s->tuned[bucket] = SrvShape{tx, lanes, block};
    return PD_OK;
}

int pd_srv_submit(pd_srv s, long n, double box, const double* x_host, const double* v_host, int steps,
                  long* ticket) {
    if (!s || n < 1 || !(box > 0) || !x_host || !v_host || steps < 1 || !ticket) return PD_EINVAL;
    if (box < 3.0 * (s->lj.r_cut + s->skin)) {
        set_error("pd_srv_submit: box %.4g is smaller than 3 (r_cut + skin)", box);
        return PD_EINVAL;
    }
    std::unique_ptr<SrvReq> r(new SrvReq());
    r->ticket = s->next_ticket++;
    r->n = n;
    r->L = box;
    r->steps = steps;
    r->bytes = estimate_bytes(n);
    r->t_submit = now_s(s);
    if ((long)r->bytes > s->budget) {
        set_error("pd_srv_submit: system of %ld particles exceeds the HBM budget", n);
        return PD_ENOMEM;
    }
    // the state to the pinned inbox (positions, then velocities at the staging
    // layout's distance), else to host vectors staged at admission
    const size_t half = (sizeof(double) * 3 * n + 63) & ~(size_t)63;
    if (char* p = s->inbox.take(r->ticket, half + sizeof(double) * 3 * n, r->in_lo, s->ev_free)) {
        const CopyJob jobs[2] = {{p, reinterpret_cast<const char*>(x_host), sizeof(double) * 3 * n},
                                 {p + half, reinterpret_cast<const char*>(v_host), sizeof(double) * 3 * n}};
        if (!s->copier) s->copier.reset(new CopyPool());
        s->copier->copy(jobs, 2);
    } else {
        r->x.assign(x_host, x_host + 3 * n);
        r->v.assign(v_host, v_host + 3 * n);
    }
    *ticket = r->ticket;
    s->queue.push_back(r->ticket);
    s->reqs[r->ticket] = std::move(r);
    return PD_OK;
}

int pd_srv_tick(pd_srv s, int* n_active, int* n_queued) {
    if (!s) return PD_EINVAL;
    AllocScope scope(s->as, s->pool);  // slot memory: stream-ordered from the server's pool
    // systems that finished in the previous step (the GPU is idle here)
    double t_ret = now_s(s);
    PD_TRY(retire_all(s, s->finished));
    s->ms[3] += 1e3 * (now_s(s) - t_ret);
    if (s->adm_pending) {
        PD_CUDA(cudaStreamWaitEvent(s->st, s->ev_adm, 0));  // admissions before the step that builds them
        s->adm_pending = false;
    }
    if (s->dirty && !s->active.empty()) PD_TRY(upload_tables(s));
    // one velocity-Verlet step of every active system; admissions are prepared
    // meanwhile on the admission stream (host work and asynchronous copies only)
    const bool stepping = !s->active.empty();
    // steps in this launch: up to 8, none past a system's last step, at most 2
    // while requests wait for a slot (they are admitted between launches)
    int K = 8;
    for (SrvReq* r : s->active) K = std::min(K, r->steps - r->done_steps + (r->first ? 1 : 0));
    if (!s->queue.empty()) K = std::min(K, 2);
    int lk = 0;
    while (lk < 3 && (2 << lk) <= K) ++lk;
    K = 1 << lk;
    double t_step = now_s(s);
    if (stepping) PD_CUDA(cudaGraphLaunch(s->gstep[lk], s->st));
    double ta = now_s(s);
    std::vector<char> used_slot(s->max_slots, 0);
    for (SrvReq* r : s->active) used_slot[r->slot] = 1;
    std::vector<SrvReq*> admitted;
    while (!s->queue.empty() && (int)(s->active.size() + admitted.size()) < s->max_slots) {
        SrvReq* r = s->reqs[s->queue.front()].get();
        if (s->used + r->bytes > (size_t)s->budget) break;
        int slot = 0;
        while (used_slot[slot]) ++slot;
        s->queue.pop_front();
        s->used += r->bytes;
        int rc = admit_one(s, r, slot);
        inbox_release(s, r);
        if (rc != PD_OK) {
            r->state = 3;
            s->used -= r->bytes;
            cudaStreamSynchronize(s->st);
            cudaStreamSynchronize(s->as);
            return rc;
        }
        used_slot[slot] = 1;
        admitted.push_back(r);
    }
    if (!admitted.empty()) {
        PD_CUDA(cudaEventRecord(s->ev_adm, s->as));
        s->adm_pending = true;
    }
    s->ms[0] += 1e3 * (now_s(s) - ta);
    if (stepping) {
        PD_CUDA(cudaStreamSynchronize(s->st));
        s->steps_run += K;
        __atomic_fetch_add(&g_launches, (unsigned long long)(GRAPH_KERNELS * K), __ATOMIC_RELAXED);
        s->ms[2] += 1e3 * (now_s(s) - t_step);
    }
    // rebuild flags and errors of the step; finished systems are retired by the next tick
    std::vector<SrvReq*> keep;
    for (SrvReq* r : s->active) {
        SrvSlot& sl = s->slots[r->slot];
        const unsigned int er = s->errs_h[r->slot];
        // the first launch of a system spends its first step on the first build and forces
        const int done = stepping ? K - (r->first ? 1 : 0) : 0;
        r->first = false;
        r->done_steps += done;
        sl.md->steps += done;
        s->particle_steps += r->n * (long)done;
        if (er & (ERR_IMG_OVERFLOW | ERR_NN_OVERFLOW | ERR_TILE_CAP | ERR_TIMEOUT | ERR_CELL_RANGE)) {
            set_error("serving: system %ld failed in a batched step (err=0x%x)", r->ticket, er);
            s->finished.push_back({r, true});
        } else if (r->done_steps >= r->steps) {
            s->finished.push_back({r, false});
        } else {
            keep.push_back(r);
        }
    }
    if (keep.size() != s->active.size() || !admitted.empty()) s->dirty = true;
    for (SrvReq* r : admitted) keep.push_back(r);
    s->active.swap(keep);
    if (s->active.empty() && !s->finished.empty()) {
        // nothing left to step: retire now rather than at the next tick
        t_ret = now_s(s);
        PD_TRY(retire_all(s, s->finished));
        s->ms[3] += 1e3 * (now_s(s) - t_ret);
    }
    if (n_queued) *n_queued = (int)s->queue.size();
    if (n_active) *n_active = (int)s->active.size();
    return PD_OK;
}

int pd_srv_completed(pd_srv s, long* tickets, int cap, int* n) {
    if (!s || !n || (cap > 0 && !tickets)) return PD_EINVAL;
    int k = 0;
    while (k < cap && k < (int)s->completed.size()) {
        tickets[k] = s->completed[k];
        ++k;
    }
    s->completed.erase(s->completed.begin(), s->completed.begin() + k);
    *n = k;
    return PD_OK;
}

int pd_srv_state(pd_srv s, long ticket, int* state) {
    if (!s || !state) return PD_EINVAL;
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return PD_EINVAL;
    *state = it->second->state;
    return PD_OK;
}

int pd_srv_result(pd_srv s, long ticket, double* x_out, double* E_out, double* times) {
    if (!s) return PD_EINVAL;
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return PD_EINVAL;
    SrvReq* r = it->second.get();
    if (r->state != 2) return PD_ESTATE;
    if (r->out_lo >= 0) {  // in the pinned outbox: positions, then energies 64-byte aligned
        const char* b = s->outbox.base + r->out_lo;
        const size_t ox = sizeof(double) * 3 * r->n, oe = (ox + 63) & ~(size_t)63;
        if (x_out) memcpy(x_out, b, ox);
        if (E_out) memcpy(E_out, b + oe, sizeof(double) * 4 * r->steps);
    } else {
        if (x_out) memcpy(x_out, r->xo.data(), sizeof(double) * r->xo.size());
        if (E_out) memcpy(E_out, r->E.data(), sizeof(double) * r->E.size());
    }
    if (times) {
        times[0] = r->t_submit;
        times[1] = r->t_admit;
        times[2] = r->t_done;
    }
    return PD_OK;
}

int pd_srv_release(pd_srv s, long ticket) {
    if (!s) return PD_EINVAL;
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end() || (it->second->state != 2 && it->second->state != 3)) return PD_EINVAL;
    if (it->second->out_lo >= 0) {
        if (PinnedFifo::Region* g = s->outbox.find(ticket)) g->done = true;
        s->outbox.trim(s->ev_free);
    }
    s->reqs.erase(it);
    return PD_OK;
}

int pd_srv_stats(pd_srv s, long* particle_steps, long* systems_done, long* ticks, long* rebuilds, double* tune_ms) {
    if (!s) return PD_EINVAL;
    if (particle_steps) *particle_steps = s->particle_steps;
    if (systems_done) *systems_done = s->systems_done;
    if (ticks) *ticks = s->steps_run;
    if (rebuilds) *rebuilds = s->rebuilds;
    if (tune_ms) *tune_ms = s->tune_ms;
    return PD_OK;
}

int pd_srv_timers(pd_srv s, double ms[4]) {
    if (!s || !ms) return PD_EINVAL;
    for (int i = 0; i < 4; ++i) ms[i] = s->ms[i];
    return PD_OK;
}

int pd_srv_tuned(pd_srv s, int* buckets, int* widths, int* lanes, int* blocks, int cap, int* n) {
    if (!s || !n) return PD_EINVAL;
    int k = 0;
    for (auto& kv : s->tuned) {
        if (k < cap) {
            if (buckets) buckets[k] = kv.first;
            if (widths) widths[k] = kv.second.tx;
            if (lanes) lanes[k] = kv.second.lanes;
            if (blocks) blocks[k] = kv.second.block;
        }
        ++k;
    }
    *n = k;
    return PD_OK;
}

}  // extern "C"
