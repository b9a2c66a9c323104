// pd_serve.cu -- serving loop: many independent LJ systems (precision form)
// resident on one GPU, stepped together by persistent batched kernels.
//
// The reference's only many-systems idiom is a test kernel reading an array of
// vector_dist / cell-list views (Vector/cuda/vector_dist_gpu_MP_tests.cu:427-781).
// Here that array is a device table of system descriptors (SysDesc) and every
// per-step phase is one persistent kernel over the work of all active systems:
//   kick-drift   256-particle chunks of every system (grid-stride, fixed mapping)
//   images       256-image chunks (skipped for systems rebuilt this step)
//   forces       tiles of every system, pulled from an atomic work queue (load
//                balance over uneven systems); the tile body is the single-system
//                mixed-form kernel's (pd_mixed_dev.cuh)
//   kick         chunks, kinetic energy per chunk
//   energies     one block per system, fixed-order sums of the tile and chunk
//                partials -> E[step]
// Partials are indexed by (system, work item), never by CTA, so a system's
// results do not depend on which other systems share the batch.  The two
// phase sequences (kick-drift; images..energies) are captured once as CUDA
// graphs: all sizes live in device memory, so admissions, retirements and
// rebuilds only rewrite the tables.  The displacement check between them is the
// one host synchronisation per step; flagged systems are rebuilt individually.
//
// Admission: FIFO; a request is admitted when a slot is free and its memory
// estimate fits both the server's HBM budget and cudaMemGetInfo's free memory.
// Autotuner: per size bucket (floor(log2 N)), the first admitted system times
// the force kernel for several tile widths and the best one is kept.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <deque>
#include <map>
#include <memory>
#include <vector>

#include "pd_device.cuh"
#include "pd_internal.cuh"
#include "pd_lj.cuh"
#include "pd_md.cuh"
#include "pd_mixed.cuh"
#include "pd_mixed_dev.cuh"
#include "pd_tile.cuh"

namespace pd {

static constexpr int SRV_P = 2;                       // lanes per particle in the batched force kernel
static constexpr int SRV_SMEM = 96 * 1024;            // staging bytes per force CTA (fixed: graph-invariant)
static constexpr unsigned SRV_CAP = SRV_SMEM / 16;    // staged records per tile
static constexpr int CHUNK = 256;

struct SysDesc {
    float4* off;
    const float4* offb;
    const float4* offK;
    const int* img_src;
    float* v;
    float* f;
    long cap, n_real, n_img;
    TileGeom tg;
    const unsigned int* csR;
    const unsigned int* csI;
    const unsigned int* nbr;
    const int* nn;
    long tstride;
    unsigned int tcap;
    float sx, sy, sz;
    long tile_base, ntiles;
    long chunk_base, nchunk;
    long img_base, nimg_chunk;
    long tpart_base, kpart_base;
    unsigned long long* maxd2;
    unsigned int* err;
    double* E;
    int* step;
    int skip_replay;
    double mass;
};

struct BatchHdr {
    int nsys;
    int pad0;
    long tot_tiles, tot_chunks, tot_img;
    unsigned int tile_ctr;
    unsigned int pad1;
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

__global__ void __launch_bounds__(CHUNK) k_b_kick_drift(const SysDesc* __restrict__ D, const BatchHdr* __restrict__ B,
                                                        float half, float dt) {
    const int nsys = B->nsys;
    const long tot = B->tot_chunks;
    for (long g = blockIdx.x; g < tot; g += gridDim.x) {
        const int s = find_sys(D, nsys, g, 1);
        const SysDesc& d = D[s];
        const long i = (g - d.chunk_base) * CHUNK + threadIdx.x;
        double mx = 0;
        if (i < d.n_real) {
            float4 o = d.off[i];
            const long cap = d.cap;
            float vx = d.v[i] + half * d.f[i];
            float vy = d.v[cap + i] + half * d.f[cap + i];
            float vz = d.v[2 * cap + i] + half * d.f[2 * cap + i];
            o.x += dt * vx;
            o.y += dt * vy;
            o.z += dt * vz;
            d.v[i] = vx;
            d.v[cap + i] = vy;
            d.v[2 * cap + i] = vz;
            d.off[i] = o;
            float4 b = d.offb[i];
            mx = (double)dist2(o.x - b.x, o.y - b.y, o.z - b.z);
        }
        mx = warp_max(mx);
        if ((threadIdx.x & 31) == 0 && mx > 0) atomic_max_nonneg(d.maxd2, mx);
    }
}

__global__ void __launch_bounds__(CHUNK) k_b_replay(const SysDesc* __restrict__ D, const BatchHdr* __restrict__ B) {
    const int nsys = B->nsys;
    const long tot = B->tot_img;
    for (long g = blockIdx.x; g < tot; g += gridDim.x) {
        const int s = find_sys(D, nsys, g, 2);
        const SysDesc& d = D[s];
        if (d.skip_replay) continue;
        const long k = (g - d.img_base) * CHUNK + threadIdx.x;
        if (k < d.n_img) {
            float4 o = d.off[d.img_src[k]], q = d.offK[k];
            float4 r = d.off[d.n_real + k];
            r.x = o.x + q.x;
            r.y = o.y + q.y;
            r.z = o.z + q.z;
            d.off[d.n_real + k] = r;
        }
    }
}

__global__ void __launch_bounds__(FBLOCK_T) k_b_force(const SysDesc* __restrict__ D, BatchHdr* __restrict__ B,
                                                      LJP<float> Pr, double* __restrict__ tpart) {
    extern __shared__ __align__(128) unsigned char tile_raw[];
    float4* sm = reinterpret_cast<float4*>(tile_raw);
    __shared__ TileShM S;
    __shared__ unsigned long long bar;
    __shared__ long cur;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    unsigned int uses = 0;
    const int nsys = B->nsys;
    const long tot = B->tot_tiles;
    for (;;) {
        // generic-proxy writes of the previous tile are ordered before the next bulk copies
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) cur = (long)atomicAdd(&B->tile_ctr, 1u);
        __syncthreads();
        const long g = cur;
        if (g >= tot) break;
        const int s = find_sys(D, nsys, g, 0);
        const SysDesc& d = D[s];
        double pe = 0, vir = 0;
        mixed_tile<SRV_P>(g - d.tile_base, d.off, d.n_real, d.tg, d.csR, d.csI, SRV_CAP, d.nbr, d.nn, d.tstride, d.sx,
                          d.sy, d.sz, Pr, d.f, d.cap, d.err, sm, S, &bar, uses, pe, vir);
        pe = block_sum<double, FBLOCK_T>(pe);
        vir = block_sum<double, FBLOCK_T>(vir);
        if (threadIdx.x == 0) {
            const long slot = d.tpart_base + (g - d.tile_base);
            tpart[2 * slot] = pe;
            tpart[2 * slot + 1] = vir;
        }
    }
}

__global__ void __launch_bounds__(CHUNK) k_b_kick(const SysDesc* __restrict__ D, const BatchHdr* __restrict__ B,
                                                  float half, double* __restrict__ kpart) {
    const int nsys = B->nsys;
    const long tot = B->tot_chunks;
    for (long g = blockIdx.x; g < tot; g += gridDim.x) {
        const int s = find_sys(D, nsys, g, 1);
        const SysDesc& d = D[s];
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

// one block per system: E[step] = (KE, PE, virial, rebuilt) in a fixed order
__global__ void __launch_bounds__(256) k_b_energy(const SysDesc* __restrict__ D, const BatchHdr* __restrict__ B,
                                                  const double* __restrict__ tpart, const double* __restrict__ kpart) {
    const int s = blockIdx.x;
    if (s >= B->nsys) return;
    const SysDesc& d = D[s];
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
        d.E[4 * st + 3] = (double)d.skip_replay;
        *d.step = st + 1;
    }
}

}  // namespace pd

using namespace pd;

// ---------------------------------------------------------------------------
struct SrvReq {
    long ticket = 0;
    long n = 0;
    double L = 0;
    int steps = 0;
    int state = 0;  // 0 queued, 1 running, 2 done, 3 failed
    std::vector<double> x, v, xo, E;
    double t_submit = 0, t_admit = 0, t_done = 0;
    size_t bytes = 0;
    pd_vd h = nullptr;
    pd_md md = nullptr;
    Buf Edev, step;
    int slot = -1;
    int bucket = 0;
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
    size_t used = 0;
    // device tables (fixed capacity: graph-invariant pointers)
    Buf desc, hdr, maxd2, errs, tpart, kpart;
    long tpart_cap = 0, kpart_cap = 0;
    std::vector<SysDesc> hdesc;
    BatchHdr hhdr;
    unsigned long long* maxd2_h = nullptr;
    cudaStream_t st = nullptr;
    cudaGraphExec_t gA = nullptr, gB = nullptr;
    int grid_force = 0, grid_chunks = 0;
    bool dirty = true;
    // autotuner: size bucket -> tile width
    bool autotune = true;
    int fixed_tx = 0;
    std::map<int, int> tuned;
    // statistics
    long particle_steps = 0, systems_done = 0, replays = 0, rebuilds = 0;
    double tune_ms = 0;
};

namespace pd {

static double now_s(pd_srv s) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - s->t0).count();
}

static size_t estimate_bytes(long n) {
    // positions (FP64 record + FP32 offsets + build copies), images (~30% for small
    // boxes), FP32 velocity / force, rows of ~100 16-bit entries, cell tables
    return (size_t)n * 700 + ((size_t)8 << 20);
}

static void fill_desc(pd_srv s, SrvReq* r, SysDesc& d) {
    pd_vd h = r->h;
    pd_md md = r->md;
    memset(&d, 0, sizeof(d));
    d.off = md->off.as<float4>();
    d.offb = md->offb.as<float4>();
    d.offK = md->offK.as<float4>();
    d.img_src = h->img_src.as<int>();
    d.v = (float*)h->props[md->mp.vel_prop].d;
    d.f = (float*)h->props[md->mp.force_prop].d;
    d.cap = h->cap;
    d.n_real = h->n_real;
    d.n_img = h->n_img;
    d.tg = md->tg;
    d.csR = md->csR.as<unsigned int>();
    d.csI = md->csI.as<unsigned int>();
    d.nbr = md->tnbr.as<unsigned int>();
    d.nn = md->tnn.as<int>();
    d.tstride = md->tstride;
    d.tcap = md->tcap;
    d.sx = (float)md->vl->cl->spacing[0];
    d.sy = (float)md->vl->cl->spacing[1];
    d.sz = (float)md->vl->cl->spacing[2];
    d.ntiles = md->ntiles;
    d.nchunk = (h->n_real + CHUNK - 1) / CHUNK;
    d.nimg_chunk = (h->n_img + CHUNK - 1) / CHUNK;
    d.maxd2 = s->maxd2.as<unsigned long long>() + r->slot;
    d.err = &h->ctrl->err;
    d.E = r->Edev.as<double>();
    d.step = r->step.as<int>();
    d.mass = md->mp.mass;
}

// rebuild the descriptor table, prefixes and partial-buffer layout
static int upload_tables(pd_srv s) {
    int ns = (int)s->active.size();
    s->hdesc.resize(ns);
    long tb = 0, cb = 0, ib = 0, tp = 0, kp = 0;
    for (int k = 0; k < ns; ++k) {
        SysDesc& d = s->hdesc[k];
        int skip = d.skip_replay;
        fill_desc(s, s->active[k], d);
        d.skip_replay = skip;
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
    s->hhdr.tile_ctr = 0;
    if (ns) PD_CUDA(cudaMemcpyAsync(s->desc.p, s->hdesc.data(), sizeof(SysDesc) * ns, cudaMemcpyHostToDevice, s->st));
    PD_CUDA(cudaMemcpyAsync(s->hdr.p, &s->hhdr, sizeof(BatchHdr), cudaMemcpyHostToDevice, s->st));
    PD_CUDA(cudaStreamSynchronize(s->st));  // host staging vectors are reused
    s->dirty = false;
    return PD_OK;
}

static int capture_graphs(pd_srv s) {
    float half = (float)(0.5 * s->dt / 1.0), dt = (float)s->dt;
    LJP<float> P;
    P.eps24 = (float)(24.0 * s->lj.eps);
    P.eps4 = (float)(4.0 * s->lj.eps);
    P.sig2 = (float)(s->lj.sigma * s->lj.sigma);
    float rc = (float)s->lj.r_cut;
    P.rc2 = rc * rc;
    PD_CUDA(cudaFuncSetAttribute(k_b_force, cudaFuncAttributeMaxDynamicSharedMemorySize, SRV_SMEM));
    int sms = 148, dev = 0, per = 1;
    PD_CUDA(cudaGetDevice(&dev));
    PD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    PD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_b_force, FBLOCK_T, SRV_SMEM));
    s->grid_force = sms * std::max(per, 1);
    s->grid_chunks = sms * 8;
    const SysDesc* D = s->desc.as<SysDesc>();
    BatchHdr* B = s->hdr.as<BatchHdr>();
    cudaGraph_t g = nullptr;
    PD_CUDA(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(s->maxd2.p, 0, sizeof(unsigned long long) * s->max_slots, s->st);
    k_b_kick_drift<<<s->grid_chunks, CHUNK, 0, s->st>>>(D, B, half, dt);
    PD_CUDA(cudaStreamEndCapture(s->st, &g));
    PD_CUDA(cudaGraphInstantiate(&s->gA, g, 0));
    cudaGraphDestroy(g);
    PD_CUDA(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(&B->tile_ctr, 0, sizeof(unsigned int), s->st);
    k_b_replay<<<s->grid_chunks, CHUNK, 0, s->st>>>(D, B);
    k_b_force<<<s->grid_force, FBLOCK_T, SRV_SMEM, s->st>>>(D, B, P, s->tpart.as<double>());
    k_b_kick<<<s->grid_chunks, CHUNK, 0, s->st>>>(D, B, half, s->kpart.as<double>());
    k_b_energy<<<s->max_slots, 256, 0, s->st>>>(D, B, s->tpart.as<double>(), s->kpart.as<double>());
    PD_CUDA(cudaStreamEndCapture(s->st, &g));
    PD_CUDA(cudaGraphInstantiate(&s->gB, g, 0));
    cudaGraphDestroy(g);
    return PD_OK;
}

static int make_system(pd_srv s, SrvReq* r, pd_vd* hout, pd_md* mout) {
    double lo[3] = {0, 0, 0}, hi[3] = {r->L, r->L, r->L};
    int bc[3] = {PD_PERIODIC, PD_PERIODIC, PD_PERIODIC};
    double rl = s->lj.r_cut + s->skin;
    double g[3] = {rl, rl, rl};
    pd_vd h = nullptr;
    PD_TRY(pd_create(3, PD_F64, r->n, lo, hi, bc, g, 0, &h));
    *hout = h;
    int vp = -1, fp = -1;
    PD_TRY(pd_add_prop(h, PD_F32, 3, &vp));
    PD_TRY(pd_add_prop(h, PD_F32, 3, &fp));
    PD_TRY(pd_h2d_pos(h, r->x.data(), 0, r->n, s->st));
    std::vector<float> vc(3 * r->n);
    for (long i = 0; i < r->n; ++i)
        for (int d = 0; d < 3; ++d) vc[(size_t)d * r->n + i] = (float)r->v[3 * i + d];
    PD_TRY(pd_h2d_prop(h, vp, vc.data(), 0, r->n, s->st));
    PD_CUDA(cudaStreamSynchronize(s->st));  // vc is a local
    pd_md_params_t mp;
    memset(&mp, 0, sizeof(mp));
    mp.dt = s->dt;
    mp.mass = 1.0;
    mp.skin = s->skin;
    mp.vel_prop = vp;
    mp.force_prop = fp;
    mp.precision = PD_PREC_MIXED;
    PD_TRY(pd_md_create(h, &s->lj, &mp, mout));
    return PD_OK;
}

static int autotune_tx_on(pd_srv s, SrvReq* r);

// time the single-system force for candidate tile widths on a throw-away copy of
// the system (so the admitted system starts from the submitted state); keep the fastest
static int autotune_tx(pd_srv s, SrvReq* r) {
    SrvReq tmp;
    tmp.n = r->n;
    tmp.L = r->L;
    tmp.x = r->x;
    tmp.v = r->v;
    int rc = make_system(s, &tmp, &tmp.h, &tmp.md);
    if (rc == PD_OK) {
        std::swap(tmp.h, r->h);
        std::swap(tmp.md, r->md);
        rc = autotune_tx_on(s, r);
        std::swap(tmp.h, r->h);
        std::swap(tmp.md, r->md);
    }
    if (tmp.md) pd_md_destroy(tmp.md);
    if (tmp.h) pd_destroy(tmp.h);
    return rc;
}

static int autotune_tx_on(pd_srv s, SrvReq* r) {
    static const int cand[] = {3, 5, 7, 9, 12};
    cudaEvent_t a, b;
    PD_CUDA(cudaEventCreate(&a));
    PD_CUDA(cudaEventCreate(&b));
    int best = 0;
    float best_ms = 1e30f;
    double t0 = now_s(s);
    for (int tx : cand) {
        r->md->tile_tx = tx;
        int rc = md_rebuild(r->md, s->st);
        if (rc != PD_OK || !r->md->tiles_active || r->md->tcap > SRV_CAP) continue;
        PD_TRY(md_forces(r->md, s->st));  // warm
        PD_CUDA(cudaEventRecord(a, s->st));
        for (int k = 0; k < 3; ++k) PD_TRY(md_forces(r->md, s->st));
        PD_CUDA(cudaEventRecord(b, s->st));
        PD_CUDA(cudaEventSynchronize(b));
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        if (ms < best_ms) {
            best_ms = ms;
            best = tx;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    s->tune_ms += 1000.0 * (now_s(s) - t0);
    if (best == 0) {
        set_error("serving: no tile width fits the batched kernel's shared memory");
        return PD_EOVERFLOW;
    }
    s->tuned[r->bucket] = best;
    return PD_OK;
}

static int admit_one(pd_srv s, SrvReq* r, int slot) {
    r->slot = slot;
    r->bucket = (int)std::floor(std::log2((double)std::max(r->n, 1L)));
    if (s->autotune && !s->tuned.count(r->bucket)) PD_TRY(autotune_tx(s, r));
    PD_TRY(make_system(s, r, &r->h, &r->md));
    r->md->tile_tx = s->autotune ? s->tuned[r->bucket] : s->fixed_tx;
    PD_TRY(r->Edev.ensure(sizeof(double) * 4 * (r->steps > 0 ? r->steps : 1)));
    PD_TRY(r->step.ensure(sizeof(int)));
    PD_CUDA(cudaMemsetAsync(r->step.p, 0, sizeof(int), s->st));
    PD_TRY(pd_md_run(r->md, 0, s->st, nullptr));  // first build + forces
    if (!r->md->tiles_active || r->md->tcap > SRV_CAP) {
        set_error("serving: system of %ld particles does not fit the batched tile kernel", r->n);
        return PD_EOVERFLOW;
    }
    r->x.clear();
    r->x.shrink_to_fit();
    r->v.clear();
    r->v.shrink_to_fit();
    r->state = 1;
    r->t_admit = now_s(s);
    return PD_OK;
}

static void free_system(SrvReq* r) {
    if (r->md) pd_md_destroy(r->md);
    if (r->h) pd_destroy(r->h);
    r->md = nullptr;
    r->h = nullptr;
    r->Edev.release();
    r->step.release();
}

static int retire(pd_srv s, SrvReq* r) {
    pd_vd h = r->h;
    PD_TRY(mixed_to_positions(h, r->md->vl->cl, r->md->off, s->st));
    std::vector<double> xs(3 * r->n);
    std::vector<long> gid(r->n);
    PD_TRY(pd_d2h_pos(h, xs.data(), 0, r->n, s->st));
    PD_TRY(pd_d2h_gid(h, gid.data(), 0, r->n, s->st));
    r->xo.assign(3 * r->n, 0.0);
    for (long i = 0; i < r->n; ++i)
        for (int d = 0; d < 3; ++d) r->xo[3 * gid[i] + d] = xs[3 * i + d];
    r->E.assign(4 * (size_t)r->steps, 0.0);
    if (r->steps > 0)
        PD_CUDA(cudaMemcpy(r->E.data(), r->Edev.p, sizeof(double) * 4 * r->steps, cudaMemcpyDeviceToHost));
    PD_TRY(read_ctrl(h, s->st));
    const bool bad = (h->ctrl_h->err & (ERR_IMG_OVERFLOW | ERR_NN_OVERFLOW)) != 0;
    free_system(r);
    r->state = bad ? 3 : 2;
    r->t_done = now_s(s);
    s->used -= r->bytes;
    s->systems_done++;
    return PD_OK;
}

}  // namespace pd

extern "C" {

int pd_srv_create(long hbm_budget_bytes, int max_slots, const pd_lj_params_t* lj, double dt, double skin,
                  pd_srv* out) {
    if (!out || !lj || max_slots < 1 || max_slots > 1024 || hbm_budget_bytes <= 0 || !(dt > 0) || skin < 0)
        return PD_EINVAL;
    pd_srv s = new pd_srv_s();
    s->budget = hbm_budget_bytes;
    s->max_slots = max_slots;
    s->lj = *lj;
    s->dt = dt;
    s->skin = skin;
    s->t0 = std::chrono::steady_clock::now();
    memset(&s->hhdr, 0, sizeof(s->hhdr));
    int r = PD_OK;
    // partial buffers sized from the budget: at most budget/700 particles in flight
    long pmax = hbm_budget_bytes / 700 + 4096L * max_slots;
    s->kpart_cap = pmax / CHUNK + 2L * max_slots;
    s->tpart_cap = pmax / 4 + 4096L * max_slots;  // small boxes have about one tile per 7 particles
    if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess ||
        (r = s->desc.ensure(sizeof(SysDesc) * max_slots)) != PD_OK || (r = s->hdr.ensure(sizeof(BatchHdr))) != PD_OK ||
        (r = s->maxd2.ensure(sizeof(unsigned long long) * max_slots)) != PD_OK ||
        (r = s->tpart.ensure(sizeof(double) * 2 * s->tpart_cap)) != PD_OK ||
        (r = s->kpart.ensure(sizeof(double) * s->kpart_cap)) != PD_OK ||
        cudaMallocHost(&s->maxd2_h, sizeof(unsigned long long) * max_slots) != cudaSuccess) {
        cudaGetLastError();
        pd_srv_destroy(s);
        set_error("pd_srv_create: allocation failed");
        return r != PD_OK ? r : PD_ENOMEM;
    }
    cudaMemset(s->hdr.p, 0, sizeof(BatchHdr));
    if ((r = capture_graphs(s)) != PD_OK) {
        pd_srv_destroy(s);
        return r;
    }
    *out = s;
    return PD_OK;
}

int pd_srv_destroy(pd_srv s) {
    if (!s) return PD_EINVAL;
    if (s->st) cudaStreamSynchronize(s->st);
    for (auto& kv : s->reqs) free_system(kv.second.get());
    if (s->gA) cudaGraphExecDestroy(s->gA);
    if (s->gB) cudaGraphExecDestroy(s->gB);
    s->desc.release();
    s->hdr.release();
    s->maxd2.release();
    s->tpart.release();
    s->kpart.release();
    if (s->maxd2_h) cudaFreeHost(s->maxd2_h);
    if (s->st) cudaStreamDestroy(s->st);
    delete s;
    return PD_OK;
}

int pd_srv_set_tuning(pd_srv s, int autotune, int tx) {
    if (!s || tx < 0 || tx > TXMAX) return PD_EINVAL;
    s->autotune = autotune != 0;
    s->fixed_tx = tx;
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
    r->x.assign(x_host, x_host + 3 * n);
    r->v.assign(v_host, v_host + 3 * n);
    r->bytes = estimate_bytes(n);
    r->t_submit = now_s(s);
    if ((long)r->bytes > s->budget) {
        set_error("pd_srv_submit: system of %ld particles exceeds the HBM budget", n);
        return PD_ENOMEM;
    }
    *ticket = r->ticket;
    s->queue.push_back(r->ticket);
    s->reqs[r->ticket] = std::move(r);
    return PD_OK;
}

int pd_srv_tick(pd_srv s, int* n_active, int* n_queued) {
    if (!s) return PD_EINVAL;
    // admission (FIFO) by slot and memory
    std::vector<char> used_slot(s->max_slots, 0);
    for (SrvReq* r : s->active) used_slot[r->slot] = 1;
    while (!s->queue.empty() && (int)s->active.size() < s->max_slots) {
        SrvReq* r = s->reqs[s->queue.front()].get();
        size_t fr = 0, tot = 0;
        PD_CUDA(cudaMemGetInfo(&fr, &tot));
        if (s->used + r->bytes > (size_t)s->budget || r->bytes + (256ul << 20) > fr) break;
        int slot = 0;
        while (used_slot[slot]) ++slot;
        s->queue.pop_front();
        s->used += r->bytes;
        int rc = admit_one(s, r, slot);
        if (rc != PD_OK) {
            free_system(r);
            r->state = 3;
            s->used -= r->bytes;
            return rc;
        }
        used_slot[slot] = 1;
        s->active.push_back(r);
        s->dirty = true;
    }
    if (n_queued) *n_queued = (int)s->queue.size();
    if (s->active.empty()) {
        if (n_active) *n_active = 0;
        return PD_OK;
    }
    if (s->dirty) PD_TRY(upload_tables(s));
    // kick-drift of every system, displacement per slot
    PD_CUDA(cudaGraphLaunch(s->gA, s->st));
    PD_CUDA(cudaMemcpyAsync(s->maxd2_h, s->maxd2.p, sizeof(unsigned long long) * s->max_slots,
                            cudaMemcpyDeviceToHost, s->st));
    PD_CUDA(cudaStreamSynchronize(s->st));
    double lim2 = 0.25 * s->skin * s->skin;
    bool changed = false;
    for (size_t k = 0; k < s->active.size(); ++k) {
        SrvReq* r = s->active[k];
        double d2;
        memcpy(&d2, &s->maxd2_h[r->slot], sizeof(double));
        int reb = (s->skin <= 0 || d2 > lim2) ? 1 : 0;
        if (reb) {
            PD_TRY(md_rebuild(r->md, s->st));
            if (!r->md->tiles_active || r->md->tcap > SRV_CAP) {
                set_error("serving: rebuilt system no longer fits the batched tile kernel");
                return PD_EOVERFLOW;
            }
            s->rebuilds++;
            changed = true;
        }
        if (s->hdesc[k].skip_replay != reb) changed = true;
        s->hdesc[k].skip_replay = reb;
    }
    if (changed || s->dirty) PD_TRY(upload_tables(s));
    PD_CUDA(cudaGraphLaunch(s->gB, s->st));
    s->replays++;
    __atomic_fetch_add(&g_launches, 5ull, __ATOMIC_RELAXED);  // kernels of the two graphs
    PD_CUDA(cudaStreamSynchronize(s->st));
    // retirement
    std::vector<SrvReq*> keep;
    for (SrvReq* r : s->active) {
        r->md->steps++;
        s->particle_steps += r->n;
        if (r->md->steps >= r->steps) {
            PD_TRY(retire(s, r));
            s->dirty = true;
        } else {
            keep.push_back(r);
        }
    }
    if (keep.size() != s->active.size()) {
        // keep the replay flags aligned with the surviving systems
        std::vector<SysDesc> nd;
        for (size_t k = 0; k < s->active.size(); ++k)
            if (s->active[k]->state == 1) nd.push_back(s->hdesc[k]);
        s->hdesc = nd;
    }
    s->active.swap(keep);
    if (n_active) *n_active = (int)s->active.size();
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
    if (x_out) memcpy(x_out, r->xo.data(), sizeof(double) * r->xo.size());
    if (E_out) memcpy(E_out, r->E.data(), sizeof(double) * r->E.size());
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
    s->reqs.erase(it);
    return PD_OK;
}

int pd_srv_stats(pd_srv s, long* particle_steps, long* systems_done, long* ticks, long* rebuilds, double* tune_ms) {
    if (!s) return PD_EINVAL;
    if (particle_steps) *particle_steps = s->particle_steps;
    if (systems_done) *systems_done = s->systems_done;
    if (ticks) *ticks = s->replays;
    if (rebuilds) *rebuilds = s->rebuilds;
    if (tune_ms) *tune_ms = s->tune_ms;
    return PD_OK;
}

int pd_srv_tuned(pd_srv s, int* buckets, int* widths, int cap, int* n) {
    if (!s || !n) return PD_EINVAL;
    int k = 0;
    for (auto& kv : s->tuned) {
        if (k < cap) {
            if (buckets) buckets[k] = kv.first;
            if (widths) widths[k] = kv.second;
        }
        ++k;
    }
    *n = k;
    return PD_OK;
}

}  // extern "C"
