// pd_core.cu -- particle storage (vector_dist on one GPU), host<->device copies,
// map (periodic wrap), kernel views, reductions, the device-wide scan.
//
// Storage layout in HBM (one vector = one pd_vd):
//   pos    float4/double4 records (x, y, z, unused) -- one 16/32-byte sector per
//          particle so neighbour gathers in the pair kernels touch one sector;
//   gid    int32 original index of the particle held by each slot;
//   props  one allocation per property, component-major [ncomp][cap].
// Real particles occupy [0, n_real) (the reference's ghostMarker), periodic
// images [n_real, n_total).
#include <algorithm>
#include <cstdarg>
#include <map>
#include <mutex>
#include <unordered_map>

#include "pd_device.cuh"
#include "pd_internal.cuh"

namespace pd {

static thread_local std::string g_err;
unsigned long long g_launches = 0;

void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
}

int check_device_ptr(const void* p, const char* who, const char* what) {
    int dev = -1;
    cudaPointerAttributes at;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        set_error("%s: %s is not a pointer the CUDA runtime knows", who, what);
        return PD_EINVAL;
    }
    if (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged) {
        set_error("%s: %s must be device memory, not host memory", who, what);
        return PD_EINVAL;
    }
    if (at.type == cudaMemoryTypeDevice && at.device != dev) {
        set_error("%s: %s is memory of device %d, the current device is %d", who, what, at.device, dev);
        return PD_EINVAL;
    }
    return PD_OK;
}

thread_local AllocCtx* g_alloc_ctx = nullptr;

// Device allocations of the library.  Inside an AllocScope (the serving loop) they
// come from the scope's memory pool, ordered on the scope's stream (freed memory
// is reused without a device-wide synchronisation).  Elsewhere from cudaMalloc
// through a bounded block cache: a freed block is kept (up to the cache limit,
// 4 GiB by default) and handed out again for a request of 1/2 to 1 times its size.
// cudaFree synchronises the device; the cache keeps that guarantee by
// synchronising once before a block freed since the last synchronisation is
// reused, so no kernel of the block's previous owner can still be running.
// Creating and destroying vectors one after another then costs no
// cudaMalloc / cudaFree (each of which took milliseconds for large blocks).
// A cudaMalloc that fails empties the cache and is tried once more.
thread_local bool g_capturing = false;  // set around the library's own stream captures

namespace {
struct BlockCache {
    struct Block {
        size_t bytes;
        int dev;
    };
    std::mutex mu;
    std::multimap<std::pair<int, size_t>, void*> free_blocks;  // by (device, size)
    std::unordered_map<void*, Block> block_of;                 // every block from cudaMalloc on this path
    size_t held = 0;
    size_t limit = (size_t)4 << 30;
    std::unordered_map<int, bool> dirty;  // per device: blocks freed since its last synchronisation

    // return every cached block to the driver (caller holds mu)
    void drain() {
        if (free_blocks.empty()) return;
        int cur = 0;
        cudaGetDevice(&cur);
        int dev = -1;
        for (auto& kv : free_blocks) {
            if (kv.first.first != dev) {
                dev = kv.first.first;
                cudaSetDevice(dev);
                cudaDeviceSynchronize();
            }
            block_of.erase(kv.second);
            cudaFree(kv.second);
        }
        cudaSetDevice(cur);
        free_blocks.clear();
        held = 0;
        dirty.clear();
    }
};
BlockCache& block_cache() {
    static BlockCache* c = new BlockCache();  // never destroyed: no CUDA calls at process exit
    return *c;
}
size_t block_round(size_t b) {
    return b <= ((size_t)1 << 20) ? ((b + 511) & ~(size_t)511) : ((b + ((size_t)2 << 20) - 1) & ~(((size_t)2 << 20) - 1));
}
}  // namespace

cudaError_t dev_alloc(void** p, size_t b) {
    if (g_alloc_ctx) return cudaMallocFromPoolAsync(p, b, g_alloc_ctx->pool, g_alloc_ctx->st);
    if (g_capturing) return cudaMalloc(p, b);
    const size_t rb = block_round(b);
    int dev = 0;
    cudaGetDevice(&dev);
    BlockCache& C = block_cache();
    std::lock_guard<std::mutex> lk(C.mu);
    auto it = C.free_blocks.lower_bound({dev, rb});
    if (it != C.free_blocks.end() && it->first.first == dev && it->first.second <= 2 * rb) {
        if (C.dirty[dev]) {
            cudaError_t e = cudaDeviceSynchronize();
            if (e != cudaSuccess) return e;
            C.dirty[dev] = false;
        }
        *p = it->second;
        C.held -= it->first.second;
        C.free_blocks.erase(it);
        return cudaSuccess;
    }
    cudaError_t e = cudaMalloc(p, rb);
    if (e == cudaErrorMemoryAllocation && !C.free_blocks.empty()) {
        cudaGetLastError();
        C.drain();
        e = cudaMalloc(p, rb);
    }
    if (e == cudaSuccess) C.block_of[*p] = {rb, dev};
    return e;
}

void dev_free(void* p) {
    if (!p) return;
    if (g_alloc_ctx) {
        cudaFreeAsync(p, g_alloc_ctx->st);
        return;
    }
    BlockCache& C = block_cache();
    std::lock_guard<std::mutex> lk(C.mu);
    auto it = C.block_of.find(p);
    if (it == C.block_of.end() || g_capturing || C.held + it->second.bytes > C.limit) {
        if (it != C.block_of.end()) C.block_of.erase(it);
        cudaFree(p);
        return;
    }
    C.free_blocks.insert({{it->second.dev, it->second.bytes}, p});
    C.held += it->second.bytes;
    C.dirty[it->second.dev] = true;
}

int Buf::ensure(size_t b) {
    if (b <= bytes && p) return PD_OK;
    // a buffer that has to grow grows by a quarter at least: sizes that creep up
    // from one rebuild to the next (images, rows, staging) reallocate rarely, and a
    // reallocation outside a stream-ordered pool synchronises the device
    if (p && bytes > 0) b = std::max(b, bytes + bytes / 4);
    dev_free(p);
    p = nullptr;
    bytes = 0;
    if (b == 0) return PD_OK;
    cudaError_t e = dev_alloc(&p, b);
    if (e != cudaSuccess) {
        p = nullptr;
        set_error("cudaMalloc(%zu): %s", b, cudaGetErrorString(e));
        cudaGetLastError();
        return PD_ENOMEM;
    }
    bytes = b;
    return PD_OK;
}

void Buf::release() {
    dev_free(p);
    p = nullptr;
    bytes = 0;
}

// ---------------------------------------------------------------------------
// exclusive scan (3 phases: per-block sums, scan of the block sums in one block,
// per-block scan plus offset).  Deterministic; n up to 2^31.
static constexpr int SCAN_BLOCK = 512;
static constexpr int SCAN_ITEMS = 8;
static constexpr int SCAN_TILE = SCAN_BLOCK * SCAN_ITEMS;

__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_reduce(const unsigned int* __restrict__ in, long n,
                                                            unsigned int* __restrict__ part) {
    long base = (long)blockIdx.x * SCAN_TILE;
    unsigned int s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        long i = base + (long)k * SCAN_BLOCK + threadIdx.x;
        if (i < n) s += in[i];
    }
    s = block_sum<unsigned int, SCAN_BLOCK>(s);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// single block: exclusive scan of nb partials in place, total to *total
__global__ void __launch_bounds__(1024) k_scan_partials(unsigned int* part, long nb, unsigned int* total) {
    __shared__ unsigned int wsum[32];
    __shared__ unsigned int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (long base = 0; base < nb; base += 1024) {
        long i = base + threadIdx.x;
        unsigned int v = (i < nb) ? part[i] : 0u;
        unsigned int x = v;
        int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[w] = x;
        __syncthreads();
        if (w == 0) {
            unsigned int y = wsum[lane];
            unsigned int z = y;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                unsigned int t = __shfl_up_sync(0xffffffffu, z, o);
                if (lane >= o) z += t;
            }
            wsum[lane] = z - y;  // exclusive warp offsets
        }
        __syncthreads();
        unsigned int excl = carry + wsum[w] + x - v;
        if (i < nb) part[i] = excl;
        __syncthreads();
        if (threadIdx.x == 1023) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_apply(const unsigned int* __restrict__ in, long n,
                                                           const unsigned int* __restrict__ part,
                                                           unsigned int* __restrict__ out) {
    __shared__ unsigned int wsum[SCAN_BLOCK / 32];
    long base = (long)blockIdx.x * SCAN_TILE;
    // each thread owns SCAN_ITEMS consecutive elements
    long i0 = base + (long)threadIdx.x * SCAN_ITEMS;
    unsigned int v[SCAN_ITEMS];
    unsigned int s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        v[k] = (i0 + k < n) ? in[i0 + k] : 0u;
        s += v[k];
    }
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned int x = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
        unsigned int y = (lane < SCAN_BLOCK / 32) ? wsum[lane] : 0u;
        unsigned int z = y;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned int t = __shfl_up_sync(0xffffffffu, z, o);
            if (lane >= o) z += t;
        }
        if (lane < SCAN_BLOCK / 32) wsum[lane] = z - y;
    }
    __syncthreads();
    unsigned int run = part[blockIdx.x] + wsum[w] + x - s;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        if (i0 + k < n) out[i0 + k] = run;
        run += v[k];
    }
}

int scan_partials(unsigned int* part, long nb, unsigned int* total_dev, cudaStream_t st) {
    if (nb <= 0) return PD_OK;
    pd::launch(k_scan_partials, 1, 1024, 0, st, part, nb, total_dev);
    PD_LAUNCH_CHECK();
    return PD_OK;
}

int scan_u32(const unsigned int* in, unsigned int* out, long n, unsigned int* total_dev, Buf& scratch,
             cudaStream_t st) {
    if (n <= 0) {
        if (total_dev) PD_CUDA(cudaMemsetAsync(total_dev, 0, sizeof(unsigned int), st));
        return PD_OK;
    }
    long nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    PD_TRY(scratch.ensure(sizeof(unsigned int) * (nb + 1)));
    unsigned int* part = scratch.as<unsigned int>();
    pd::launch(k_scan_reduce, (unsigned)nb, SCAN_BLOCK, 0, st, in, n, part);
    pd::launch(k_scan_partials, 1, 1024, 0, st, part, nb, total_dev);
    pd::launch(k_scan_apply, (unsigned)nb, SCAN_BLOCK, 0, st, in, n, part, out);
    PD_LAUNCH_CHECK();
    return PD_OK;
}

// ---------------------------------------------------------------------------
// storage

template <class T>
__global__ void k_expand_pos(const T* __restrict__ xyz, long n, typename V4<T>::type* __restrict__ pos, long off) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        typename V4<T>::type r;
        r.x = xyz[3 * i];
        r.y = xyz[3 * i + 1];
        r.z = xyz[3 * i + 2];
        r.w = T(0);
        st4(pos, off + i, r);
    }
}

template <class T>
__global__ void k_pack_pos(const typename V4<T>::type* __restrict__ pos, long off, long n, T* __restrict__ xyz) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        typename V4<T>::type r = ld4(pos, off + i);
        xyz[3 * i] = r.x;
        xyz[3 * i + 1] = r.y;
        xyz[3 * i + 2] = r.z;
    }
}

__global__ void k_iota(int* g, long off, long n) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        g[off + i] = (int)(off + i);
}

// grow every per-particle array to hold `need` particles, keeping [0, n_total)
int alloc_storage(pd_vd h, long cap, void** pos, int** gid, std::vector<char*>& props) {
    *pos = nullptr;
    *gid = nullptr;
    props.assign(h->props.size(), nullptr);
    bool ok = dev_alloc(pos, (size_t)cap * h->pos_bytes) == cudaSuccess &&
              dev_alloc((void**)gid, sizeof(int) * cap) == cudaSuccess;
    for (size_t p = 0; ok && p < h->props.size(); ++p)
        ok = dev_alloc((void**)&props[p], (size_t)h->props[p].esize * h->props[p].ncomp * cap) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        free_storage(*pos, *gid, props);
        *pos = nullptr;
        *gid = nullptr;
        set_error("cudaMalloc failed for the storage of %ld particles", cap);
        return PD_ENOMEM;
    }
    return PD_OK;
}

void free_storage(void* pos, int* gid, const std::vector<char*>& props) {
    dev_free(pos);
    dev_free(gid);
    for (char* p : props) dev_free(p);
}

int ensure_capacity(pd_vd h, long need, cudaStream_t st) {
    if (need <= h->cap) return PD_OK;
    long ncap = need + need / 4 + 1024;
    void* np = nullptr;
    int* ng = nullptr;
    std::vector<char*> nprops;
    PD_TRY(alloc_storage(h, ncap, &np, &ng, nprops));
    if (h->pos && h->n_total) {
        PD_CUDA(cudaMemcpyAsync(np, h->pos, (size_t)h->n_total * h->pos_bytes, cudaMemcpyDeviceToDevice, st));
        PD_CUDA(cudaMemcpyAsync(ng, h->gid, sizeof(int) * h->n_total, cudaMemcpyDeviceToDevice, st));
    }
    for (size_t p = 0; p < h->props.size(); ++p) {
        Prop& P = h->props[p];
        if (P.d && h->n_total)
            for (int c = 0; c < P.ncomp; ++c)
                PD_CUDA(cudaMemcpyAsync(nprops[p] + (size_t)c * ncap * P.esize, P.d + (size_t)c * h->cap * P.esize,
                                        (size_t)h->n_total * P.esize, cudaMemcpyDeviceToDevice, st));
    }
    PD_CUDA(cudaStreamSynchronize(st));
    dev_free(h->pos);
    dev_free(h->gid);
    for (size_t p = 0; p < h->props.size(); ++p) {
        dev_free(h->props[p].d);
        h->props[p].d = nprops[p];
    }
    // a spare of the old capacity no longer fits
    free_storage(h->spare_pos, h->spare_gid, h->spare_props);
    h->spare_pos = nullptr;
    h->spare_gid = nullptr;
    h->spare_props.clear();
    h->spare_cap = 0;
    h->pos = np;
    h->gid = ng;
    h->cap = ncap;
    h->epoch++;
    return PD_OK;
}

int set_ctrl_n_img(pd_vd h, long n_img, cudaStream_t st) {
    h->ctrl_h->n_img = (unsigned int)n_img;
    PD_CUDA(cudaMemcpyAsync(&h->ctrl->n_img, &h->ctrl_h->n_img, sizeof(unsigned int), cudaMemcpyHostToDevice, st));
    return PD_OK;
}

int read_ctrl(pd_vd h, cudaStream_t st) {
    PD_CUDA(cudaMemcpyAsync(h->ctrl_h, h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
    PD_CUDA(cudaStreamSynchronize(st));
    return PD_OK;
}

template <class T>
__global__ void k_wrap(typename V4<T>::type* __restrict__ pos, long n, T lo0, T lo1, T lo2, T hi0, T hi1, T hi2,
                       int per0, int per1, int per2) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        typename V4<T>::type r = ld4(pos, i);
        if (per0) r.x = periodic_l(r.x, hi0, lo0);
        if (per1) r.y = periodic_l(r.y, hi1, lo1);
        if (per2) r.z = periodic_l(r.z, hi2, lo2);
        st4(pos, i, r);
    }
}

int wrap_positions(pd_vd h, long n, cudaStream_t st) {
    if (n <= 0) return PD_OK;
    unsigned g = grid_for(n, 256);
    if (h->dtype == PD_F64)
        pd::launch(k_wrap<double>, g, 256, 0, st, (double4*)h->pos, n, h->lo[0], h->lo[1], h->lo[2], h->hi[0], h->hi[1],
                                          h->hi[2], h->bc[0] == PD_PERIODIC, h->bc[1] == PD_PERIODIC,
                                          h->bc[2] == PD_PERIODIC);
    else
        pd::launch(k_wrap<float>, g, 256, 0, st, (float4*)h->pos, n, (float)h->lo[0], (float)h->lo[1], (float)h->lo[2],
                                         (float)h->hi[0], (float)h->hi[1], (float)h->hi[2], h->bc[0] == PD_PERIODIC,
                                         h->bc[1] == PD_PERIODIC, h->bc[2] == PD_PERIODIC);
    PD_LAUNCH_CHECK();
    return PD_OK;
}

// reductions over [0, n) of one component (reduce_local)
template <class T, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_reduce(const T* __restrict__ x, long n, int op, double* __restrict__ part) {
    double acc = (op == PD_RED_ADD) ? 0.0 : -1.0 / 0.0;
    for (long i = blockIdx.x * (long)BLOCK + threadIdx.x; i < n; i += (long)gridDim.x * BLOCK) {
        double v = (double)x[i];
        acc = (op == PD_RED_ADD) ? acc + v : fmax(acc, v);
    }
    __shared__ double sh[BLOCK];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = BLOCK / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            sh[threadIdx.x] = (op == PD_RED_ADD) ? sh[threadIdx.x] + sh[threadIdx.x + s]
                                                 : fmax(sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

}  // namespace pd

using namespace pd;

// ---------------------------------------------------------------------------
extern "C" {

const char* pd_last_error(void) { return g_err.c_str(); }

unsigned long long pd_launch_count(void) { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }

int pd_empty_cache(void) {
    BlockCache& C = block_cache();
    std::lock_guard<std::mutex> lk(C.mu);
    C.drain();
    return PD_OK;
}

int pd_set_cache_limit(long bytes, long* held) {
    BlockCache& C = block_cache();
    std::lock_guard<std::mutex> lk(C.mu);
    if (bytes >= 0) {
        C.limit = (size_t)bytes;
        if (C.held > C.limit) C.drain();
    }
    if (held) *held = (long)C.held;
    return PD_OK;
}

int pd_device_info(int* sm_count, long* free_bytes, long* total_bytes) {
    int dev = 0;
    PD_CUDA(cudaGetDevice(&dev));
    if (sm_count) PD_CUDA(cudaDeviceGetAttribute(sm_count, cudaDevAttrMultiProcessorCount, dev));
    size_t f = 0, t = 0;
    PD_CUDA(cudaMemGetInfo(&f, &t));
    if (free_bytes) *free_bytes = (long)f;
    if (total_bytes) *total_bytes = (long)t;
    return PD_OK;
}

int pd_create(int dim, int dtype, long n, const double* lo, const double* hi, const int* bc, const double* ghost,
              int opts, pd_vd* out) {
    (void)opts;
    if (!out || dim != 3 || (dtype != PD_F32 && dtype != PD_F64) || n < 0 || !lo || !hi || !bc || !ghost) {
        set_error("pd_create: invalid argument (dim must be 3, dtype PD_F32/PD_F64)");
        return PD_EINVAL;
    }
    for (int d = 0; d < 3; ++d) {
        if (!(hi[d] > lo[d]) || ghost[d] < 0 || (bc[d] != PD_PERIODIC && bc[d] != PD_NON_PERIODIC)) {
            set_error("pd_create: invalid box/ghost/bc in dimension %d", d);
            return PD_EINVAL;
        }
    }
    pd_vd h = new pd_vd_s();
    h->dtype = dtype;
    h->pos_bytes = dtype == PD_F64 ? 32 : 16;
    for (int d = 0; d < 3; ++d) {
        h->lo[d] = lo[d];
        h->hi[d] = hi[d];
        h->g[d] = ghost[d];
        h->bc[d] = bc[d];
    }
    if (cudaMalloc(&h->ctrl, sizeof(Ctrl)) != cudaSuccess || cudaMallocHost(&h->ctrl_h, sizeof(Ctrl)) != cudaSuccess) {
        cudaGetLastError();
        set_error("pd_create: control block allocation failed");
        delete h;
        return PD_ENOMEM;
    }
    memset(h->ctrl_h, 0, sizeof(Ctrl));
    cudaMemset(h->ctrl, 0, sizeof(Ctrl));
    int r = ensure_capacity(h, n > 0 ? n : 1, 0);
    if (r != PD_OK) {
        pd_destroy(h);
        return r;
    }
    h->n_real = h->n_total = n;
    if (n > 0) {
        pd::launch(k_iota, grid_for(n, 256), 256, 0, (cudaStream_t)0, h->gid, 0L, n);
        if (cudaGetLastError() != cudaSuccess) {
            pd_destroy(h);
            return PD_ECUDA;
        }
        cudaMemset(h->pos, 0, (size_t)n * h->pos_bytes);
    }
    *out = h;
    return PD_OK;
}

int pd_destroy(pd_vd h) {
    if (!h) return PD_EINVAL;
    dev_free(h->pos);
    dev_free(h->gid);
    for (auto& P : h->props) dev_free(P.d);
    free_storage(h->spare_pos, h->spare_gid, h->spare_props);
    h->img_src.release();
    h->img_shift.release();
    h->img_cnt.release();
    h->img_start.release();
    h->boxes.release();
    h->box_sv.release();
    h->shifts.release();
    h->scan_scratch.release();
    h->tmp.release();
    h->tmp2.release();
    h->red.release();
    if (h->ctrl) cudaFree(h->ctrl);
    if (h->ctrl_h) cudaFreeHost(h->ctrl_h);
    delete h;
    return PD_OK;
}

int pd_add_prop(pd_vd h, int type, int ncomp, int* prop_id) {
    if (!h || type_size(type) == 0 || ncomp < 1 || ncomp > 64 || h->props.size() >= 16) {
        set_error("pd_add_prop: invalid argument");
        return PD_EINVAL;
    }
    Prop P;
    P.type = type;
    P.ncomp = ncomp;
    P.esize = type_size(type);
    PD_CUDA(dev_alloc((void**)&P.d, (size_t)P.esize * ncomp * h->cap));
    PD_CUDA(cudaMemset(P.d, 0, (size_t)P.esize * ncomp * h->cap));
    h->props.push_back(P);
    if (prop_id) *prop_id = (int)h->props.size() - 1;
    h->epoch++;
    return PD_OK;
}

int pd_size(pd_vd h, long* size_local, long* size_with_ghost) {
    if (!h) return PD_EINVAL;
    if (size_local) *size_local = h->n_real;
    if (size_with_ghost) *size_with_ghost = h->n_total;
    return PD_OK;
}

int pd_resize(pd_vd h, long n) {
    if (!h || n < 0) return PD_EINVAL;
    long old = h->n_real;
    PD_TRY(ensure_capacity(h, n > 0 ? n : 1, 0));
    if (n > old) {
        pd::launch(k_iota, grid_for(n - old, 256), 256, 0, (cudaStream_t)0, h->gid, old, n - old);
        PD_LAUNCH_CHECK();
    }
    h->n_real = h->n_total = n;
    h->img_valid = false;
    h->epoch++;
    return PD_OK;
}

int pd_h2d_pos(pd_vd h, const void* host_xyz, long offset, long count, void* stream) {
    if (!h || !host_xyz || offset < 0 || count < 0 || offset + count > h->n_total) {
        set_error("pd_h2d_pos: range [%ld,%ld) outside size %ld", offset, offset + count, h ? h->n_total : 0);
        return PD_EINVAL;
    }
    if (count == 0) return PD_OK;
    cudaStream_t st = S(stream);
    size_t es = h->dtype == PD_F64 ? 8 : 4;
    PD_TRY(h->tmp.ensure(es * 3 * count));
    PD_CUDA(cudaMemcpyAsync(h->tmp.p, host_xyz, es * 3 * count, cudaMemcpyDefault, st));  // host or device source
    unsigned g = grid_for(count, 256);
    if (h->dtype == PD_F64)
        pd::launch(k_expand_pos<double>, g, 256, 0, st, h->tmp.as<double>(), count, (double4*)h->pos, offset);
    else
        pd::launch(k_expand_pos<float>, g, 256, 0, st, h->tmp.as<float>(), count, (float4*)h->pos, offset);
    PD_LAUNCH_CHECK();
    return PD_OK;
}

int pd_d2h_pos(pd_vd h, void* host_xyz, long offset, long count, void* stream) {
    if (!h || !host_xyz || offset < 0 || count < 0 || offset + count > h->n_total) {
        set_error("pd_d2h_pos: bad range");
        return PD_EINVAL;
    }
    if (count == 0) return PD_OK;
    cudaStream_t st = S(stream);
    size_t es = h->dtype == PD_F64 ? 8 : 4;
    PD_TRY(h->tmp.ensure(es * 3 * count));
    unsigned g = grid_for(count, 256);
    if (h->dtype == PD_F64)
        pd::launch(k_pack_pos<double>, g, 256, 0, st, (const double4*)h->pos, offset, count, h->tmp.as<double>());
    else
        pd::launch(k_pack_pos<float>, g, 256, 0, st, (const float4*)h->pos, offset, count, h->tmp.as<float>());
    PD_LAUNCH_CHECK();
    PD_CUDA(cudaMemcpyAsync(host_xyz, h->tmp.p, es * 3 * count, cudaMemcpyDefault, st));  // host or device target
    PD_CUDA(cudaStreamSynchronize(st));
    return PD_OK;
}

int pd_h2d_prop(pd_vd h, int prop, const void* host, long offset, long count, void* stream) {
    if (!h || prop < 0 || prop >= (int)h->props.size() || !host || offset < 0 || count < 0 ||
        offset + count > h->n_total) {
        set_error("pd_h2d_prop: bad argument");
        return PD_EINVAL;
    }
    Prop& P = h->props[prop];
    cudaStream_t st = S(stream);
    for (int c = 0; c < P.ncomp; ++c)
        PD_CUDA(cudaMemcpyAsync(P.d + ((size_t)c * h->cap + offset) * P.esize,
                                (const char*)host + (size_t)c * count * P.esize, (size_t)count * P.esize,
                                cudaMemcpyDefault, st));  // host or device source
    return PD_OK;
}

int pd_d2h_prop(pd_vd h, int prop, void* host, long offset, long count, void* stream) {
    if (!h || prop < 0 || prop >= (int)h->props.size() || !host || offset < 0 || count < 0 ||
        offset + count > h->n_total) {
        set_error("pd_d2h_prop: bad argument");
        return PD_EINVAL;
    }
    Prop& P = h->props[prop];
    cudaStream_t st = S(stream);
    for (int c = 0; c < P.ncomp; ++c)
        PD_CUDA(cudaMemcpyAsync((char*)host + (size_t)c * count * P.esize,
                                P.d + ((size_t)c * h->cap + offset) * P.esize, (size_t)count * P.esize,
                                cudaMemcpyDefault, st));  // host or device target
    PD_CUDA(cudaStreamSynchronize(st));
    return PD_OK;
}

int pd_d2h_gid(pd_vd h, long* host, long offset, long count, void* stream) {
    if (!h || !host || offset < 0 || count < 0 || offset + count > h->n_total) return PD_EINVAL;
    std::vector<int> tmp(count);
    cudaStream_t st = S(stream);
    if (count) {
        PD_CUDA(cudaMemcpyAsync(tmp.data(), h->gid + offset, sizeof(int) * count, cudaMemcpyDeviceToHost, st));
        PD_CUDA(cudaStreamSynchronize(st));
    }
    for (long i = 0; i < count; ++i) host[i] = tmp[i];
    return PD_OK;
}

int pd_map(pd_vd h, int opt, void* stream) {
    (void)opt;
    if (!h) return PD_EINVAL;
    if (h->ghost_pending) {
        set_error("map: an Ighost_get is waiting for its ghost_wait");
        return PD_ESTATE;
    }
    // drop the ghost (vector_dist_comm.hpp:1969-1970), wrap (apply_bc_each_part)
    h->n_total = h->n_real;
    h->img_valid = false;
    PD_TRY(wrap_positions(h, h->n_real, S(stream)));
    h->epoch++;
    return PD_OK;
}

int pd_view(pd_vd h, pd_view_t* out) {
    if (!h || !out) return PD_EINVAL;
    memset(out, 0, sizeof(*out));
    out->pos = h->pos;
    out->n_prop = (int)h->props.size();
    for (size_t p = 0; p < h->props.size(); ++p) {
        out->prop[p] = h->props[p].d;
        out->prop_type[p] = h->props[p].type;
        out->prop_ncomp[p] = h->props[p].ncomp;
    }
    out->dtype = h->dtype;
    out->stride = h->cap;
    out->size_local = h->n_real;
    out->size = h->n_total;
    out->epoch = h->epoch;
    return PD_OK;
}

int pd_domain_iterator(pd_vd h, int n_thr, int with_ghost, pd_launch_t* out) {
    if (!h || !out || n_thr <= 0 || n_thr > 1024) return PD_EINVAL;
    long n = with_ghost ? h->n_total : h->n_real;
    out->thr[0] = n_thr;
    out->thr[1] = out->thr[2] = 1;
    out->wthr[0] = (unsigned)((n + n_thr - 1) / n_thr);
    if (out->wthr[0] == 0) out->wthr[0] = 1;
    out->wthr[1] = out->wthr[2] = 1;
    return PD_OK;
}

int pd_reduce(pd_vd h, int prop, int comp, int op, void* stream, double* out) {
    if (!h || !out || prop < 0 || prop >= (int)h->props.size() || (op != PD_RED_ADD && op != PD_RED_MAX)) return PD_EINVAL;
    Prop& P = h->props[prop];
    if (comp < 0 || comp >= P.ncomp) return PD_EINVAL;
    cudaStream_t st = S(stream);
    long n = h->n_real;
    if (n == 0) {
        *out = (op == PD_RED_ADD) ? 0.0 : -1.0 / 0.0;
        return PD_OK;
    }
    unsigned g = grid_for(n, 256, 296);
    PD_TRY(h->red.ensure(sizeof(double) * g));
    const char* base = P.d + (size_t)comp * h->cap * P.esize;
    switch (P.type) {
        case PD_F64: pd::launch(k_reduce<double, 256>, g, 256, 0, st, (const double*)base, n, op, h->red.as<double>()); break;
        case PD_F32: pd::launch(k_reduce<float, 256>, g, 256, 0, st, (const float*)base, n, op, h->red.as<double>()); break;
        case PD_I32: pd::launch(k_reduce<int, 256>, g, 256, 0, st, (const int*)base, n, op, h->red.as<double>()); break;
        case PD_U32: pd::launch(k_reduce<unsigned int, 256>, g, 256, 0, st, (const unsigned int*)base, n, op, h->red.as<double>()); break;
        case PD_I64: pd::launch(k_reduce<long long, 256>, g, 256, 0, st, (const long long*)base, n, op, h->red.as<double>()); break;
    }
    PD_LAUNCH_CHECK();
    std::vector<double> part(g);
    PD_CUDA(cudaMemcpyAsync(part.data(), h->red.p, sizeof(double) * g, cudaMemcpyDeviceToHost, st));
    PD_CUDA(cudaStreamSynchronize(st));
    double acc = (op == PD_RED_ADD) ? 0.0 : -1.0 / 0.0;
    for (unsigned i = 0; i < g; ++i) acc = (op == PD_RED_ADD) ? acc + part[i] : std::max(acc, part[i]);
    *out = acc;
    return PD_OK;
}

}  // extern "C"
