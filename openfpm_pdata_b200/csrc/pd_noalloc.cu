// pd_noalloc.cu -- cell-list counting sort that allocates no device memory.
//
// pd_celllist_update grows its scratch buffers with cudaMalloc on demand.  Some
// callers cannot allow that: real-time or plugin hosts whose device memory is
// owned by a pool of the host application (the plugin gets a budget, not the
// allocator), and callers that must not let cudaMalloc/cudaFree synchronise the
// device under running work.  For them this entry point sorts particles into
// cells using a file-scope __device__ array as its only scratch; the caller
// passes inputs and outputs.
//
// The scratch array is part of the library's device image: every GPU that
// loads the library holds it (about 8.4 MB) until the process exits.  Its
// device address is looked up once per device with cudaGetSymbolAddress the
// first time the entry point runs with that device current; that first call
// should therefore come before any stream capture.  All calls share the one
// array and it keeps the last call's contents (the counts are cleared on every
// call), so calls that overlap on the GPU -- on different streams, or from
// different host threads -- race and must be serialised by the caller.  A
// position that is NaN or outside the grid is clamped into a border cell, as in
// pd_celllist_update; the optional caller-owned device word `status` is cleared
// and then receives PD_STATIC_OUT_OF_GRID for such a call (read it after the
// stream's work: nothing here synchronises).  Pointers are checked to be device
// memory of the current device before any launch.
#include <mutex>

#include "pd_device.cuh"
#include "pd_internal.cuh"

namespace pd {
namespace noalloc {

static constexpr long MAX_PART = 1L << 19;   // particles per call
static constexpr long MAX_CELLS = 1L << 19;  // cells (including padding) per call
static constexpr int BLOCK = 256;
static constexpr int TILE = 2048;            // scan elements per block
static constexpr long MAX_PARTS = (MAX_CELLS + 1 + TILE - 1) / TILE + 1;
// layout (uint32 words): counts[MAX_CELLS+1] | cell_of[MAX_PART] | slot[MAX_PART] | tmp[MAX_PART] | parts[MAX_PARTS]
static constexpr long OFF_CELL_OF = MAX_CELLS + 1;
static constexpr long OFF_SLOT = OFF_CELL_OF + MAX_PART;
static constexpr long OFF_TMP = OFF_SLOT + MAX_PART;
static constexpr long OFF_PARTS = OFF_TMP + MAX_PART;
static constexpr long WORDS = OFF_PARTS + MAX_PARTS;

static __device__ __align__(256) unsigned int g_scratch[WORDS];

static std::mutex g_mu;
static unsigned int* g_addr[256] = {};

// device address of g_scratch for the current device (looked up once per device)
static int scratch_address(unsigned int** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 256) {
        set_error("pd_celllist_build_static: no current CUDA device (%s)", cudaGetErrorString(e));
        return PD_ECUDA;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p) {
            set_error("pd_celllist_build_static: cudaGetSymbolAddress failed (%s)", cudaGetErrorString(e));
            return PD_ECUDA;
        }
        g_addr[dev] = static_cast<unsigned int*>(p);
    }
    *out = g_addr[dev];
    return PD_OK;
}

__global__ void k_zero(unsigned int* a, long n) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) a[i] = 0u;
}

template <class T>
__global__ void k_hash_xyz(const T* __restrict__ xyz, long n, Grid<T> G, unsigned int* __restrict__ cnt,
                           unsigned int* __restrict__ cell_of, unsigned int* __restrict__ slot,
                           unsigned int* __restrict__ status) {
    unsigned int bad = 0;
    for (long base = blockIdx.x * (long)blockDim.x; base < n; base += (long)gridDim.x * blockDim.x) {
        long i = base + threadIdx.x;
        bool ok = i < n;
        unsigned int act = __ballot_sync(0xffffffffu, ok);
        if (ok) {
            unsigned int c = (unsigned int)G.cell(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], bad);
            cell_of[i] = c;
            slot[i] = warp_agg_inc(cnt, c, act);
        }
    }
    if (bad && status) atomicOr(status, PD_STATIC_OUT_OF_GRID);
}

// scan of m counts: per-block totals, exclusive scan of the totals in one block, apply
__global__ void __launch_bounds__(BLOCK) k_block_tot(const unsigned int* __restrict__ in, long m,
                                                     unsigned int* __restrict__ parts) {
    long b = (long)blockIdx.x * TILE;
    unsigned int s = 0;
    for (int k = threadIdx.x; k < TILE; k += BLOCK)
        if (b + k < m) s += in[b + k];
    s = block_sum<unsigned int, BLOCK>(s);
    if (threadIdx.x == 0) parts[blockIdx.x] = s;
}

__global__ void k_tot_scan(unsigned int* parts, long nb) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        unsigned int run = 0;
        for (long i = 0; i < nb; ++i) {
            unsigned int v = parts[i];
            parts[i] = run;
            run += v;
        }
    }
}

__global__ void __launch_bounds__(BLOCK) k_apply(const unsigned int* __restrict__ in, long m,
                                                 const unsigned int* __restrict__ parts, int* __restrict__ out) {
    __shared__ unsigned int wsum[BLOCK / 32];
    __shared__ unsigned int carry;
    long b = (long)blockIdx.x * TILE;
    if (threadIdx.x == 0) carry = parts[blockIdx.x];
    __syncthreads();
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int k0 = 0; k0 < TILE; k0 += BLOCK) {
        long i = b + k0 + threadIdx.x;
        unsigned int v = i < m ? in[i] : 0u;
        unsigned int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[w] = x;
        __syncthreads();
        if (w == 0) {
            unsigned int y = lane < BLOCK / 32 ? wsum[lane] : 0u;
            unsigned int z = y;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                unsigned int t = __shfl_up_sync(0xffffffffu, z, o);
                if (lane >= o) z += t;
            }
            if (lane < BLOCK / 32) wsum[lane] = z - y;
        }
        __syncthreads();
        unsigned int excl = carry + wsum[w] + x - v;
        if (i < m) out[i] = (int)excl;
        __syncthreads();
        if (threadIdx.x == BLOCK - 1) carry = excl + v;
        __syncthreads();
    }
}

__global__ void k_scatter(long n, const unsigned int* __restrict__ cell_of, const unsigned int* __restrict__ slot,
                          const int* __restrict__ start, unsigned int* __restrict__ tmp) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        tmp[start[cell_of[i]] + slot[i]] = (unsigned int)i;
}

// one warp per cell: members in ascending index order (stable in-cell order)
__global__ void __launch_bounds__(BLOCK) k_stabilise(long ncells, const int* __restrict__ start,
                                                     const unsigned int* __restrict__ in, int* __restrict__ out) {
    __shared__ int cell_sort_buf[BLOCK / 32][CELL_SORT_SMEM];
    long warp = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5;
    long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    for (long c = warp; c < ncells; c += nwarps) {
        const int s = start[c], e = start[c + 1];
        warp_cell_order(reinterpret_cast<const int*>(in) + s, out + s, (unsigned int)(e - s),
                        cell_sort_buf[threadIdx.x >> 5]);
    }
}

template <class T>
static int run(const void* pos_xyz, long n, const double* box_lo, const double* spacing, const int* gs, int pad,
               int* cell_start, int* sorted_ids, unsigned int* status, cudaStream_t st) {
    unsigned int* S = nullptr;
    PD_TRY(scratch_address(&S));
    long ncells = (long)gs[0] * gs[1] * gs[2];
    Grid<T> G;
    for (int d = 0; d < 3; ++d) {
        G.lo[d] = (T)box_lo[d];
        G.sp[d] = (T)spacing[d];
        G.gs[d] = gs[d];
    }
    G.pad = pad;
    unsigned int* cnt = S;
    unsigned int* cell_of = S + OFF_CELL_OF;
    unsigned int* slot = S + OFF_SLOT;
    unsigned int* tmp = S + OFF_TMP;
    unsigned int* parts = S + OFF_PARTS;
    long m = ncells + 1;
    long nb = (m + TILE - 1) / TILE;
    pd::launch(k_zero, grid_for(m, BLOCK), BLOCK, 0, st, cnt, m);
    if (status) pd::launch(k_zero, 1, 32, 0, st, status, 1L);
    if (n > 0)
        pd::launch(k_hash_xyz<T>, grid_for(n, BLOCK), BLOCK, 0, st, static_cast<const T*>(pos_xyz), n, G, cnt,
                   cell_of, slot, status);
    pd::launch(k_block_tot, (unsigned)nb, BLOCK, 0, st, (const unsigned int*)cnt, m, parts);
    pd::launch(k_tot_scan, 1, 32, 0, st, parts, nb);
    pd::launch(k_apply, (unsigned)nb, BLOCK, 0, st, (const unsigned int*)cnt, m, (const unsigned int*)parts,
               cell_start);
    if (n > 0) {
        pd::launch(k_scatter, grid_for(n, BLOCK), BLOCK, 0, st, n, (const unsigned int*)cell_of,
                   (const unsigned int*)slot, (const int*)cell_start, tmp);
        pd::launch(k_stabilise, grid_for(ncells * 32, BLOCK), BLOCK, 0, st, ncells, (const int*)cell_start,
                   (const unsigned int*)tmp, sorted_ids);
    }
    PD_LAUNCH_CHECK();
    return PD_OK;
}

}  // namespace noalloc
}  // namespace pd

using namespace pd;

extern "C" {

int pd_celllist_build_static(int dtype, const void* pos_xyz, long n, const double* box_lo, const double* spacing,
                             const int* gs, int pad, int* cell_start, int* sorted_ids, unsigned int* status,
                             void* stream) {
    if ((dtype != PD_F32 && dtype != PD_F64) || n < 0 || !box_lo || !spacing || !gs || !cell_start ||
        (n > 0 && (!pos_xyz || !sorted_ids)) || pad < 0) {
        set_error("pd_celllist_build_static: invalid argument");
        return PD_EINVAL;
    }
    for (int d = 0; d < 3; ++d)
        if (gs[d] < 1 || !(spacing[d] > 0)) {
            set_error("pd_celllist_build_static: grid size and spacing must be positive");
            return PD_EINVAL;
        }
    long ncells = (long)gs[0] * gs[1] * gs[2];
    if (n > noalloc::MAX_PART || ncells > noalloc::MAX_CELLS) {
        set_error("pd_celllist_build_static: %ld particles / %ld cells exceed the static scratch limit of "
                  "%ld particles and %ld cells; use pd_celllist_update",
                  n, ncells, noalloc::MAX_PART, noalloc::MAX_CELLS);
        return PD_EINVAL;
    }
    // device memory of the current device only: a host pointer would reach the kernels
    static const char* who = "pd_celllist_build_static";
    PD_TRY(check_device_ptr(cell_start, who, "cell_start"));
    if (n > 0) {
        PD_TRY(check_device_ptr(pos_xyz, who, "pos_xyz"));
        PD_TRY(check_device_ptr(sorted_ids, who, "sorted_ids"));
    }
    if (status) PD_TRY(check_device_ptr(status, who, "status"));
    cudaStream_t st = S(stream);
    if (dtype == PD_F64)
        return noalloc::run<double>(pos_xyz, n, box_lo, spacing, gs, pad, cell_start, sorted_ids, status, st);
    return noalloc::run<float>(pos_xyz, n, box_lo, spacing, gs, pad, cell_start, sorted_ids, status, st);
}

}  // extern "C"
