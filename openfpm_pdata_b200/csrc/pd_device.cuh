// pd_device.cuh -- device-side helpers shared by the kernels of libpdgpu.so.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace pd {

template <class T> struct V4;
template <> struct V4<double> { typedef double4 type; };
template <> struct V4<float> { typedef float4 type; };

// 32-byte double4 record read as two 16-byte vector loads; float4 as one.
__device__ __forceinline__ double4 ld4(const double4* p, long i) {
    const double2* q = reinterpret_cast<const double2*>(p + i);
    double2 a = __ldg(q), b = __ldg(q + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ float4 ld4(const float4* p, long i) { return __ldg(p + i); }
// bring the line holding *p into L2 (no register result)
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }
__device__ __forceinline__ void st4(double4* p, long i, double4 v) {
    double2* q = reinterpret_cast<double2*>(p + i);
    q[0] = make_double2(v.x, v.y);
    q[1] = make_double2(v.z, v.w);
}
__device__ __forceinline__ void st4(float4* p, long i, float4 v) { p[i] = v; }

// openfpm::math::periodic_l (CartDecomposition_gpu.cuh:67-74 applies it per periodic dim)
template <class T> __device__ __forceinline__ T periodic_l(T pos, T p2, T p1) {
    T r = pos;
    if (pos >= p2) {
        r = p1 + (pos - p2);
    } else if (pos < p1) {
        r = p2 - (p1 - pos);
        if (r == p2) r = p1;
    }
    return r;
}

// cell grid of a cell list: ik = clamp(floor((x - lo)/spacing) + pad, 0, gs-1);
// c = i0 + gs0*(i1 + gs1*i2).  Division (not a reciprocal multiply) so that the
// result is the correctly rounded quotient on both the GPU and the host oracle.
template <class T> struct Grid {
    T lo[3];
    T sp[3];
    int gs[3];
    int pad;
    __device__ __forceinline__ int coord(int d, T x, unsigned int& bad) const {
        T q = floor((x - lo[d]) / sp[d]);
        int i;
        if (!(q > T(-1e9)) || !(q < T(1e9))) {  // NaN / inf / absurd
            bad = 1u;
            i = 0;
        } else {
            i = (int)q + pad;
        }
        if (i < 0) { i = 0; bad = 1u; }
        if (i > gs[d] - 1) { i = gs[d] - 1; bad = 1u; }
        return i;
    }
    __device__ __forceinline__ int cell(T x, T y, T z, unsigned int& bad) const {
        int i0 = coord(0, x, bad), i1 = coord(1, y, bad), i2 = coord(2, z, bad);
        return i0 + gs[0] * (i1 + gs[1] * i2);
    }
};

template <class T> __device__ __forceinline__ T dist2(T dx, T dy, T dz) {
    return fma(dz, dz, fma(dy, dy, dx * dx));
}

// warp-aggregated atomic increment of counter[key]: one atomic per distinct key
// in the warp; returns this lane's slot (non-deterministic across warps, which
// the stabilising pass of the counting sort removes).
__device__ __forceinline__ unsigned int warp_agg_inc(unsigned int* counter, unsigned int key, unsigned int active) {
    unsigned int peers = __match_any_sync(active, key);
    int lane = threadIdx.x & 31;
    int leader = __ffs(peers) - 1;
    unsigned int base = 0;
    if (lane == leader) base = atomicAdd(counter + key, (unsigned int)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    unsigned int lower = peers & ((1u << lane) - 1u);
    return base + __popc(lower);
}

// Stable order of one cell after the atomic-slot scatter: one warp writes the n
// distinct indices in[0..n) to out[0..n) in ascending order.  n <= 32: each lane's
// rank from shuffles; n <= cap: bitonic sort in `wbuf` (the warp's `cap` ints of
// shared memory, a power of two); larger: each member's rank counted against
// 32-wide chunks of the cell broadcast through shuffles.
static constexpr unsigned int CELL_SORT_SMEM = 512;
__device__ __forceinline__ void warp_cell_order(const int* __restrict__ in, int* __restrict__ out, unsigned int n,
                                                int* wbuf, unsigned int cap = CELL_SORT_SMEM) {
    const int lane = threadIdx.x & 31;
    if (n == 0) return;
    if (n == 1) {
        if (lane == 0) out[0] = in[0];
        return;
    }
    if (n <= 32) {
        const int v = lane < (int)n ? in[lane] : 0x7fffffff;
        unsigned int rank = 0;
        for (int j = 0; j < (int)n; ++j) rank += (__shfl_sync(0xffffffffu, v, j) < v) ? 1u : 0u;
        if (lane < (int)n) out[rank] = v;
        return;
    }
    if (n <= cap) {
        unsigned int P = 64;
        while (P < n) P <<= 1;
        for (unsigned int i = lane; i < P; i += 32) wbuf[i] = i < n ? in[i] : 0x7fffffff;
        __syncwarp();
        for (unsigned int k = 2; k <= P; k <<= 1)
            for (unsigned int j = k >> 1; j > 0; j >>= 1) {
                for (unsigned int i = lane; i < P; i += 32) {
                    const unsigned int o = i ^ j;
                    if (o > i) {
                        const int a = wbuf[i], b = wbuf[o];
                        if ((a > b) == ((i & k) == 0)) {
                            wbuf[i] = b;
                            wbuf[o] = a;
                        }
                    }
                }
                __syncwarp();
            }
        for (unsigned int i = lane; i < n; i += 32) out[i] = wbuf[i];
        __syncwarp();
        return;
    }
    for (unsigned int a0 = 0; a0 < n; a0 += 32) {
        const int v = a0 + lane < n ? in[a0 + lane] : 0x7fffffff;
        unsigned int rank = 0;
        for (unsigned int j0 = 0; j0 < n; j0 += 32) {
            const int w = j0 + lane < n ? in[j0 + lane] : 0x7fffffff;
            const int m = (int)min(32u, n - j0);
            for (int j = 0; j < m; ++j) rank += (__shfl_sync(0xffffffffu, w, j) < v) ? 1u : 0u;
        }
        if (a0 + lane < n) out[rank] = v;
    }
}

template <class T> __device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
template <class T> __device__ __forceinline__ T warp_max(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// deterministic block sum into out[blockIdx.x] (fixed shuffle tree + fixed warp order)
template <class T, int BLOCK> __device__ __forceinline__ T block_sum(T v) {
    __shared__ T sh[BLOCK / 32];
    v = warp_sum(v);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = v;
    __syncthreads();
    T r = 0;
    if (w == 0) {
        r = (l < BLOCK / 32) ? sh[l] : T(0);
        r = warp_sum(r);
    }
    __syncthreads();
    return r;  // valid in thread 0
}

// block maximum of non-negative values (valid in thread 0)
template <class T, int BLOCK> __device__ __forceinline__ T block_max(T v) {
    __shared__ T sh[BLOCK / 32];
    v = warp_max(v);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = v;
    __syncthreads();
    T r = 0;
    if (w == 0) {
        r = (l < BLOCK / 32) ? sh[l] : T(0);
        r = warp_max(r);
    }
    __syncthreads();
    return r;
}

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* a, double v) {
    atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

// ---------------------------------------------------------------------------
// 1-D bulk copies global -> shared through the TMA engine (cp.async.bulk, no
// tensor map, no multicast) completing on an mbarrier.  Addresses and sizes must
// be multiples of 16 bytes (positions are 16- or 32-byte records).
__device__ __forceinline__ unsigned int smem_u32(const void* p) {
    return static_cast<unsigned int>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned int bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned int bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned int phase) {
    unsigned int ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0u;
}
// bounded wait on phase `phase`; false after `limit` polls
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned int phase, unsigned int limit) {
    for (unsigned int it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}

}  // namespace pd
