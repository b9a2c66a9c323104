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

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* a, double v) {
    atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

}  // namespace pd
