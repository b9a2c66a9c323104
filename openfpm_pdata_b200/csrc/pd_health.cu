// Failure detection of the bounded device waits, exercised without a fault.
//
// Every tile kernel stages its neighbourhood with cp.async.bulk copies that
// complete an mbarrier, and waits on it with a bounded number of polls
// (mbar_wait_bounded); a wait that gives up sets ERR_TIMEOUT, waits once more
// for copies in flight and returns, and the host turns the bit into an error
// status.  pd_selftest_wait runs that staging pattern on one CTA: with the copy
// issued the phase completes; without it nothing ever completes the phase, so
// the wait gives up after `limit` polls and the status comes back as
// PD_ETIMEOUT with the context still usable.
#include "pd_device.cuh"
#include "pd_internal.cuh"

namespace pd {

__global__ void k_wait_selftest(const float4* __restrict__ src, float4* __restrict__ dst, int issue,
                                unsigned int limit, unsigned int* __restrict__ status) {
    __shared__ __align__(16) float4 buf[1];
    __shared__ unsigned long long bar;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_arrive_expect_tx(&bar, (unsigned int)sizeof(float4));
        if (issue) bulk_g2s(buf, src, (unsigned int)sizeof(float4), &bar);
    }
    const bool ok = mbar_wait_bounded(&bar, 0, limit);
    __syncthreads();
    if (threadIdx.x == 0) {
        *status = ok ? 0u : ERR_TIMEOUT;
        if (ok) dst[0] = buf[0];
    }
}

// Vector FMA throughput: eight independent chains per thread (enough in flight to
// hide the pipeline latency), a*b+c with b, c fixed; each FMA counts two flops.
template <class T>
__global__ void __launch_bounds__(256) k_fma_rate(T* __restrict__ out, int iters, T b, T c) {
    T a0 = (T)threadIdx.x, a1 = a0 + T(1), a2 = a0 + T(2), a3 = a0 + T(3), a4 = a0 + T(4), a5 = a0 + T(5),
      a6 = a0 + T(6), a7 = a0 + T(7);
    for (int k = 0; k < iters; ++k) {
        a0 = fma(a0, b, c);
        a1 = fma(a1, b, c);
        a2 = fma(a2, b, c);
        a3 = fma(a3, b, c);
        a4 = fma(a4, b, c);
        a5 = fma(a5, b, c);
        a6 = fma(a6, b, c);
        a7 = fma(a7, b, c);
    }
    out[blockIdx.x * (long)blockDim.x + threadIdx.x] = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
}

template <class T> static int fma_rate(double* tflops) {
    int dev = 0, sms = 148;
    PD_CUDA(cudaGetDevice(&dev));
    PD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = sms * 8, threads = 256, iters = 1 << 14;
    Buf out;
    PD_TRY(out.ensure(sizeof(T) * (size_t)blocks * threads));
    cudaEvent_t e0, e1;
    PD_CUDA(cudaEventCreate(&e0));
    PD_CUDA(cudaEventCreate(&e1));
    const T b = (T)0.999999, c = (T)1e-7;
    pd::launch(k_fma_rate<T>, blocks, threads, 0, (cudaStream_t)0, out.as<T>(), iters, b, c);  // warm-up
    PD_CUDA(cudaEventRecord(e0, 0));
    pd::launch(k_fma_rate<T>, blocks, threads, 0, (cudaStream_t)0, out.as<T>(), iters, b, c);
    PD_CUDA(cudaEventRecord(e1, 0));
    PD_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    PD_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    out.release();
    *tflops = 2.0 * 8.0 * (double)iters * blocks * threads / (ms * 1e-3) / 1e12;
    return PD_OK;
}

}  // namespace pd

using namespace pd;

extern "C" {

int pd_selftest_wait(long limit, int issue_copy, const float* in4, float* out4) {
    if (limit < 1 || limit > (1L << 30) || !in4 || !out4) return PD_EINVAL;
    void* d = nullptr;
    PD_CUDA(cudaMalloc(&d, 2 * sizeof(float4) + sizeof(unsigned int)));
    float4* src = (float4*)d;
    float4* dst = src + 1;
    unsigned int* status = (unsigned int*)(src + 2);
    unsigned int st_h = ~0u;
    cudaError_t e = cudaMemcpy(src, in4, sizeof(float4), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(dst, 0, sizeof(float4) + sizeof(unsigned int));
    if (e == cudaSuccess) {
        pd::launch(k_wait_selftest, 1, 32, 0, (cudaStream_t)0, (const float4*)src, dst, issue_copy,
                   (unsigned int)limit, status);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(&st_h, status, sizeof(unsigned int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(out4, dst, sizeof(float4), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) {
        set_error("pd_selftest_wait: %s", cudaGetErrorString(e));
        return PD_ECUDA;
    }
    if (st_h & ERR_TIMEOUT) {
        set_error("pd_selftest_wait: the bounded wait gave up after %ld polls", limit);
        return PD_ETIMEOUT;
    }
    return PD_OK;
}

int pd_measure_fma_rate(int dtype, double* tflops) {
    if (!tflops || (dtype != PD_F32 && dtype != PD_F64)) return PD_EINVAL;
    return dtype == PD_F64 ? fma_rate<double>(tflops) : fma_rate<float>(tflops);
}

}  // extern "C"
