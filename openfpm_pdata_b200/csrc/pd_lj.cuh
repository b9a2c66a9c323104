// pd_lj.cuh -- Lennard-Jones 12-6 pair term shared by the LJ kernels.
//   F_i += 24 eps (2 (s/r)^12 - (s/r)^6) / r^2 * (x_i - x_j)      (r < r_cut)
//   U   += 4 eps ((s/r)^12 - (s/r)^6),  W += F.r
#pragma once
#include "pd_device.cuh"

namespace pd {

template <class T> struct LJP {
    T eps24, eps4, sig2, rc2;
    // precision form only: squared distances in [rc2lo, rc2hi) lie within the FP32
    // rounding of r2 from the cutoff and are decided again in FP64 against rc2d;
    // pairs below rclose2 are evaluated in FP64 with the *d parameters
    T rc2lo, rc2hi, rclose2;
    double rc2d, eps24d, eps4d, sig2d;
};

// Cutoff decision of the precision form.  dx, dy, dz are exact (the offsets lie on
// the quantum grid, see pd_mixed.cu), so r2 = fma(dz,dz, fma(dy,dy, dx*dx)) in FP32
// carries only its own three roundings; outside the band it decides like FP64.  In
// the band the same formula in FP64 (the FP32 products are exact there) decides.
__device__ __forceinline__ bool in_cut_exact(float r2, float dx, float dy, float dz, const LJP<float>& P) {
    bool in = r2 < P.rc2lo;
    if (r2 >= P.rc2lo && r2 < P.rc2hi) {
        const double x = dx, y = dy, z = dz;
        in = fma(z, z, fma(y, y, x * x)) < P.rc2d;
    }
    return in;
}

// Reciprocal from the hardware approximation y0 = rcp.approx.ftz.f64(x), whose
// relative error |e| = |1 - x y0| is below 2^-20: 1/x = y0 / (1 - e) =
// y0 (1 + e + e^2 + e^3 + ...), and the series to e^2 leaves e^3 < 2^-60, below
// the double rounding, so one correction y0 + y0 (e + e^2) -- three fused
// multiply-adds, cubic convergence where a Newton-Raphson step (y' = y + y e) is
// quadratic and needs two -- gives the reciprocal within 2 ulp
// (tests/test_gpu_recip.py; Markstein, "Computation of elementary functions on the
// IBM RISC System/6000", IBM J. Res. Dev. 34, 1990).  Valid for normal positive
// arguments, which is what squared pair distances are.
__device__ __forceinline__ double recip(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-x, y, 1.0);
    return fma(fma(e, e, e), y, y);
}
// a / x by the same series with a folded into the correction: a y0 (1 + e + e^2).
// NaN for x = 0 (the caller selects the result away).
__device__ __forceinline__ double div_by(double a, double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-x, y, 1.0);
    const double ay = a * y;
    return fma(fma(e, e, e), ay, ay);
}
// FP32: hardware approximation (rcp.approx.ftz.f32, ~1 ulp) plus one refinement step
__device__ __forceinline__ float recip(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    float e = fmaf(-x, y, 1.0f);
    return fmaf(y, e, y);
}

// FP32 a / x: the approximation is within about 1 ulp, so one correction a y0 (1 + e)
// leaves e^2 below the float rounding.  NaN for x = 0 (the caller selects it away).
__device__ __forceinline__ float div_by(float a, float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    const float e = fmaf(-x, y, 1.0f);
    const float ay = a * y;
    return fmaf(e, ay, ay);
}

template <class T>
__device__ __forceinline__ void lj_acc(const LJP<T>& P, T r2, T dx, T dy, T dz, T& fx, T& fy, T& fz, T& e, T& w) {
    T ir2 = recip(r2);
    T s2 = P.sig2 * ir2;
    T s6 = s2 * s2 * s2;
    T ff = P.eps24 * ir2 * s6 * (T(2) * s6 - T(1));
    fx += ff * dx;
    fy += ff * dy;
    fz += ff * dz;
    e += P.eps4 * s6 * (s6 - T(1));
    w += ff * r2;
}

}  // namespace pd
