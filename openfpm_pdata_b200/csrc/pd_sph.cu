// pd_sph.cu -- weakly compressible SPH on the tiled neighbour structure.
//
// The reference has no SPH physics (its pair functors are test sums,
// vector_dist_gpu_unit_tests.cu:46-119); the scheme is the standard WCSPH one:
//   kernel      cubic spline, support 2h (Monaghan & Lattanzio 1985)
//   EOS         p = B ((rho/rho0)^7 - 1), B = c0^2 rho0 / 7 (Tait; Monaghan 1994)
//   viscosity   Pi_ab = -alpha c0 mu_ab / rho_bar, mu_ab = h v_ab.r_ab / (r^2 + 0.01 h^2)
//               for v_ab.r_ab < 0 (Monaghan 1992)
//   momentum    dv_a/dt = -sum_b m (p_a/rho_a^2 + p_b/rho_b^2 + Pi_ab) grad W_ab + g
//   continuity  drho_a/dt = sum_b m v_ab . grad W_ab
// Wall particles (type 1) are fixed; their density evolves (dynamic boundary).
// Time stepping: v += dt/2 a, rho += dt/2 drho, x += dt v (fluid), rates,
// v += dt/2 a, rho += dt/2 drho.
//
// Per step the pair kernel stages, for every tile, two records per particle
// with the same 1-D TMA bulk copies: (x, y, z, p) from the position array (the
// pressure lives in the position record's fourth word) and (vx, vy, vz, rho)
// from a packed auxiliary array written by the integrator.
#include <algorithm>

#include "pd_device.cuh"
#include "pd_internal.cuh"
#include "pd_lj.cuh"
#include "pd_sph.cuh"
#include "pd_tile.cuh"

namespace pd {

template <class T> struct SphK {
    T h, m, c0, rho0, B, alpha, gz, eta2, dw3, r2c, inv_h, visc;  // visc = -alpha c0 h
};

template <class T> __device__ __forceinline__ T eos(const SphK<T>& P, T rho) {
    T x = rho / P.rho0;
    T x2 = x * x;
    T x7 = x2 * x2 * x2 * x;
    return P.B * (x7 - T(1));
}

__device__ __forceinline__ double rsqrt_t(double x) { return rsqrt(x); }
__device__ __forceinline__ float rsqrt_t(float x) { return rsqrtf(x); }

// (dW/dr)/r of the cubic spline from r and 1/r, q = r/h
template <class T> __device__ __forceinline__ T dwdr_over_r(const SphK<T>& P, T r, T inv_r) {
    T q = r * P.inv_h;
    T d;
    if (q < T(1)) d = (T(-3) * q + T(2.25) * q * q);
    else if (q < T(2)) d = T(-0.75) * (T(2) - q) * (T(2) - q);
    else d = T(0);
    return P.dw3 * d * inv_r;
}

// the staged pressure term p / rho^2 (the same operations as p_b / (rho_b rho_b) per pair)
template <class T> __device__ __forceinline__ T p_over_rho2(const SphK<T>& P, T rho) { return eos(P, rho) / (rho * rho); }

// p / rho^2 into the position record, (v, rho) into the auxiliary record
template <class T>
__global__ void k_sph_pack(typename V4<T>::type* __restrict__ pos, typename V4<T>::type* __restrict__ aux,
                           const T* __restrict__ v, const T* __restrict__ rho, long cap, long n, SphK<T> P) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        typename V4<T>::type x = ld4(pos, i);
        T r = rho[i];
        x.w = p_over_rho2(P, r);
        st4(pos, i, x);
        typename V4<T>::type a;
        a.x = v[i];
        a.y = v[cap + i];
        a.z = v[2 * cap + i];
        a.w = r;
        st4(aux, i, a);
    }
}

// first half kick + drift; refreshes pressure and the auxiliary record
template <class T>
__global__ void __launch_bounds__(256) k_sph_kick_drift(typename V4<T>::type* __restrict__ pos,
                                                        const typename V4<T>::type* __restrict__ xb,
                                                        typename V4<T>::type* __restrict__ aux, T* __restrict__ v,
                                                        const T* __restrict__ a, T* __restrict__ rho,
                                                        const T* __restrict__ drho, const int* __restrict__ type,
                                                        long cap, long n, T half, T dt, SphK<T> P,
                                                        unsigned long long* __restrict__ maxd2) {
    double mx = 0;
    for (long i = blockIdx.x * 256L + threadIdx.x; i < n; i += (long)gridDim.x * 256) {
        typename V4<T>::type x = ld4(pos, i);
        T vx = v[i], vy = v[cap + i], vz = v[2 * cap + i];
        if (type[i] == 0) {
            vx += half * a[i];
            vy += half * a[cap + i];
            vz += half * a[2 * cap + i];
            x.x += dt * vx;
            x.y += dt * vy;
            x.z += dt * vz;
            v[i] = vx;
            v[cap + i] = vy;
            v[2 * cap + i] = vz;
            typename V4<T>::type b = ld4(xb, i);
            mx = fmax(mx, (double)dist2(x.x - b.x, x.y - b.y, x.z - b.z));
        }
        T r = rho[i] + half * drho[i];
        rho[i] = r;
        x.w = p_over_rho2(P, r);
        st4(pos, i, x);
        typename V4<T>::type au;
        au.x = vx;
        au.y = vy;
        au.z = vz;
        au.w = r;
        st4(aux, i, au);
    }
    mx = warp_max(mx);
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(maxd2, mx);
}

// second half kick; kinetic energy of the fluid and sum of densities (fixed-order partials)
template <class T>
__global__ void __launch_bounds__(256) k_sph_kick(T* __restrict__ v, const T* __restrict__ a, T* __restrict__ rho,
                                                  const T* __restrict__ drho, const int* __restrict__ type, long cap,
                                                  long n, T half, double m, double* __restrict__ kpart,
                                                  double* __restrict__ rpart) {
    double ke = 0, rs = 0;
    for (long i = blockIdx.x * 256L + threadIdx.x; i < n; i += (long)gridDim.x * 256) {
        if (type[i] == 0) {
            T vx = v[i] + half * a[i];
            T vy = v[cap + i] + half * a[cap + i];
            T vz = v[2 * cap + i] + half * a[2 * cap + i];
            v[i] = vx;
            v[cap + i] = vy;
            v[2 * cap + i] = vz;
            ke += 0.5 * m * ((double)vx * vx + (double)vy * vy + (double)vz * vz);
        }
        T r = rho[i] + half * drho[i];
        rho[i] = r;
        rs += (double)r;
    }
    ke = block_sum<double, 256>(ke);
    rs = block_sum<double, 256>(rs);
    if (threadIdx.x == 0) {
        kpart[blockIdx.x] = ke;
        rpart[2 * blockIdx.x] = rs;
        rpart[2 * blockIdx.x + 1] = 0.0;
    }
}

// The end of one step and the start of the next in one pass: k_sph_kick of the step
// (kinetic energy and density partials) and k_sph_kick_drift of the next, the same
// operations in the same order, each array read and written once.
template <class T>
__global__ void __launch_bounds__(256) k_sph_kick_kick_drift(typename V4<T>::type* __restrict__ pos,
                                                             const typename V4<T>::type* __restrict__ xb,
                                                             typename V4<T>::type* __restrict__ aux,
                                                             T* __restrict__ v, const T* __restrict__ a,
                                                             T* __restrict__ rho, const T* __restrict__ drho,
                                                             const int* __restrict__ type, long cap, long n, T half,
                                                             T dt, SphK<T> P, double m,
                                                             unsigned long long* __restrict__ maxd2,
                                                             double* __restrict__ kpart, double* __restrict__ rpart) {
    double mx = 0, ke = 0, rs = 0;
    for (long i = blockIdx.x * 256L + threadIdx.x; i < n; i += (long)gridDim.x * 256) {
        typename V4<T>::type x = ld4(pos, i);
        T vx = v[i], vy = v[cap + i], vz = v[2 * cap + i];
        if (type[i] == 0) {
            const T ax = a[i], ay = a[cap + i], az = a[2 * cap + i];
            vx = vx + half * ax;  // the step's closing half kick
            vy = vy + half * ay;
            vz = vz + half * az;
            ke += 0.5 * m * ((double)vx * vx + (double)vy * vy + (double)vz * vz);
            vx = vx + half * ax;  // the next step's opening half kick and drift
            vy = vy + half * ay;
            vz = vz + half * az;
            x.x += dt * vx;
            x.y += dt * vy;
            x.z += dt * vz;
            v[i] = vx;
            v[cap + i] = vy;
            v[2 * cap + i] = vz;
            typename V4<T>::type b = ld4(xb, i);
            mx = fmax(mx, (double)dist2(x.x - b.x, x.y - b.y, x.z - b.z));
        }
        const T dr = drho[i];
        T r = rho[i] + half * dr;
        rs += (double)r;
        r = r + half * dr;
        rho[i] = r;
        x.w = p_over_rho2(P, r);
        st4(pos, i, x);
        typename V4<T>::type au;
        au.x = vx;
        au.y = vy;
        au.z = vz;
        au.w = r;
        st4(aux, i, au);
    }
    mx = warp_max(mx);
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(maxd2, mx);
    ke = block_sum<double, 256>(ke);
    rs = block_sum<double, 256>(rs);
    if (threadIdx.x == 0) {
        kpart[blockIdx.x] = ke;
        rpart[2 * blockIdx.x] = rs;
        rpart[2 * blockIdx.x + 1] = 0.0;
    }
}

struct TileShS {
    unsigned int cR[9][TXMAX + 3];
    unsigned int oR[9];
    unsigned int total;
    int ncol;
    unsigned long long bar;
};

// rates of every particle of a tile; no periodic images in this configuration
template <class T, int P>
__global__ void __launch_bounds__(FBLOCK_T) k_vtile_sph(const typename V4<T>::type* __restrict__ pos,
                                                        const typename V4<T>::type* __restrict__ aux, TileGeom tg,
                                                        const unsigned int* __restrict__ csR, unsigned int cap,
                                                        const unsigned int* __restrict__ nbr,
                                                        const int* __restrict__ nn, long stride, int mwords,
                                                        const int* __restrict__ type, SphK<T> K, T* __restrict__ acc,
                                                        T* __restrict__ drho, long cap_p,
                                                        unsigned int* __restrict__ err) {
    typedef typename V4<T>::type T4;
    extern __shared__ __align__(128) unsigned char tile_raw[];
    T4* sp = reinterpret_cast<T4*>(tile_raw);
    T4* sa = sp + cap;
    __shared__ TileShS S;
    {
        long t = blockIdx.x;
        int tx = (int)(t % tg.ntx);
        long rest = t / tg.ntx;
        int y = (int)(rest % tg.ny) + tg.pad;
        int z = (int)(rest / tg.ny) + tg.pad;
        int x0 = tg.pad + tx * tg.TX;
        int x1 = min(x0 + tg.TX, tg.gs0 - tg.pad);
        int ncol = x1 - x0 + 3;
        for (int e = threadIdx.x; e < 9 * ncol; e += blockDim.x) {
            int r = e / ncol, j = e % ncol;
            int dz = r / 3 - 1, dy = r % 3 - 1;
            long c = (long)(x0 - 1 + j) + (long)tg.gs0 * ((y + dy) + (long)tg.gs1 * (z + dz));
            S.cR[r][j] = csR[c];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned int o = 0;
            for (int r = 0; r < 9; ++r) {
                S.oR[r] = o;
                o += S.cR[r][ncol - 1] - S.cR[r][0];
            }
            S.total = o;
            S.ncol = ncol;
        }
        __syncthreads();
    }
    const int ncol = S.ncol;
    const unsigned int ib = S.cR[4][1], ie = S.cR[4][ncol - 2];
    if (ib == ie) return;
    if (S.total > cap) {
        if (threadIdx.x == 0) atomicOr(err, ERR_TILE_CAP);
        return;
    }
    if (threadIdx.x == 0) mbar_init(&S.bar, 1);
    __syncthreads();
    if (threadIdx.x < 32) {
        // one lane a copy: lane 2r row r's position records, 2r + 1 its velocity records
        const unsigned int lane = threadIdx.x;
        if (lane == 0) mbar_arrive_expect_tx(&S.bar, 2u * S.total * (unsigned int)sizeof(T4));
        __syncwarp();
        if (lane < 18u) {
            const int r = (int)(lane >> 1), nc = ncol - 1;
            const unsigned int lr = S.cR[r][nc] - S.cR[r][0];
            if (lr) {
                if (lane & 1u) bulk_g2s(sa + S.oR[r], aux + S.cR[r][0], lr * (unsigned int)sizeof(T4), &S.bar);
                else bulk_g2s(sp + S.oR[r], pos + S.cR[r][0], lr * (unsigned int)sizeof(T4), &S.bar);
            }
        }
    }
    bool waited = mbar_wait_bounded(&S.bar, 0, 1u << 24);
    if (!waited) {
        atomicOr(err, ERR_TIMEOUT);
        mbar_wait_bounded(&S.bar, 0, 1u << 24);
    }
    if (!__syncthreads_and(waited ? 1 : 0)) return;

    const unsigned int base = S.oR[4] - S.cR[4][0];
    // rounds of the whole CTA over the tile's particles: P lanes per row while a
    // round is full, more lanes per row (up to a warp) in the last, partial round;
    // every thread takes part in every round (the shuffles need whole warps)
    unsigned int first = ib;
    while (first < ie) {
        const unsigned int left = ie - first;
        unsigned int q = P;
        while (q < 32u && left * (q << 1) <= (unsigned int)FBLOCK_T) q <<= 1;
        const unsigned int cnt = min(left, (unsigned int)FBLOCK_T / q);
        const int sub = (int)(threadIdx.x % q);
        const int Q = (int)q;
        const bool active = threadIdx.x / q < cnt;
        const unsigned int i = first + (active ? threadIdx.x / q : 0u);
        const unsigned int li = base + i;
        const T4 xi = sp[li];
        const T4 ai = sa[li];
        const T pa_r = xi.w;
        const unsigned int* row = nbr + i;
        // row words read four iterations ahead (register shift ring); the first four
        // together with the row length (within the buffer's mwords words per particle)
        unsigned int q0 = sub < mwords ? __ldg(row + (long)sub * stride) : 0u;
        unsigned int q1 = sub + Q < mwords ? __ldg(row + (long)(sub + Q) * stride) : 0u;
        unsigned int q2 = sub + 2 * Q < mwords ? __ldg(row + (long)(sub + 2 * Q) * stride) : 0u;
        unsigned int q3 = sub + 3 * Q < mwords ? __ldg(row + (long)(sub + 3 * Q) * stride) : 0u;
        const int words = active ? (nn[i] + 1) >> 1 : 0;
        T ax = 0, ay = 0, az = 0, dr = 0;
        for (int k = sub; k < words; k += Q) {
            const unsigned int pair = q0;
            q0 = q1;
            q1 = q2;
            q2 = q3;
            q3 = k + 4 * Q < words ? __ldg(row + (long)(k + 4 * Q) * stride) : 0u;
#pragma unroll
            for (int hh = 0; hh < 2; ++hh) {
                const unsigned int l = hh ? (pair >> 16) : (pair & 0xffffu);
                const T4 xq = sp[l];
                const T dx = xi.x - xq.x, dy = xi.y - xq.y, dz = xi.z - xq.z;
                const T r2 = dist2(dx, dy, dz);
                const bool in = r2 < K.r2c && l != li;
                if (sizeof(T) == 4) {
                    // FP32: every pair through the same instructions (faster here); pairs
                    // outside the support and the particle itself get a zero gradient
                    const T4 aq = sa[l];
                    const T r2s = in ? r2 : T(1);
                    const T inv_r = rsqrt_t(r2s);
                    const T dwr = in ? dwdr_over_r(K, r2s * inv_r, inv_r) : T(0);
                    const T vx = ai.x - aq.x, vy = ai.y - aq.y, vz = ai.z - aq.z;
                    const T vr = vx * dx + vy * dy + vz * dz;
                    // -alpha c0 mu / rho_bar, mu = h vr / (r^2 + eta^2), approaching pairs only
                    const T pi_ab =
                        vr < T(0) ? K.visc * vr * recip((r2 + K.eta2) * (T(0.5) * (ai.w + aq.w))) : T(0);
                    const T coef = -K.m * (pa_r + xq.w + pi_ab) * dwr;
                    ax += coef * dx;
                    ay += coef * dy;
                    az += coef * dz;
                    dr += K.m * vr * dwr;
                } else if (in) {
                    // FP64: the branch (the select form measured slower)
                    const T4 aq = sa[l];
                    const T inv_r = rsqrt_t(r2);
                    const T dwr = dwdr_over_r(K, r2 * inv_r, inv_r);
                    const T vx = ai.x - aq.x, vy = ai.y - aq.y, vz = ai.z - aq.z;
                    const T vr = vx * dx + vy * dy + vz * dz;
                    T pi_ab = 0;
                    if (vr < T(0)) pi_ab = K.visc * vr * recip((r2 + K.eta2) * (T(0.5) * (ai.w + aq.w)));
                    const T coef = -K.m * (pa_r + xq.w + pi_ab) * dwr;
                    ax += coef * dx;
                    ay += coef * dy;
                    az += coef * dz;
                    dr += K.m * vr * dwr;
                }
            }
        }
        for (unsigned int o = 1; o < q; o <<= 1) {
            ax += __shfl_xor_sync(0xffffffffu, ax, o);
            ay += __shfl_xor_sync(0xffffffffu, ay, o);
            az += __shfl_xor_sync(0xffffffffu, az, o);
            dr += __shfl_xor_sync(0xffffffffu, dr, o);
        }
        if (active && sub == 0) {
            const bool fluid = type[i] == 0;
            acc[i] = fluid ? ax : T(0);
            acc[cap_p + i] = fluid ? ay : T(0);
            acc[2 * cap_p + i] = fluid ? az + K.gz : T(0);
            drho[i] = dr;
        }
        first += cnt;
    }
}

// ---------------------------------------------------------------------------
template <class T> static SphK<T> sphk(const pd_sph_params_t& sp) {
    SphK<T> K;
    K.h = (T)sp.h;
    K.m = (T)sp.mass;
    K.c0 = (T)sp.c0;
    K.rho0 = (T)sp.rho0;
    K.B = K.c0 * K.c0 * K.rho0 / T(7);
    K.alpha = (T)sp.alpha;
    K.gz = (T)sp.gz;
    K.eta2 = T(0.01) * K.h * K.h;
    const T pi = (T)3.14159265358979323846;
    T w3 = T(1) / (pi * K.h * K.h * K.h);
    K.dw3 = w3 / K.h;
    T two_h = T(2) * K.h;
    K.r2c = two_h * two_h;
    K.inv_h = T(1) / K.h;
    K.visc = -K.alpha * K.c0 * K.h;
    return K;
}

int sph_pack(pd_vd h, const pd_sph_params_t& sp, int vel_prop, Buf& aux, cudaStream_t st) {
    long n = h->n_real;
    PD_TRY(aux.ensure((size_t)h->pos_bytes * (h->cap > 0 ? h->cap : 1)));
    if (n == 0) return PD_OK;
    const Prop& V = h->props[vel_prop];
    const Prop& R = h->props[sp.rho_prop];
    if (h->dtype == PD_F64)
        pd::launch(k_sph_pack<double>, grid_for(n, 256), 256, 0, st, (double4*)h->pos, aux.as<double4>(),
                   (const double*)V.d, (const double*)R.d, h->cap, n, sphk<double>(sp));
    else
        pd::launch(k_sph_pack<float>, grid_for(n, 256), 256, 0, st, (float4*)h->pos, aux.as<float4>(),
                   (const float*)V.d, (const float*)R.d, h->cap, n, sphk<float>(sp));
    PD_LAUNCH_CHECK();
    return PD_OK;
}

int sph_kick_drift(pd_vd h, const pd_sph_params_t& sp, int vel_prop, int acc_prop, const Buf& xb, Buf& aux,
                   int nblk, double dt, cudaStream_t st) {
    long n = h->n_real;
    const Prop& V = h->props[vel_prop];
    const Prop& A = h->props[acc_prop];
    const Prop& R = h->props[sp.rho_prop];
    const Prop& D = h->props[sp.drho_prop];
    const Prop& Ty = h->props[sp.type_prop];
    if (h->dtype == PD_F64)
        pd::launch(k_sph_kick_drift<double>, nblk, 256, 0, st, (double4*)h->pos, (const double4*)xb.as<double4>(),
                   aux.as<double4>(), (double*)V.d, (const double*)A.d, (double*)R.d, (const double*)D.d,
                   (const int*)Ty.d, h->cap, n, 0.5 * dt, dt, sphk<double>(sp), &h->ctrl->maxdisp2);
    else
        pd::launch(k_sph_kick_drift<float>, nblk, 256, 0, st, (float4*)h->pos, (const float4*)xb.as<float4>(),
                   aux.as<float4>(), (float*)V.d, (const float*)A.d, (float*)R.d, (const float*)D.d,
                   (const int*)Ty.d, h->cap, n, (float)(0.5 * dt), (float)dt, sphk<float>(sp), &h->ctrl->maxdisp2);
    PD_LAUNCH_CHECK();
    return PD_OK;
}

int sph_kick(pd_vd h, const pd_sph_params_t& sp, int vel_prop, int acc_prop, int nblk, double dt, double* kpart,
             double* rpart, cudaStream_t st) {
    long n = h->n_real;
    const Prop& V = h->props[vel_prop];
    const Prop& A = h->props[acc_prop];
    const Prop& R = h->props[sp.rho_prop];
    const Prop& D = h->props[sp.drho_prop];
    const Prop& Ty = h->props[sp.type_prop];
    if (h->dtype == PD_F64)
        pd::launch(k_sph_kick<double>, nblk, 256, 0, st, (double*)V.d, (const double*)A.d, (double*)R.d,
                   (const double*)D.d, (const int*)Ty.d, h->cap, n, 0.5 * dt, sp.mass, kpart, rpart);
    else
        pd::launch(k_sph_kick<float>, nblk, 256, 0, st, (float*)V.d, (const float*)A.d, (float*)R.d,
                   (const float*)D.d, (const int*)Ty.d, h->cap, n, (float)(0.5 * dt), sp.mass, kpart, rpart);
    PD_LAUNCH_CHECK();
    return PD_OK;
}

int sph_kick_kick_drift(pd_vd h, const pd_sph_params_t& sp, int vel_prop, int acc_prop, const Buf& xb, Buf& aux,
                        int nblk, double dt, double* kpart, double* rpart, cudaStream_t st) {
    long n = h->n_real;
    const Prop& V = h->props[vel_prop];
    const Prop& A = h->props[acc_prop];
    const Prop& R = h->props[sp.rho_prop];
    const Prop& D = h->props[sp.drho_prop];
    const Prop& Ty = h->props[sp.type_prop];
    if (h->dtype == PD_F64)
        pd::launch(k_sph_kick_kick_drift<double>, nblk, 256, 0, st, (double4*)h->pos,
                   (const double4*)xb.as<double4>(), aux.as<double4>(), (double*)V.d, (const double*)A.d,
                   (double*)R.d, (const double*)D.d, (const int*)Ty.d, h->cap, n, 0.5 * dt, dt, sphk<double>(sp),
                   sp.mass, &h->ctrl->maxdisp2, kpart, rpart);
    else
        pd::launch(k_sph_kick_kick_drift<float>, nblk, 256, 0, st, (float4*)h->pos, (const float4*)xb.as<float4>(),
                   aux.as<float4>(), (float*)V.d, (const float*)A.d, (float*)R.d, (const float*)D.d,
                   (const int*)Ty.d, h->cap, n, (float)(0.5 * dt), (float)dt, sphk<float>(sp), sp.mass,
                   &h->ctrl->maxdisp2, kpart, rpart);
    PD_LAUNCH_CHECK();
    return PD_OK;
}

template <class T, int P>
static int launch_sph(pd_vd h, const TileGeom& tg, long ntiles, const unsigned int* csR, unsigned int cap,
                      const Buf& nbr, const Buf& nn, long stride, const Buf& aux, const pd_sph_params_t& sp,
                      int acc_prop, cudaStream_t st) {
    typedef typename V4<T>::type T4;
    int smem = (int)(2 * cap * sizeof(T4));
    if (smem < 32) smem = 32;
    const int mwords = (int)std::min<long>((long)(nbr.bytes / (4 * (size_t)stride)), 1L << 30);
    PD_CUDA(cudaFuncSetAttribute(k_vtile_sph<T, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    const Prop& A = h->props[acc_prop];
    const Prop& D = h->props[sp.drho_prop];
    const Prop& Ty = h->props[sp.type_prop];
    pd::launch(k_vtile_sph<T, P>, (unsigned)ntiles, FBLOCK_T, (size_t)smem, st, (const T4*)h->pos,
               (const T4*)aux.as<T4>(), tg, csR, cap, (const unsigned int*)nbr.as<unsigned int>(),
               (const int*)nn.as<int>(), stride, mwords, (const int*)Ty.d, sphk<T>(sp), (T*)A.d, (T*)D.d, h->cap,
               &h->ctrl->err);
    PD_LAUNCH_CHECK();
    return PD_OK;
}

int sph_rates(pd_vd h, const TileGeom& tg, long ntiles, const unsigned int* csR, unsigned int cap, const Buf& nbr,
              const Buf& nn, long stride, const Buf& aux, const pd_sph_params_t& sp, int acc_prop, int P,
              cudaStream_t st) {
    if (h->dtype == PD_F64) {
        if (P == 4) return launch_sph<double, 4>(h, tg, ntiles, csR, cap, nbr, nn, stride, aux, sp, acc_prop, st);
        if (P == 1) return launch_sph<double, 1>(h, tg, ntiles, csR, cap, nbr, nn, stride, aux, sp, acc_prop, st);
        return launch_sph<double, 2>(h, tg, ntiles, csR, cap, nbr, nn, stride, aux, sp, acc_prop, st);
    }
    if (P == 4) return launch_sph<float, 4>(h, tg, ntiles, csR, cap, nbr, nn, stride, aux, sp, acc_prop, st);
    if (P == 1) return launch_sph<float, 1>(h, tg, ntiles, csR, cap, nbr, nn, stride, aux, sp, acc_prop, st);
    return launch_sph<float, 2>(h, tg, ntiles, csR, cap, nbr, nn, stride, aux, sp, acc_prop, st);
}

bool sph_tile_fits(pd_vd h, unsigned int tmax) { return 2L * tmax * h->pos_bytes <= 200L * 1024 && tmax <= 65535u; }

}  // namespace pd
