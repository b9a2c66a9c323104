// pd_md.cu -- Lennard-Jones pair kernels and the velocity-Verlet driver.
//
// The reference has no LJ physics (its pair functors are test sums,
// vector_dist_gpu_unit_tests.cu:46-119, and vector_dist_performance_common.hpp:18-85);
// the kernels follow that functor pattern -- one thread per domain particle
// walking its neighbours -- with the LJ 12-6 pair force of a plain cutoff:
//   F_i = sum_j 24 eps (2 (s/r)^12 - (s/r)^6) / r^2 * (x_i - x_j),   r < r_cut
//   U   = 1/2 sum_i sum_j 4 eps ((s/r)^12 - (s/r)^6)
// Velocity Verlet (Swope et al. 1982): v += dt/2 f/m; x += dt v; [rebuild or
// refresh images]; f = F(x); v += dt/2 f/m.  Energies are reduced in FP64 with a
// fixed block order (deterministic).
#include <utility>
#include "pd_device.cuh"
#include "pd_internal.cuh"
#include "pd_lj.cuh"
#include "pd_tile.cuh"
#include "pd_mixed.cuh"
#include "pd_sph.cuh"
#include "pd_md.cuh"

namespace pd {

static constexpr int FBLOCK = 256;

template <class T>
__global__ void __launch_bounds__(FBLOCK) k_lj_verlet(const typename V4<T>::type* __restrict__ pos, long n,
                                                      const int* __restrict__ nbr, const int* __restrict__ nn,
                                                      long stride, LJP<T> P, T* __restrict__ f, long fcap,
                                                      double* __restrict__ part) {
    double pe = 0, vir = 0;
    for (long i = blockIdx.x * (long)FBLOCK + threadIdx.x; i < n; i += (long)gridDim.x * FBLOCK) {
        typename V4<T>::type xi = ld4(pos, i);
        int m = nn[i];
        T fx = 0, fy = 0, fz = 0, e = 0, w = 0;
        const int* row = nbr + i;
#pragma unroll 4
        for (int k = 0; k < m; ++k) {
            int q = __ldg(row + (long)k * stride);
            typename V4<T>::type xq = ld4(pos, q);
            T dx = xi.x - xq.x, dy = xi.y - xq.y, dz = xi.z - xq.z;
            T r2 = dist2(dx, dy, dz);
            if (r2 < P.rc2 && q != (int)i) lj_acc(P, r2, dx, dy, dz, fx, fy, fz, e, w);
        }
        f[i] = fx;
        f[fcap + i] = fy;
        f[2 * fcap + i] = fz;
        pe += 0.5 * (double)e;
        vir += 0.5 * (double)w;
    }
    pe = block_sum<double, FBLOCK>(pe);
    vir = block_sum<double, FBLOCK>(vir);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = pe;
        part[2 * blockIdx.x + 1] = vir;
    }
}

// the half-list pair rule: an image is kept iff it lies after p in (x, y, z) order
template <class T4> __device__ __forceinline__ bool lex_after(const T4& a, const T4& b) {
    return a.x > b.x || (a.x == b.x && (a.y > b.y || (a.y == b.y && a.z > b.z)));
}

// LJ from a symmetric (half) Verlet list: each pair once, the reaction added to
// the partner (a domain particle or a periodic image) with atomics; image forces
// are folded onto their sources by ghost_put<add_>.  Energies count each pair
// once.  The forces must be zero on entry (domain and images).
template <class T>
__global__ void __launch_bounds__(FBLOCK) k_lj_verlet_sym(const typename V4<T>::type* __restrict__ pos, long n,
                                                          const int* __restrict__ nbr, const int* __restrict__ nn,
                                                          long stride, LJP<T> P, T* __restrict__ f, long fcap,
                                                          double* __restrict__ part) {
    double pe = 0, vir = 0;
    for (long i = blockIdx.x * (long)FBLOCK + threadIdx.x; i < n; i += (long)gridDim.x * FBLOCK) {
        typename V4<T>::type xi = ld4(pos, i);
        int m = nn[i];
        T fx = 0, fy = 0, fz = 0, e = 0, w = 0;
        const int* row = nbr + i;
        for (int k = 0; k < m; ++k) {
            int q = __ldg(row + (long)k * stride);
            typename V4<T>::type xq = ld4(pos, q);
            T dx = xi.x - xq.x, dy = xi.y - xq.y, dz = xi.z - xq.z;
            T r2 = dist2(dx, dy, dz);
            if (r2 < P.rc2 && q != (int)i) {
                T gx = 0, gy = 0, gz = 0;
                lj_acc(P, r2, dx, dy, dz, gx, gy, gz, e, w);
                fx += gx;
                fy += gy;
                fz += gz;
                atomicAdd(f + q, -gx);
                atomicAdd(f + fcap + q, -gy);
                atomicAdd(f + 2 * fcap + q, -gz);
            }
        }
        atomicAdd(f + i, fx);
        atomicAdd(f + fcap + i, fy);
        atomicAdd(f + 2 * fcap + i, fz);
        pe += (double)e;
        vir += (double)w;
    }
    pe = block_sum<double, FBLOCK>(pe);
    vir = block_sum<double, FBLOCK>(vir);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = pe;
        part[2 * blockIdx.x + 1] = vir;
    }
}

// LJ through the cell list (27-cell walk over the cell-ordered positions pcs,
// whose 4th word holds the original index)
template <class T> struct IdxDec;
template <> struct IdxDec<double> {
    __device__ static int dec(double w) { return (int)__double_as_longlong(w); }
};
template <> struct IdxDec<float> {
    __device__ static int dec(float w) { return __float_as_int(w); }
};

template <class T>
__global__ void __launch_bounds__(FBLOCK) k_lj_cell(const typename V4<T>::type* __restrict__ pos, long n,
                                                    const typename V4<T>::type* __restrict__ pcs,
                                                    const unsigned int* __restrict__ cs, Grid<T> G, LJP<T> P,
                                                    T* __restrict__ f, long fcap, int sym,
                                                    double* __restrict__ part) {
    double pe = 0, vir = 0;
    const T half = sym ? T(1) : T(0.5);
    for (long i = blockIdx.x * (long)FBLOCK + threadIdx.x; i < n; i += (long)gridDim.x * FBLOCK) {
        typename V4<T>::type xi = ld4(pos, i);
        unsigned int bad = 0;
        int c0 = G.coord(0, xi.x, bad), c1 = G.coord(1, xi.y, bad), c2 = G.coord(2, xi.z, bad);
        T fx = 0, fy = 0, fz = 0, e = 0, w = 0;
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy) {
                int y = c1 + dy, z = c2 + dz;
                if (y < 0 || z < 0 || y >= G.gs[1] || z >= G.gs[2]) continue;
                int xa = max(c0 - 1, 0), xb = min(c0 + 1, G.gs[0] - 1);
                long rb = (long)G.gs[0] * (y + (long)G.gs[1] * z);
                unsigned int a = cs[rb + xa], b = cs[rb + xb + 1];
                for (unsigned int k = a; k < b; ++k) {
                    typename V4<T>::type xq = ld4(pcs, k);
                    const int qi = IdxDec<T>::dec(xq.w);
                    if (qi == (int)i) continue;
                    // symmetric cell list: each pair once (the half-list rule of pd_verlet.cu)
                    if (sym && !(qi < n ? qi > (int)i : lex_after(xq, xi))) continue;
                    T dx = xi.x - xq.x, dy2 = xi.y - xq.y, dz2 = xi.z - xq.z;
                    T r2 = dist2(dx, dy2, dz2);
                    if (r2 < P.rc2) {
                        if (sym) {
                            T gx = 0, gy = 0, gz = 0;
                            lj_acc(P, r2, dx, dy2, dz2, gx, gy, gz, e, w);
                            fx += gx;
                            fy += gy;
                            fz += gz;
                            atomicAdd(f + qi, -gx);
                            atomicAdd(f + fcap + qi, -gy);
                            atomicAdd(f + 2 * fcap + qi, -gz);
                        } else {
                            lj_acc(P, r2, dx, dy2, dz2, fx, fy, fz, e, w);
                        }
                    }
                }
            }
        if (sym) {
            atomicAdd(f + i, fx);
            atomicAdd(f + fcap + i, fy);
            atomicAdd(f + 2 * fcap + i, fz);
        } else {
            f[i] = fx;
            f[fcap + i] = fy;
            f[2 * fcap + i] = fz;
        }
        pe += (double)(half * e);
        vir += (double)(half * w);
    }
    pe = block_sum<double, FBLOCK>(pe);
    vir = block_sum<double, FBLOCK>(vir);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = pe;
        part[2 * blockIdx.x + 1] = vir;
    }
}

template <class T>
__global__ void k_gather_cs2(const typename V4<T>::type* __restrict__ pos, const int* __restrict__ sorted, long n,
                             typename V4<T>::type* __restrict__ out) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        int i = sorted[k];
        typename V4<T>::type r = ld4(pos, i);
        if (sizeof(T) == 8) r.w = __longlong_as_double((long long)i);
        else r.w = __int_as_float(i);
        st4(out, k, r);
    }
}

// the same gather bounded by the device count of real particles + images
template <class T>
__global__ void k_gather_cs2_dev(const typename V4<T>::type* __restrict__ pos, const int* __restrict__ sorted,
                                 long bound, const unsigned int* __restrict__ n_img, long n_real,
                                 typename V4<T>::type* __restrict__ out) {
    long n = n_real + (long)*n_img;
    if (n > bound) n = bound;
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        int i = sorted[k];
        typename V4<T>::type r = ld4(pos, i);
        if (sizeof(T) == 8) r.w = __longlong_as_double((long long)i);
        else r.w = __int_as_float(i);
        st4(out, k, r);
    }
}

// v += h f ; x += dt v ; largest |x - xb|^2
template <class T>
__global__ void __launch_bounds__(FBLOCK) k_kick_drift(typename V4<T>::type* __restrict__ pos,
                                                       const typename V4<T>::type* __restrict__ xb, T* __restrict__ v,
                                                       const T* __restrict__ f, long cap, long n, T half, T dt,
                                                       unsigned long long* __restrict__ maxd2, T* __restrict__ sxy,
                                                       T* __restrict__ sz) {
    double mx = 0;
    for (long i = blockIdx.x * (long)FBLOCK + threadIdx.x; i < n; i += (long)gridDim.x * FBLOCK) {
        typename V4<T>::type x = ld4(pos, i);
        T vx = v[i] + half * f[i];
        T vy = v[cap + i] + half * f[cap + i];
        T vz = v[2 * cap + i] + half * f[2 * cap + i];
        x.x += dt * vx;
        x.y += dt * vy;
        x.z += dt * vz;
        v[i] = vx;
        v[cap + i] = vy;
        v[2 * cap + i] = vz;
        st4(pos, i, x);
        if (sxy) {  // the pair kernel's staging copies
            sxy[2 * i] = x.x;
            sxy[2 * i + 1] = x.y;
            sz[i] = x.z;
        }
        typename V4<T>::type b = ld4(xb, i);
        T dx = x.x - b.x, dy = x.y - b.y, dz = x.z - b.z;
        mx = fmax(mx, (double)dist2(dx, dy, dz));
    }
    mx = warp_max(mx);
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(maxd2, mx);
}

// The end of one step and the start of the next in one pass: v += h f (the
// closing half kick, kinetic energy partials of that step), then v += h f and
// x += dt v (the next step's opening half kick and drift), largest |x - xb|^2.
// The same operations in the same order as k_kick followed by k_kick_drift.
template <class T>
__global__ void __launch_bounds__(FBLOCK) k_kick_kick_drift(typename V4<T>::type* __restrict__ pos,
                                                            const typename V4<T>::type* __restrict__ xb,
                                                            T* __restrict__ v, const T* __restrict__ f, long cap, long n,
                                                            T half, T dt, double mass,
                                                            unsigned long long* __restrict__ maxd2,
                                                            double* __restrict__ part, T* __restrict__ sxy,
                                                            T* __restrict__ sz) {
    double ke = 0, mx = 0;
    for (long i = blockIdx.x * (long)FBLOCK + threadIdx.x; i < n; i += (long)gridDim.x * FBLOCK) {
        const T fx = f[i], fy = f[cap + i], fz = f[2 * cap + i];
        T vx = v[i] + half * fx;
        T vy = v[cap + i] + half * fy;
        T vz = v[2 * cap + i] + half * fz;
        ke += 0.5 * mass * ((double)vx * vx + (double)vy * vy + (double)vz * vz);
        vx = vx + half * fx;
        vy = vy + half * fy;
        vz = vz + half * fz;
        typename V4<T>::type x = ld4(pos, i);
        x.x += dt * vx;
        x.y += dt * vy;
        x.z += dt * vz;
        v[i] = vx;
        v[cap + i] = vy;
        v[2 * cap + i] = vz;
        st4(pos, i, x);
        if (sxy) {  // the pair kernel's staging copies
            sxy[2 * i] = x.x;
            sxy[2 * i + 1] = x.y;
            sz[i] = x.z;
        }
        typename V4<T>::type b = ld4(xb, i);
        T dx = x.x - b.x, dy = x.y - b.y, dz = x.z - b.z;
        mx = fmax(mx, (double)dist2(dx, dy, dz));
    }
    mx = warp_max(mx);
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(maxd2, mx);
    ke = block_sum<double, FBLOCK>(ke);
    if (threadIdx.x == 0) part[blockIdx.x] = ke;
}

// v += h f ; kinetic energy partial sums
template <class T>
__global__ void __launch_bounds__(FBLOCK) k_kick(T* __restrict__ v, const T* __restrict__ f, long cap, long n, T half,
                                                 double mass, double* __restrict__ part) {
    double ke = 0;
    for (long i = blockIdx.x * (long)FBLOCK + threadIdx.x; i < n; i += (long)gridDim.x * FBLOCK) {
        T vx = v[i] + half * f[i];
        T vy = v[cap + i] + half * f[cap + i];
        T vz = v[2 * cap + i] + half * f[2 * cap + i];
        v[i] = vx;
        v[cap + i] = vy;
        v[2 * cap + i] = vz;
        ke += 0.5 * mass * ((double)vx * vx + (double)vy * vy + (double)vz * vz);
    }
    ke = block_sum<double, FBLOCK>(ke);
    if (threadIdx.x == 0) part[blockIdx.x] = ke;
}

// KE only (initial state)
template <class T>
__global__ void __launch_bounds__(FBLOCK) k_ke(const T* __restrict__ v, long cap, long n, double mass,
                                               double* __restrict__ part) {
    double ke = 0;
    for (long i = blockIdx.x * (long)FBLOCK + threadIdx.x; i < n; i += (long)gridDim.x * FBLOCK) {
        double vx = v[i], vy = v[cap + i], vz = v[2 * cap + i];
        ke += 0.5 * mass * (vx * vx + vy * vy + vz * vz);
    }
    ke = block_sum<double, FBLOCK>(ke);
    if (threadIdx.x == 0) part[blockIdx.x] = ke;
}

template <class T> __global__ void k_recip_check(const T* __restrict__ x, T* __restrict__ y, long n) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        y[i] = recip(x[i]);
}

// first stage of a fixed-order sum of (pe, vir) pairs: block b sums a fixed chunk
__global__ void k_sum_pairs(const double* __restrict__ in, long n, long chunk, double* __restrict__ out) {
    double a = 0, b = 0;
    long beg = (long)blockIdx.x * chunk, end = min(beg + chunk, n);
    for (long i = beg + threadIdx.x; i < end; i += 256) {
        a += in[2 * i];
        b += in[2 * i + 1];
    }
    a = block_sum<double, 256>(a);
    b = block_sum<double, 256>(b);
    if (threadIdx.x == 0) {
        out[2 * blockIdx.x] = a;
        out[2 * blockIdx.x + 1] = b;
    }
}

// the same for (pe, vir, ke) triples: out[3b + q]
__global__ void k_sum_triples(const double* __restrict__ in, long n, long chunk, double* __restrict__ out) {
    double a = 0, b = 0, c = 0;
    long beg = (long)blockIdx.x * chunk, end = min(beg + chunk, n);
    for (long i = beg + threadIdx.x; i < end; i += 256) {
        a += in[3 * i];
        b += in[3 * i + 1];
        c += in[3 * i + 2];
    }
    a = block_sum<double, 256>(a);
    b = block_sum<double, 256>(b);
    c = block_sum<double, 256>(c);
    if (threadIdx.x == 0) {
        out[3 * blockIdx.x] = a;
        out[3 * blockIdx.x + 1] = b;
        out[3 * blockIdx.x + 2] = c;
    }
}

// E = (KE, PE, virial, rebuilt) from nb (pe, vir, ke) triples
__global__ void k_energy3(const double* __restrict__ part, int nb, const unsigned int* __restrict__ rebuilt,
                          double* __restrict__ E) {
    double a = 0, b = 0, c = 0;
    for (int i = threadIdx.x; i < nb; i += 256) {
        a += part[3 * i + 2];
        b += part[3 * i];
        c += part[3 * i + 1];
    }
    a = block_sum<double, 256>(a);
    b = block_sum<double, 256>(b);
    c = block_sum<double, 256>(c);
    if (threadIdx.x == 0) {
        E[0] = a;
        E[1] = b;
        E[2] = c;
        E[3] = rebuilt ? (double)*rebuilt : 0.0;
    }
}

// E[s] = (KE, PE, virial, rebuilt) from the fixed-order partials
__global__ void k_energy(const double* __restrict__ fpart, int nbf, const double* __restrict__ kpart, int nbk,
                         const unsigned int* __restrict__ rebuilt, double* __restrict__ E) {
    __shared__ double sh[3][256];
    double a = 0, b = 0, c = 0;
    for (int i = threadIdx.x; i < nbk; i += 256) a += kpart[i];
    for (int i = threadIdx.x; i < nbf; i += 256) {
        b += fpart[2 * i];
        c += fpart[2 * i + 1];
    }
    sh[0][threadIdx.x] = a;
    sh[1][threadIdx.x] = b;
    sh[2][threadIdx.x] = c;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int q = 0; q < 3; ++q) sh[q][threadIdx.x] += sh[q][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        E[0] = sh[0][0];
        E[1] = sh[1][0];
        E[2] = sh[2][0];
        E[3] = rebuilt ? (double)*rebuilt : 0.0;
    }
}

// k_energy writing the row of a device step counter, which it advances (captured
// steps: the same graph writes successive rows)
__global__ void k_energy_idx(const double* __restrict__ fpart, int nbf, const double* __restrict__ kpart, int nbk,
                             double rebuilt, double* __restrict__ E, int* __restrict__ idx) {
    __shared__ double sh[3][256];
    double a = 0, b = 0, c = 0;
    for (int i = threadIdx.x; i < nbk; i += 256) a += kpart[i];
    for (int i = threadIdx.x; i < nbf; i += 256) {
        b += fpart[2 * i];
        c += fpart[2 * i + 1];
    }
    sh[0][threadIdx.x] = a;
    sh[1][threadIdx.x] = b;
    sh[2][threadIdx.x] = c;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int q = 0; q < 3; ++q) sh[q][threadIdx.x] += sh[q][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double* e = E + 4 * (long)*idx;
        e[0] = sh[0][0];
        e[1] = sh[1][0];
        e[2] = sh[2][0];
        e[3] = rebuilt;
        *idx += 1;
    }
}

}  // namespace pd


namespace pd {

template <class T> static LJP<T> ljp(const pd_lj_params_t& lj) {
    LJP<T> P{};
    P.eps24 = (T)(24.0 * lj.eps);
    P.eps4 = (T)(4.0 * lj.eps);
    P.sig2 = (T)(lj.sigma * lj.sigma);
    T rc = (T)lj.r_cut;
    P.rc2 = rc * rc;
    return P;
}

template <class T> static Grid<T> grid_of(pd_cl cl) {
    Grid<T> G;
    for (int d = 0; d < 3; ++d) {
        G.lo[d] = (T)cl->box_lo[d];
        G.sp[d] = (T)cl->spacing[d];
        G.gs[d] = cl->gs[d];
    }
    G.pad = cl->pad;
    return G;
}

// forces of [0, n_real) into force_prop; partials (pe, vir) per block into part
static int lj_launch(pd_vd h, pd_vl vl, pd_cl cl, const pd_lj_params_t& lj, int force_prop, double* part, int nblk,
                     cudaStream_t st) {
    Prop& F = h->props[force_prop];
    long n = h->n_real;
    if (vl) {
        if (vl->sym) {
            // forces of domain particles and images start at zero (the images receive reactions)
            for (int c = 0; c < 3; ++c)
                PD_CUDA(cudaMemsetAsync(F.d + (size_t)c * h->cap * F.esize, 0, (size_t)h->n_total * F.esize, st));
            if (h->dtype == PD_F64)
                pd::launch(k_lj_verlet_sym<double>, nblk, FBLOCK, 0, st, (const double4*)h->pos, n,
                           (const int*)vl->nbr.as<int>(), (const int*)vl->nn.as<int>(), vl->stride, ljp<double>(lj),
                           (double*)F.d, h->cap, part);
            else
                pd::launch(k_lj_verlet_sym<float>, nblk, FBLOCK, 0, st, (const float4*)h->pos, n,
                           (const int*)vl->nbr.as<int>(), (const int*)vl->nn.as<int>(), vl->stride, ljp<float>(lj),
                           (float*)F.d, h->cap, part);
        } else if (h->dtype == PD_F64)
            pd::launch(k_lj_verlet<double>, nblk, FBLOCK, 0, st, (const double4*)h->pos, n, vl->nbr.as<int>(),
                                                         vl->nn.as<int>(), vl->stride, ljp<double>(lj), (double*)F.d,
                                                         h->cap, part);
        else
            pd::launch(k_lj_verlet<float>, nblk, FBLOCK, 0, st, (const float4*)h->pos, n, vl->nbr.as<int>(), vl->nn.as<int>(),
                                                        vl->stride, ljp<float>(lj), (float*)F.d, h->cap, part);
    } else {
        // cell-ordered copy of all positions for the walk
        long nt = h->n_total;
        const int sym = (cl->opt & PD_CL_SYMMETRIC) ? 1 : 0;
        if (sym)  // the images receive reactions: domain and image forces start at zero
            for (int c = 0; c < 3; ++c)
                PD_CUDA(cudaMemsetAsync(F.d + (size_t)c * h->cap * F.esize, 0, (size_t)nt * F.esize, st));
        PD_TRY(h->tmp.ensure((size_t)(nt > 0 ? nt : 1) * h->pos_bytes));
        unsigned g = grid_for(nt, 256);
        if (h->dtype == PD_F64) {
            pd::launch(k_gather_cs2<double>, g, 256, 0, st, (const double4*)h->pos, cl->sorted.as<int>(), nt,
                                                    h->tmp.as<double4>());
            pd::launch(k_lj_cell<double>, nblk, FBLOCK, 0, st, (const double4*)h->pos, n, h->tmp.as<double4>(),
                                                       cl->cell_start.as<unsigned int>(), grid_of<double>(cl),
                                                       ljp<double>(lj), (double*)F.d, h->cap, sym, part);
        } else {
            pd::launch(k_gather_cs2<float>, g, 256, 0, st, (const float4*)h->pos, cl->sorted.as<int>(), nt,
                                                   h->tmp.as<float4>());
            pd::launch(k_lj_cell<float>, nblk, FBLOCK, 0, st, (const float4*)h->pos, n, h->tmp.as<float4>(),
                                                      cl->cell_start.as<unsigned int>(), grid_of<float>(cl),
                                                      ljp<float>(lj), (float*)F.d, h->cap, sym, part);
        }
    }
    PD_LAUNCH_CHECK();
    return PD_OK;
}

int force_blocks(long n) {
    int sms = 148;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    long want = (n + FBLOCK - 1) / FBLOCK;
    long cap = (long)sms * 8;
    if (want > cap) want = cap;
    if (want < 1) want = 1;
    return (int)want;
}

// Tiled structure: the real particles are already in cell order (sort_cl holds
// their cell starts); sort the images by cell too, then build the tile-local rows.
static int md_tiles(pd_md md, pd_cl cl, cudaStream_t st) {
    pd_vd h = md->h;
    long nc1 = cl->ncells + 1;
    PD_TRY(md->csR.ensure(sizeof(unsigned int) * nc1));
    PD_TRY(md->csI.ensure(sizeof(unsigned int) * nc1));
    PD_CUDA(cudaMemcpyAsync(md->csR.p, cl->cell_start.p, sizeof(unsigned int) * nc1, cudaMemcpyDeviceToDevice, st));
    long m = h->n_img, n = h->n_real;
    PD_TRY(cl_build(h, cl, m, nullptr, st, n));
    PD_CUDA(cudaMemcpyAsync(md->csI.p, cl->cell_start.p, sizeof(unsigned int) * nc1, cudaMemcpyDeviceToDevice, st));
    h->img_gen_order = false;  // the images are sorted into cell order below
    if (m > 0) {
        const int* ids = cl->sorted.as<int>();
        size_t need = std::max((size_t)m * h->pos_bytes, (size_t)m * sizeof(int));
        PD_TRY(h->tmp2.ensure(need));
        char* pos_img = (char*)h->pos + (size_t)n * h->pos_bytes;
        PD_TRY(gather_bytes(pos_img, h->tmp2.p, ids, m, h->pos_bytes, st));
        PD_CUDA(cudaMemcpyAsync(pos_img, h->tmp2.p, (size_t)m * h->pos_bytes, cudaMemcpyDeviceToDevice, st));
        PD_TRY(gather_bytes(h->gid + n, h->tmp2.p, ids, m, 4, st));
        PD_CUDA(cudaMemcpyAsync(h->gid + n, h->tmp2.p, sizeof(int) * m, cudaMemcpyDeviceToDevice, st));
        PD_TRY(gather_bytes(h->img_src.p, h->tmp2.p, ids, m, 4, st));
        PD_CUDA(cudaMemcpyAsync(h->img_src.p, h->tmp2.p, sizeof(int) * m, cudaMemcpyDeviceToDevice, st));
        PD_TRY(gather_bytes(h->img_shift.p, h->tmp2.p, ids, m, 1, st));
        PD_CUDA(cudaMemcpyAsync(h->img_shift.p, h->tmp2.p, (size_t)m, cudaMemcpyDeviceToDevice, st));
    }
    int tx_req = md->tile_tx;
    if (tx_req == 0 && md->physics == 0) {
        // LJ: the widest tile with at most about 184 domain particles on average, from
        // the occupancy of the cells inside the box (the grid's ghost layers hold
        // images only).  A CTA of 256 threads at two lanes a particle takes 128 in a
        // first round; a second round of up to 64 runs at four lanes each, so most
        // lanes are busy in both while tiles stay below 192 (the rows are about
        // equally long).
        double inner = 1;
        for (int d = 0; d < 3; ++d) inner *= std::max(1.0, (h->hi[d] - h->lo[d]) / cl->spacing[d]);
        const double occ = std::max((double)n / inner, 1e-3);
        tx_req = std::max(1, std::min(TXMAX, (int)(184.0 / occ)));
    }
    PD_TRY(tile_plan(cl, n, tx_req, md->tg, md->ntiles));
    unsigned int tmax = 0, cmax = 0;
    for (;;) {
        PD_TRY(tile_sizes(h, md->tg, md->ntiles, md->csR.as<unsigned int>(), md->csI.as<unsigned int>(), tmax, cmax,
                          st));
        if (md->physics == 1 ? sph_tile_fits(h, tmax) : tile_fits(h, tmax)) break;
        // the densest tile does not fit: narrower tiles (the width is a performance choice only)
        if (md->tg.TX <= 1) return PD_OK;  // stays on global rows
        PD_TRY(tile_plan(cl, n, md->tg.TX / 2, md->tg, md->ntiles));
    }
    if (md->tile_tx == 0 && md->physics == 1 && md->tg.TX > 1) {
        // automatic width for SPH: the densest tile's two staged records within about
        // 60 KB in FP64 (tiles of two or more cells, three CTAs per SM) or 48 KB in
        // FP32; the mean occupancy counts the empty part of the tank, so the width
        // is rescaled from the measured largest tile
        const long target = (h->dtype == PD_F64 ? 60L : 48L) * 1024 / (2L * h->pos_bytes);
        if ((long)tmax > target) {
            int tx = (int)((double)(md->tg.TX + 2) * (double)target / (double)tmax) - 2;
            if (tx < 1) tx = 1;
            if (tx < md->tg.TX) {
                PD_TRY(tile_plan(cl, n, tx, md->tg, md->ntiles));
                PD_TRY(tile_sizes(h, md->tg, md->ntiles, md->csR.as<unsigned int>(), md->csI.as<unsigned int>(), tmax,
                                  cmax, st));
            }
        }
    }
    md->tcap = tmax;
    PD_TRY(tile_build(h, md->tg, md->ntiles, md->csR.as<unsigned int>(), md->csI.as<unsigned int>(), md->tcap,
                      md->vl->r_cut, md->pos32, md->tnbr, md->tnn, md->tstride, md->tmax_nn, st));
    PD_TRY(md->tpart.ensure(sizeof(double) * 3 * ((md->ntiles > 0 ? md->ntiles : 1) + 256)));
    md->tiles_active = true;
    return PD_OK;
}

// wrap, sort the real particles into cell order, periodic images, neighbour structure
// the FP64 tiled pair kernel reads (x, y) / z copies of the positions, refreshed by
// the rebuild, the drift (real particles) and the image replay
static bool md_split(pd_md md) {
    return md->physics == 0 && !md->mixed && md->tiles_active && !md->mp.use_cell_list && md->h->dtype == PD_F64;
}

// The properties the cell-order reorder carries: all but those the step recomputes
// before it reads them (the force; for SPH also the density rate), so that every
// other property stays with its particle.
static unsigned long md_reorder_mask(pd_md md) {
    const int np = (int)md->h->props.size();
    unsigned long m = np >= 64 ? ~0ul : ((1ul << np) - 1);
    m &= ~(1ul << md->mp.force_prop);
    if (md->physics == 1) m &= ~(1ul << md->sp.drho_prop);
    return m;
}

int md_rebuild(pd_md md, cudaStream_t st) {
    pd_vd h = md->h;
    if (md->mixed && md->off_valid) PD_TRY(mixed_to_positions(h, md->vl->cl, md->off, st));
    h->n_total = h->n_real;
    h->img_valid = false;
    PD_TRY(wrap_positions(h, h->n_real, st));
    pd_cl sort_cl = md->mp.use_cell_list ? md->cl : md->vl->cl;
    PD_TRY(cl_build(h, sort_cl, h->n_real, nullptr, st));
    // the plain FP64 path: the reorder also writes the build positions and the pair
    // kernel's staging copies of the real particles
    const bool split_cand = md->physics == 0 && !md->mixed && !md->mp.use_cell_list && h->dtype == PD_F64;
    bool extra_done = false;
    PD_TRY(md->xb.ensure((size_t)(h->n_real > 0 ? h->n_real : 1) * h->pos_bytes));  // room for the build positions
    if (split_cand) {
        const size_t cap = (size_t)(h->cap > 0 ? h->cap : 1);
        PD_TRY(md->sxy.ensure(cap * sizeof(double2)));
        PD_TRY(md->sz.ensure(cap * sizeof(double)));
        const ReorderExtra ex{md->xb.as<double4>(), md->sxy.as<double2>(), md->sz.as<double>()};
        PD_TRY(cl_reorder(h, sort_cl, h->n_real, md_reorder_mask(md), true, true, st, md->swap_reorder, &ex,
                          &extra_done));
    } else {
        PD_TRY(cl_reorder(h, sort_cl, h->n_real, md_reorder_mask(md), true, true, st, md->swap_reorder));
    }
    if (h->nbox == 0) PD_TRY(ghost_boxes_upload(h, st));
    PD_TRY(ghost_generate(h, 0, true, st));
    if (md->mp.use_cell_list) {
        PD_TRY(cl_build(h, md->cl, h->n_total, nullptr, st));
    } else {
        md->tiles_active = false;
        if (md->use_tiles || md->mixed || md->physics == 1) PD_TRY(md_tiles(md, sort_cl, st));
        if (md->physics == 1) {
            if (!md->tiles_active) {
                set_error("SPH: a tile's neighbourhood does not fit in shared memory");
                return PD_EOVERFLOW;
            }
            PD_TRY(sph_pack(h, md->sp, md->mp.vel_prop, md->aux, st));
        }
        if (md->mixed) {
            if (!md->tiles_active) {
                set_error("precision form: a tile's neighbourhood does not fit in shared memory");
                return PD_EOVERFLOW;
            }
            PD_TRY(mixed_from_positions(h, md->vl->cl, md->off, md->offK, st));
            md->off_valid = true;
            PD_TRY(md->offb.ensure(sizeof(float4) * (size_t)(h->n_real > 0 ? h->n_real : 1)));
            PD_CUDA(cudaMemcpyAsync(md->offb.p, md->off.p, sizeof(float4) * h->n_real, cudaMemcpyDeviceToDevice, st));
        } else {
            if (!md->tiles_active) PD_TRY(verlet_build(h, md->vl, h->n_real, nullptr, st, true));
            if (!extra_done)
                PD_CUDA(cudaMemcpyAsync(md->xb.p, h->pos, (size_t)h->n_real * h->pos_bytes, cudaMemcpyDeviceToDevice,
                                        st));
            if (md_split(md)) {
                // the reorder wrote the real particles' copies, unless the images grew the
                // vector's capacity since (tile_split then takes larger, new buffers)
                const size_t cap = (size_t)(h->cap > 0 ? h->cap : 1);
                const bool kept = extra_done && md->sxy.bytes >= cap * sizeof(double2) &&
                                  md->sz.bytes >= cap * sizeof(double);
                const long first = kept ? h->n_real : 0;
                PD_TRY(tile_split(h, md->sxy, md->sz, first, h->n_total - first, st));
            }
        }
    }
    h->epoch++;
    md->builds++;
    return PD_OK;
}

int md_forces(pd_md md, cudaStream_t st, const DriftArgs* drift) {
    if (drift && !(md->tiles_active && md->physics == 0 && !md->mixed)) {
        set_error("md_forces: the fused drift is the plain tiled path's");
        return PD_EINVAL;
    }
    if (md->physics == 1)
        return sph_rates(md->h, md->tg, md->ntiles, md->csR.as<unsigned int>(), md->tcap, md->tnbr, md->tnn,
                         md->tstride, md->aux, md->sp, md->mp.force_prop, md->tile_p, st);
    if (md->mixed)
        return mixed_lj(md->h, md->vl->cl, md->tg, md->ntiles, md->csR.as<unsigned int>(), md->csI.as<unsigned int>(),
                        md->tcap, md->off, md->tnbr, md->tnn, md->tstride, md->lj, md->mp.force_prop,
                        md->tpart.as<double>(), md->tile_p, md->tile_block, st);
    if (md->tiles_active)
        return tile_lj(md->h, md->tg, md->ntiles, md->csR.as<unsigned int>(), md->csI.as<unsigned int>(), md->tcap,
                       md->tnbr, md->tnn, md->tstride, md->lj, md->mp.force_prop, md->tpart.as<double>(), true,
                       md->tile_p, md->sxy, md->sz, st, drift);
    return lj_launch(md->h, md->mp.use_cell_list ? nullptr : md->vl, md->mp.use_cell_list ? md->cl : nullptr, md->lj,
                     md->mp.force_prop, md->fpart.as<double>(), md->nblk, st);
}

}  // namespace pd

using namespace pd;

namespace pd {

// One velocity-Verlet step of the LJ driver in cell-list mode (cell list rebuilt
// every step) with no host synchronisation: the image count stays on the device
// (ghost_generate without the read-back, capacity img_cap) and bounds the image
// cell sort and the gather.  The same operations as the synchronous step.
template <class T>
static int md_step_cl(pd_md md, cudaStream_t st, long img_cap) {
    typedef typename V4<T>::type T4;
    pd_vd h = md->h;
    pd_cl cl = md->cl;
    const long n = h->n_real;
    Prop& V = h->props[md->mp.vel_prop];
    Prop& F = h->props[md->mp.force_prop];
    const T half = (T)(0.5 * md->mp.dt / md->mp.mass);
    PD_CUDA(cudaMemsetAsync(&h->ctrl->maxdisp2, 0, sizeof(unsigned long long), st));
    pd::launch(k_kick_drift<T>, md->nblk, FBLOCK, 0, st, (T4*)h->pos, md->xb.as<T4>(), (T*)V.d, (const T*)F.d, h->cap,
               n, half, (T)md->mp.dt, &h->ctrl->maxdisp2, (T*)nullptr, (T*)nullptr);
    PD_LAUNCH_CHECK();
    h->n_total = n;
    h->img_valid = false;
    PD_TRY(wrap_positions(h, n, st));
    PD_TRY(cl_build(h, cl, n, nullptr, st));
    PD_TRY(cl_reorder(h, cl, n, md_reorder_mask(md), true, true, st));
    PD_TRY(ghost_generate(h, img_cap, false, st));
    PD_TRY(cl_build(h, cl, n + img_cap, &h->ctrl->n_img, st));
    const long bound = n + img_cap;
    PD_TRY(h->tmp.ensure((size_t)bound * h->pos_bytes));
    pd::launch(k_gather_cs2_dev<T>, grid_for(bound, 256), 256, 0, st, (const T4*)h->pos, cl->sorted.as<int>(), bound,
               (const unsigned int*)&h->ctrl->n_img, n, h->tmp.as<T4>());
    pd::launch(k_lj_cell<T>, md->nblk, FBLOCK, 0, st, (const T4*)h->pos, n, h->tmp.as<T4>(),
               cl->cell_start.as<unsigned int>(), grid_of<T>(cl), ljp<T>(md->lj), (T*)F.d, h->cap, 0,
               md->fpart.as<double>());
    pd::launch(k_kick<T>, md->nblk, FBLOCK, 0, st, (T*)V.d, (const T*)F.d, h->cap, n, half, md->mp.mass,
               md->kpart.as<double>());
    pd::launch(k_energy_idx, 1, 256, 0, st, (const double*)md->fpart.as<double>(), md->nblk,
               (const double*)md->kpart.as<double>(), md->nblk, 1.0, md->E.as<double>(), md->eidx.as<int>());
    PD_LAUNCH_CHECK();
    return PD_OK;
}

static int md_step_cl_any(pd_md md, cudaStream_t st, long img_cap) {
    return md->h->dtype == PD_F64 ? md_step_cl<double>(md, st, img_cap) : md_step_cl<float>(md, st, img_cap);
}

// every buffer address and size a captured cell-list step uses: the graph holds
// them as raw values, so it is captured again when any of them changed
static std::vector<uintptr_t> cl_graph_key(pd_md md) {
    pd_vd h = md->h;
    pd_cl cl = md->cl;
    std::vector<uintptr_t> k = {(uintptr_t)h->pos, (uintptr_t)h->gid, (uintptr_t)h->cap, (uintptr_t)h->n_real,
                                (uintptr_t)md->E.p, (uintptr_t)md->eidx.p, (uintptr_t)md->kpart.p,
                                (uintptr_t)md->fpart.p, (uintptr_t)md->xb.p, (uintptr_t)cl->cell_start.p,
                                (uintptr_t)cl->cell_cnt.p, (uintptr_t)cl->sorted.p, (uintptr_t)cl->sorted_tmp.p,
                                (uintptr_t)cl->cell_of.p, (uintptr_t)cl->slot.p, (uintptr_t)h->tmp.p,
                                (uintptr_t)h->tmp2.p, (uintptr_t)h->img_src.p, (uintptr_t)h->img_shift.p,
                                (uintptr_t)h->img_cnt.p, (uintptr_t)h->img_start.p, (uintptr_t)h->boxes.p,
                                (uintptr_t)h->shifts.p, (uintptr_t)h->scan_scratch.p, (uintptr_t)md->gcl_img_cap};
    for (auto& P : h->props) k.push_back((uintptr_t)P.d);
    return k;
}

// cell-list mode: the first step of a run sizes every buffer, the step is
// captured once as a CUDA graph (on a private stream: the legacy stream cannot
// capture) and the remaining steps are graph launches on the caller's stream
static int md_run_cl_graph(pd_md md, int steps, cudaStream_t st, double* E) {
    pd_vd h = md->h;
    if (!md->ready) {
        PD_TRY(md_rebuild(md, st));
        PD_TRY(md_forces(md, st));
        md->ready = true;
        md->gcl_img_cap = 0;
    }
    PD_TRY(md->E.ensure(sizeof(double) * 4 * (steps + 1)));
    PD_TRY(md->eidx.ensure(sizeof(int)));
    PD_CUDA(cudaMemsetAsync(md->eidx.p, 0, sizeof(int), st));
    int s0 = 0;
    if (md->gcl && cl_graph_key(md) != md->gcl_key) {
        // something the graph captured was reallocated or resized since: capture again
        PD_CUDA(cudaStreamSynchronize(st));
        cudaGraphExecDestroy(md->gcl);
        md->gcl = nullptr;
    }
    if (!md->gcl) {
        PD_TRY(read_ctrl(h, st));
        const long m = h->ctrl_h->n_img;
        md->gcl_img_cap = m + m / 2 + 1024;
        PD_TRY(ensure_capacity(h, h->n_real + md->gcl_img_cap + 1, st));
        if (steps > 0) {
            PD_TRY(md_step_cl_any(md, st, md->gcl_img_cap));  // also sizes the buffers the graph uses
            s0 = 1;
        }
        PD_CUDA(cudaStreamSynchronize(st));
        if (!md->gst) PD_CUDA(cudaStreamCreateWithFlags(&md->gst, cudaStreamNonBlocking));
        cudaGraph_t g = nullptr;
        const unsigned long long l0 = pd_launch_count();
        PD_CUDA(cudaStreamBeginCapture(md->gst, cudaStreamCaptureModeThreadLocal));
        g_capturing = true;
        int rc = md_step_cl_any(md, md->gst, md->gcl_img_cap);
        g_capturing = false;
        cudaError_t ce = cudaStreamEndCapture(md->gst, &g);
        md->gcl_kernels = pd_launch_count() - l0;
        __atomic_fetch_sub(&g_launches, md->gcl_kernels, __ATOMIC_RELAXED);  // captured, not launched
        if (rc != PD_OK || ce != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            set_error("cell-list step capture failed: %s", cudaGetErrorString(ce));
            return rc != PD_OK ? rc : PD_ECUDA;
        }
        ce = cudaGraphInstantiate(&md->gcl, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) {
            md->gcl = nullptr;
            set_error("cell-list step graph: %s", cudaGetErrorString(ce));
            return PD_ECUDA;
        }
        md->gcl_key = cl_graph_key(md);
    }
    for (int s = s0; s < steps; ++s) PD_CUDA(cudaGraphLaunch(md->gcl, st));
    __atomic_fetch_add(&g_launches, (unsigned long long)(steps - s0) * md->gcl_kernels, __ATOMIC_RELAXED);
    md->steps += steps;
    md->builds += steps;
    if (E && steps > 0) PD_CUDA(cudaMemcpyAsync(E, md->E.p, sizeof(double) * 4 * steps, cudaMemcpyDeviceToHost, st));
    PD_CUDA(cudaStreamSynchronize(st));
    PD_TRY(read_ctrl(h, st));
    h->n_img = h->ctrl_h->n_img;
    h->n_total = h->n_real + h->n_img;
    h->img_valid = true;
    h->img_gen_order = false;  // the step may leave the images in cell order
    if (h->ctrl_h->err & (ERR_IMG_OVERFLOW | ERR_NN_OVERFLOW | ERR_CAP_OVERFLOW)) {
        set_error("pd_md_run: device capacity overflow (err=0x%x)", h->ctrl_h->err);
        return PD_EOVERFLOW;
    }
    return PD_OK;
}

}  // namespace pd

extern "C" {

int pd_selftest_recip(int dtype, const void* x_host, void* out_host, long n) {
    if ((dtype != PD_F32 && dtype != PD_F64) || !x_host || !out_host || n < 0) return PD_EINVAL;
    if (n == 0) return PD_OK;
    size_t es = dtype == PD_F64 ? 8 : 4;
    Buf a, b;
    PD_TRY(a.ensure(es * n));
    PD_TRY(b.ensure(es * n));
    PD_CUDA(cudaMemcpy(a.p, x_host, es * n, cudaMemcpyHostToDevice));
    if (dtype == PD_F64) pd::launch(k_recip_check<double>, grid_for(n, 256), 256, 0, (cudaStream_t)0, a.as<const double>(), b.as<double>(), n);
    else pd::launch(k_recip_check<float>, grid_for(n, 256), 256, 0, (cudaStream_t)0, a.as<const float>(), b.as<float>(), n);
    PD_LAUNCH_CHECK();
    PD_CUDA(cudaMemcpy(out_host, b.p, es * n, cudaMemcpyDeviceToHost));
    a.release();
    b.release();
    return PD_OK;
}

int pd_lj_forces(pd_vd h, pd_vl vl, pd_cl cl, const pd_lj_params_t* lj, int force_prop, void* stream,
                 double* energy) {
    if (!h || !lj || (!vl && !cl) || force_prop < 0 || force_prop >= (int)h->props.size()) return PD_EINVAL;
    Prop& F = h->props[force_prop];
    if (F.type != h->dtype || F.ncomp < 3) {
        set_error("pd_lj_forces: force property must have 3 components of the vector's dtype");
        return PD_EINVAL;
    }
    if (vl && vl->n_dom != h->n_real) {
        set_error("pd_lj_forces: Verlet list is stale (update it after map/ghost_get)");
        return PD_ESTALE;
    }
    if (!vl && cl->n_part != h->n_total) {
        set_error("pd_lj_forces: cell list is stale");
        return PD_ESTALE;
    }
    cudaStream_t st = S(stream);
    int nblk = force_blocks(h->n_real);
    PD_TRY(h->red.ensure(sizeof(double) * 2 * nblk));
    if (h->n_real > 0) PD_TRY(lj_launch(h, vl, cl, *lj, force_prop, h->red.as<double>(), nblk, st));
    if (energy) {
        std::vector<double> part(2 * nblk, 0.0);
        if (h->n_real > 0)
            PD_CUDA(cudaMemcpyAsync(part.data(), h->red.p, sizeof(double) * 2 * nblk, cudaMemcpyDeviceToHost, st));
        PD_CUDA(cudaStreamSynchronize(st));
        energy[0] = energy[1] = 0;
        for (int b = 0; b < nblk; ++b) {
            energy[0] += part[2 * b];
            energy[1] += part[2 * b + 1];
        }
    }
    return PD_OK;
}

int pd_md_create(pd_vd h, const pd_lj_params_t* lj, const pd_md_params_t* mp, pd_md* out) {
    if (!h || !lj || !mp || !out) return PD_EINVAL;
    int np = (int)h->props.size();
    if (mp->vel_prop < 0 || mp->vel_prop >= np || mp->force_prop < 0 || mp->force_prop >= np ||
        mp->vel_prop == mp->force_prop) {
        set_error("pd_md_create: bad property ids");
        return PD_EINVAL;
    }
    if (mp->precision != PD_PREC_FP64 && mp->precision != PD_PREC_MIXED) return PD_EINVAL;
    int want = mp->precision == PD_PREC_MIXED ? PD_F32 : h->dtype;
    if (h->props[mp->vel_prop].type != want || h->props[mp->vel_prop].ncomp != 3 ||
        h->props[mp->force_prop].type != want || h->props[mp->force_prop].ncomp != 3) {
        set_error("pd_md_create: velocity and force must be 3-component properties of the vector's dtype "
                  "(PD_F32 in the mixed form)");
        return PD_EINVAL;
    }
    if (mp->precision == PD_PREC_MIXED && (h->dtype != PD_F64 || mp->use_cell_list)) {
        set_error("pd_md_create: the mixed form needs a PD_F64 vector and the Verlet list");
        return PD_EINVAL;
    }
    if (!(mp->dt > 0) || !(mp->mass > 0) || !(lj->r_cut > 0) || !(lj->sigma > 0)) return PD_EINVAL;
    double rlist = lj->r_cut + (mp->skin > 0 ? mp->skin : 0);
    for (int d = 0; d < 3; ++d)
        if (h->bc[d] == PD_PERIODIC && h->g[d] < rlist) {
            set_error("pd_md_create: ghost %.6g in dimension %d is smaller than r_cut + skin %.6g", h->g[d], d, rlist);
            return PD_EINVAL;
        }
    pd_md md = new pd_md_s();
    md->h = h;
    md->lj = *lj;
    md->mp = *mp;
    md->mixed = mp->precision == PD_PREC_MIXED;
    int r;
    if (mp->use_cell_list) {
        r = pd_celllist_create(h, lj->r_cut, PD_CL_NON_SYMMETRIC, 1, (double)1.013f, &md->cl);
    } else {
        r = pd_verlet_create(h, rlist, &md->vl);
    }
    if (r != PD_OK) {
        delete md;
        return r;
    }
    if (md->mixed) mixed_set_quantum(md->vl->cl, mp->skin);
    md->nblk = force_blocks(h->n_real);
    if ((r = md->fpart.ensure(sizeof(double) * 2 * md->nblk)) != PD_OK ||
        (r = md->kpart.ensure(sizeof(double) * md->nblk)) != PD_OK ||
        (r = md->xb.ensure((size_t)(h->n_real > 0 ? h->n_real : 1) * h->pos_bytes)) != PD_OK) {
        pd_md_destroy(md);
        return r;
    }
    *out = md;
    return PD_OK;
}

int pd_sph_create(pd_vd h, const pd_sph_params_t* sp, const pd_md_params_t* mp, pd_md* out) {
    if (!h || !sp || !mp || !out) return PD_EINVAL;
    int np = (int)h->props.size();
    auto okp = [&](int p, int type, int nc) {
        return p >= 0 && p < np && h->props[p].type == type && h->props[p].ncomp == nc;
    };
    int D = h->dtype;
    if (!okp(mp->vel_prop, D, 3) || !okp(mp->force_prop, D, 3) || !okp(sp->rho_prop, D, 1) ||
        !okp(sp->drho_prop, D, 1) || !okp(sp->type_prop, PD_I32, 1)) {
        set_error("pd_sph_create: velocity/acceleration (3 comps), density and its rate (1 comp) in the vector's "
                  "dtype, type as PD_I32");
        return PD_EINVAL;
    }
    for (int d = 0; d < 3; ++d)
        if (h->bc[d] == PD_PERIODIC) {
            set_error("pd_sph_create: the SPH driver supports non-periodic boxes (walls) only");
            return PD_EINVAL;
        }
    if (!(mp->dt > 0) || !(sp->h > 0) || !(sp->mass > 0) || !(sp->rho0 > 0) || mp->use_cell_list ||
        mp->precision != PD_PREC_FP64)
        return PD_EINVAL;
    pd_md md = new pd_md_s();
    md->h = h;
    md->mp = *mp;
    md->sp = *sp;
    md->physics = 1;
    md->tile_p = 4;  // narrow SPH tiles: four lanes per particle keep the CTA busy
    md->lj.eps = md->lj.sigma = 1.0;
    md->lj.r_cut = 2.0 * sp->h;
    double rlist = 2.0 * sp->h + (mp->skin > 0 ? mp->skin : 0);
    int r = pd_verlet_create(h, rlist, &md->vl);
    if (r != PD_OK) {
        delete md;
        return r;
    }
    md->nblk = force_blocks(h->n_real);
    if ((r = md->fpart.ensure(sizeof(double) * 2 * md->nblk)) != PD_OK ||
        (r = md->kpart.ensure(sizeof(double) * md->nblk)) != PD_OK ||
        (r = md->rpart.ensure(sizeof(double) * 2 * md->nblk)) != PD_OK ||
        (r = md->xb.ensure((size_t)(h->n_real > 0 ? h->n_real : 1) * h->pos_bytes)) != PD_OK) {
        pd_md_destroy(md);
        return r;
    }
    *out = md;
    return PD_OK;
}

int pd_md_destroy(pd_md md) {
    if (!md) return PD_EINVAL;
    if (md->swap_reorder && md->h) {
        // the reorder's spare storage lives with the vector; without a driver it has no use
        pd_vd h = md->h;
        free_storage(h->spare_pos, h->spare_gid, h->spare_props);
        h->spare_pos = nullptr;
        h->spare_gid = nullptr;
        h->spare_props.clear();
        h->spare_cap = 0;
    }
    if (md->vl) pd_verlet_destroy(md->vl);
    if (md->cl) pd_celllist_destroy(md->cl);
    md->xb.release();
    md->fpart.release();
    md->kpart.release();
    md->E.release();
    md->csR.release();
    md->csI.release();
    md->tnbr.release();
    md->tnn.release();
    md->tpart.release();
    md->pos32.release();
    md->sxy.release();
    md->sz.release();
    md->sxy2.release();
    md->sz2.release();
    md->off.release();
    md->offb.release();
    md->offK.release();
    md->aux.release();
    md->rpart.release();
    md->eidx.release();
    if (md->gcl) cudaGraphExecDestroy(md->gcl);
    if (md->gst) cudaStreamDestroy(md->gst);
    for (cudaEvent_t e : md->evp) cudaEventDestroy(e);
    delete md;
    return PD_OK;
}

// energies of step s of the plain LJ path (kinetic partials in kpart, pair partials
// of that step's force launch, the rebuild flag in the control block)
static int md_energy(pd_md md, int s, cudaStream_t st) {
    pd_vd h = md->h;
    if (md->physics == 1) {
        // WCSPH: kinetic energy of the fluid, sum of densities
        pd::launch(k_energy, 1, 256, 0, st, (const double*)md->rpart.as<double>(), md->nblk,
                   (const double*)md->kpart.as<double>(), md->nblk, (const unsigned int*)&h->ctrl->rebuild,
                   md->E.as<double>() + 4 * s);
    } else if (md->tiles_active) {
        const int nb2 = 256;
        long chunk = (md->ntiles + nb2 - 1) / nb2;
        double* stage = md->tpart.as<double>() + 2 * md->ntiles;
        pd::launch(k_sum_pairs, nb2, 256, 0, st, (const double*)md->tpart.as<double>(), md->ntiles, chunk, stage);
        pd::launch(k_energy, 1, 256, 0, st, (const double*)stage, nb2, (const double*)md->kpart.as<double>(),
                   md->nblk, (const unsigned int*)&h->ctrl->rebuild, md->E.as<double>() + 4 * s);
    } else {
        pd::launch(k_energy, 1, 256, 0, st, (const double*)md->fpart.as<double>(), md->nblk,
                   (const double*)md->kpart.as<double>(), md->nblk, (const unsigned int*)&h->ctrl->rebuild,
                   md->E.as<double>() + 4 * s);
    }
    PD_LAUNCH_CHECK();
    return PD_OK;
}

// energies of step s from the per-tile (pe, vir, ke) triples of a pair kernel that drifted
static int md_energy_drift(pd_md md, int s, cudaStream_t st) {
    const int nb2 = 256;
    long chunk = (md->ntiles + nb2 - 1) / nb2;
    double* stage = md->tpart.as<double>() + 3 * md->ntiles;
    pd::launch(k_sum_triples, nb2, 256, 0, st, (const double*)md->tpart.as<double>(), md->ntiles, chunk, stage);
    pd::launch(k_energy3, 1, 256, 0, st, (const double*)stage, nb2, (const unsigned int*)&md->h->ctrl->rebuild,
               md->E.as<double>() + 4 * s);
    PD_LAUNCH_CHECK();
    return PD_OK;
}

// Fold the per-phase times of the last timed run into the totals (its events are
// complete: the run synchronised before it returned).
static void md_fold_timing(pd_md md) {
    const size_t steps = md->ev_rebuilt.size();
    for (size_t s = 0; s < steps; ++s) {
        float t[5];
        for (int k = 0; k < 5; ++k) cudaEventElapsedTime(&t[k], md->evp[6 * s + k], md->evp[6 * s + k + 1]);
        md->ms[0] += t[0] + t[4];  // (fused) kick-drift and the previous step's energies; closing kick
        md->cnt[0] += 1;
        md->ms[md->ev_rebuilt[s] ? 1 : 2] += t[2];
        md->cnt[md->ev_rebuilt[s] ? 1 : 2] += 1;
        md->ms[3] += t[3];
        md->cnt[3] += 1;
    }
    md->ev_rebuilt.clear();
}

int pd_md_run(pd_md md, int steps, void* stream, double* E) {
    if (!md || steps < 0) return PD_EINVAL;
    if (md_cluster_eligible(md)) return md_run_cluster(md, steps, S(stream), E);
    if (md->mp.use_cell_list && md->physics == 0 && !md->mixed && !md->timing)
        return md_run_cl_graph(md, steps, S(stream), E);
    pd_vd h = md->h;
    cudaStream_t st = S(stream);
    long n = h->n_real;
    PD_TRY(md->E.ensure(sizeof(double) * 4 * (steps + 1)));
    Prop& V = h->props[md->mp.vel_prop];
    Prop& F = h->props[md->mp.force_prop];
    if (!md->ready) {
        PD_TRY(md_rebuild(md, st));
        PD_TRY(md_forces(md, st));
        md->ready = true;
    }
    double half = 0.5 * md->mp.dt / md->mp.mass;
    double lim = 0.5 * md->mp.skin;
    double lim2 = lim * lim;
    // a step's closing half kick is fused with the next step's kick-drift
    // (k_kick_kick_drift, k_sph_kick_kick_drift); the step's energies follow it, the
    // last step's closing kick runs after the loop
    const bool fused = md->physics == 0 || md->physics == 1;
    // timing: six events per step, read after the run (no synchronisation in the loop)
    if (md->timing)
        while (md->evp.size() < (size_t)6 * steps) {
            cudaEvent_t e;
            PD_CUDA(cudaEventCreate(&e));
            md->evp.push_back(e);
        }
    md_fold_timing(md);  // the previous run's events are recorded again below
    std::vector<unsigned char> rebuilt_at(md->timing ? steps : 0, 0);
#define PD_EV(k) \
    if (md->timing) PD_CUDA(cudaEventRecord(md->evp[6 * (size_t)s + (k)], st))
    for (int s = 0; s < steps; ++s) {
        unsigned int rebuilt = 0;
        const bool split = md_split(md);  // the drift also refreshes the pair kernel's staging copies
        PD_EV(0);
        if (md->drifted) {
            // the previous step's pair kernel made this step's kick and drift (and the
            // previous step's closing kick and energies)
            md->drifted = false;
        } else {
            PD_CUDA(cudaMemsetAsync(&h->ctrl->maxdisp2, 0, sizeof(unsigned long long), st));
            if (fused && s > 0 && md->physics == 1) {
                PD_TRY(sph_kick_kick_drift(h, md->sp, md->mp.vel_prop, md->mp.force_prop, md->xb, md->aux, md->nblk,
                                           md->mp.dt, md->kpart.as<double>(), md->rpart.as<double>(), st));
                PD_TRY(md_energy(md, s - 1, st));
            } else if (fused && s > 0 && md->mixed) {
                PD_TRY(mixed_kick_kick_drift(h, md->vl->cl, md->off, md->offb, md->mp.vel_prop, md->mp.force_prop, md->nblk, half,
                                             md->mp.dt, md->mp.mass, md->kpart.as<double>(), st));
                PD_TRY(md_energy(md, s - 1, st));
            } else if (fused && s > 0) {
                if (h->dtype == PD_F64)
                    pd::launch(k_kick_kick_drift<double>, md->nblk, FBLOCK, 0, st, (double4*)h->pos,
                               (const double4*)md->xb.as<double4>(), (double*)V.d, (const double*)F.d, h->cap, n, half,
                               md->mp.dt, md->mp.mass, &h->ctrl->maxdisp2, md->kpart.as<double>(), split ? md->sxy.as<double>() : nullptr,
                               split ? md->sz.as<double>() : nullptr);
                else
                    pd::launch(k_kick_kick_drift<float>, md->nblk, FBLOCK, 0, st, (float4*)h->pos,
                               (const float4*)md->xb.as<float4>(), (float*)V.d, (const float*)F.d, h->cap, n, (float)half,
                               (float)md->mp.dt, md->mp.mass, &h->ctrl->maxdisp2, md->kpart.as<double>(), (float*)nullptr,
                               (float*)nullptr);
                PD_LAUNCH_CHECK();
                PD_TRY(md_energy(md, s - 1, st));
            } else if (md->physics == 1)
                PD_TRY(sph_kick_drift(h, md->sp, md->mp.vel_prop, md->mp.force_prop, md->xb, md->aux, md->nblk,
                                      md->mp.dt, st));
            else if (md->mixed)
                PD_TRY(mixed_kick_drift(h, md->vl->cl, md->off, md->offb, md->mp.vel_prop, md->mp.force_prop, md->nblk, half,
                                        md->mp.dt, st));
            else if (h->dtype == PD_F64)
                pd::launch(k_kick_drift<double>, md->nblk, FBLOCK, 0, st, (double4*)h->pos, md->xb.as<double4>(), (double*)V.d,
                                                                  (const double*)F.d, h->cap, n, half, md->mp.dt,
                                                                  &h->ctrl->maxdisp2, split ? md->sxy.as<double>() : nullptr,
                                                                  split ? md->sz.as<double>() : nullptr);
            else
                pd::launch(k_kick_drift<float>, md->nblk, FBLOCK, 0, st, (float4*)h->pos, md->xb.as<float4>(), (float*)V.d,
                                                                 (const float*)F.d, h->cap, n, (float)half,
                                                                 (float)md->mp.dt, &h->ctrl->maxdisp2, (float*)nullptr,
                                                                 (float*)nullptr);
            PD_LAUNCH_CHECK();
        }
        PD_EV(1);
        bool rb = md->mp.skin <= 0 || md->mp.use_cell_list;
        if (!rb) {
            PD_CUDA(cudaMemcpyAsync(&h->ctrl_h->maxdisp2, &h->ctrl->maxdisp2, sizeof(unsigned long long),
                                    cudaMemcpyDeviceToHost, st));
            PD_CUDA(cudaStreamSynchronize(st));
            double d2;
            memcpy(&d2, &h->ctrl_h->maxdisp2, sizeof(double));
            rb = d2 > lim2;
        }
        PD_EV(2);
        if (rb) {
            PD_TRY(md_rebuild(md, st));
            rebuilt = 1;
        } else if (md->mixed) {
            PD_TRY(mixed_replay(h, md->off, md->offK, st));
        } else {
            PD_TRY(ghost_replay(h, 0ul, true, nullptr, h->n_img, st));
            if (split) PD_TRY(tile_split(h, md->sxy, md->sz, h->n_real, h->n_img, st));
        }
        PD_EV(3);
        // plain FP64 tiled steps with a next step in this run: the pair kernel also
        // makes this step's closing kick and the next step's kick and drift, into the
        // second pair of staging copies, which then become the current ones
        const bool drift = fused && !md->mixed && md_split(md) && s + 1 < steps;
        if (drift) {
            const size_t cap = (size_t)(h->cap > 0 ? h->cap : 1);
            PD_TRY(md->sxy2.ensure(cap * sizeof(double2)));
            PD_TRY(md->sz2.ensure(cap * sizeof(double)));
            PD_CUDA(cudaMemsetAsync(&h->ctrl->maxdisp2, 0, sizeof(unsigned long long), st));
            DriftArgs D{(double4*)h->pos, md->xb.as<const double4>(), (double*)V.d, h->cap, half, md->mp.dt,
                        md->mp.mass, md->sxy2.as<double2>(), md->sz2.as<double>(), &h->ctrl->maxdisp2};
            PD_TRY(md_forces(md, st, &D));
            std::swap(md->sxy, md->sxy2);
            std::swap(md->sz, md->sz2);
            md->drifted = true;
        } else {
            PD_TRY(md_forces(md, st));
        }
        PD_EV(4);
        if (md->timing) rebuilt_at[s] = (unsigned char)rebuilt;
        if (fused) {
            // the rebuild flag of this step, read by its energies
            h->ctrl_h->rebuild = rebuilt;
            PD_CUDA(cudaMemcpyAsync(&h->ctrl->rebuild, &h->ctrl_h->rebuild, sizeof(unsigned int),
                                    cudaMemcpyHostToDevice, st));
            if (drift) PD_TRY(md_energy_drift(md, s, st));
            md->steps++;
            PD_EV(5);
            continue;
        }
        if (md->physics == 1)
            PD_TRY(sph_kick(h, md->sp, md->mp.vel_prop, md->mp.force_prop, md->nblk, md->mp.dt,
                            md->kpart.as<double>(), md->rpart.as<double>(), st));
        else if (md->mixed)
            PD_TRY(mixed_kick(h, md->mp.vel_prop, md->mp.force_prop, md->nblk, half, md->mp.mass,
                              md->kpart.as<double>(), st));
        else if (h->dtype == PD_F64)
            pd::launch(k_kick<double>, md->nblk, FBLOCK, 0, st, (double*)V.d, (const double*)F.d, h->cap, n, half,
                                                        md->mp.mass, md->kpart.as<double>());
        else
            pd::launch(k_kick<float>, md->nblk, FBLOCK, 0, st, (float*)V.d, (const float*)F.d, h->cap, n, (float)half,
                                                       md->mp.mass, md->kpart.as<double>());
        PD_LAUNCH_CHECK();
        h->ctrl_h->rebuild = rebuilt;
        PD_CUDA(cudaMemcpyAsync(&h->ctrl->rebuild, &h->ctrl_h->rebuild, sizeof(unsigned int), cudaMemcpyHostToDevice, st));
        if (md->physics == 1) {
            pd::launch(k_energy, 1, 256, 0, st, (const double*)md->rpart.as<double>(), md->nblk,
                       (const double*)md->kpart.as<double>(), md->nblk, (const unsigned int*)&h->ctrl->rebuild,
                       md->E.as<double>() + 4 * s);
        } else if (md->tiles_active) {
            const int nb2 = 256;
            long chunk = (md->ntiles + nb2 - 1) / nb2;
            double* stage = md->tpart.as<double>() + 2 * md->ntiles;
            pd::launch(k_sum_pairs, nb2, 256, 0, st, (const double*)md->tpart.as<double>(), md->ntiles, chunk, stage);
            pd::launch(k_energy, 1, 256, 0, st, (const double*)stage, nb2, (const double*)md->kpart.as<double>(),
                       md->nblk, (const unsigned int*)&h->ctrl->rebuild, md->E.as<double>() + 4 * s);
        }
        else
            pd::launch(k_energy, 1, 256, 0, st, (const double*)md->fpart.as<double>(), md->nblk,
                       (const double*)md->kpart.as<double>(), md->nblk, (const unsigned int*)&h->ctrl->rebuild,
                       md->E.as<double>() + 4 * s);
        PD_LAUNCH_CHECK();
        md->steps++;
        PD_EV(5);
    }
#undef PD_EV
    if (fused && steps > 0 && md->physics == 1) {
        PD_TRY(sph_kick(h, md->sp, md->mp.vel_prop, md->mp.force_prop, md->nblk, md->mp.dt, md->kpart.as<double>(),
                        md->rpart.as<double>(), st));
        PD_TRY(md_energy(md, steps - 1, st));
    } else if (fused && steps > 0 && md->mixed) {
        PD_TRY(mixed_kick(h, md->mp.vel_prop, md->mp.force_prop, md->nblk, half, md->mp.mass, md->kpart.as<double>(),
                          st));
        PD_TRY(md_energy(md, steps - 1, st));
    } else if (fused && steps > 0) {
        // the last step's closing half kick and energies
        if (h->dtype == PD_F64)
            pd::launch(k_kick<double>, md->nblk, FBLOCK, 0, st, (double*)V.d, (const double*)F.d, h->cap, n, half,
                       md->mp.mass, md->kpart.as<double>());
        else
            pd::launch(k_kick<float>, md->nblk, FBLOCK, 0, st, (float*)V.d, (const float*)F.d, h->cap, n, (float)half,
                       md->mp.mass, md->kpart.as<double>());
        PD_LAUNCH_CHECK();
        PD_TRY(md_energy(md, steps - 1, st));
    }
    if (md->mixed) PD_TRY(mixed_to_positions(h, md->vl->cl, md->off, st));  // the vector's positions are current
    if (E && steps > 0) {
        PD_CUDA(cudaMemcpyAsync(E, md->E.p, sizeof(double) * 4 * steps, cudaMemcpyDeviceToHost, st));
    }
    // the energies and the error word in one synchronisation
    PD_TRY(read_ctrl(h, st));
    if (md->timing) md->ev_rebuilt = std::move(rebuilt_at);  // read by pd_md_timers or the next run
    if (h->ctrl_h->err & (ERR_IMG_OVERFLOW | ERR_NN_OVERFLOW)) {
        set_error("pd_md_run: device capacity overflow (err=0x%x)", h->ctrl_h->err);
        return PD_EOVERFLOW;
    }
    return PD_OK;
}

int pd_md_set_timing(pd_md md, int on) {
    if (!md) return PD_EINVAL;
    md->timing = on != 0;
    md->ev_rebuilt.clear();
    for (int i = 0; i < 4; ++i) {
        md->ms[i] = 0;
        md->cnt[i] = 0;
    }
    return PD_OK;
}

int pd_md_launch_shape(pd_md md, int* cluster_ctas, int* tile_tx, int* threads_per_particle) {
    if (!md || !cluster_ctas || !tile_tx || !threads_per_particle) return PD_EINVAL;
    *cluster_ctas = md->cluster_ctas;
    *tile_tx = md->tiles_active ? md->tg.TX : 0;
    *threads_per_particle = md->tiles_active ? md->tile_p : 0;
    return PD_OK;
}

int pd_md_timers(pd_md md, double* ms, long* counts) {
    if (!md || !ms || !counts) return PD_EINVAL;
    md_fold_timing(md);
    for (int i = 0; i < 4; ++i) {
        ms[i] = md->ms[i];
        counts[i] = md->cnt[i];
    }
    return PD_OK;
}

int pd_md_set_tiles(pd_md md, int on, int tx, int threads_per_particle) {
    if (!md || tx < 0 || tx > TXMAX) return PD_EINVAL;
    int p = threads_per_particle <= 0 ? 2 : threads_per_particle;
    if (p != 1 && p != 2 && p != 4) return PD_EINVAL;
    md->use_tiles = on != 0;
    md->tile_tx = tx;
    md->tile_p = p;
    md->ready = false;  // rebuild with the new structure at the next run
    return PD_OK;
}

int pd_md_set_block(pd_md md, int threads) {
    if (!md || (threads != FBLOCK_T && threads != FBLOCK_T / 2)) return PD_EINVAL;
    md->tile_block = threads;
    return PD_OK;
}

int pd_md_verlet_get(pd_md md, int* counts, int* idx, long idx_cap, int* tiled) {
    if (!md || !counts) return PD_EINVAL;
    if (tiled) *tiled = md->tiles_active ? 1 : 0;
    if (!md->tiles_active) {
        if (!md->vl) return PD_ESTATE;
        return pd_verlet_get(md->vl, counts, idx, idx_cap, nullptr);
    }
    pd_vd h = md->h;
    long n = h->n_real;
    if (n == 0) return PD_OK;
    PD_CUDA(cudaMemcpy(counts, md->tnn.p, sizeof(int) * n, cudaMemcpyDeviceToHost));
    if (!idx) return PD_OK;
    long tot = 0;
    int mx = 0;
    for (long i = 0; i < n; ++i) {
        tot += counts[i];
        mx = std::max(mx, counts[i]);
    }
    if (tot > idx_cap) return PD_EINVAL;
    Buf out;
    PD_TRY(out.ensure(sizeof(int) * (size_t)md->tstride * (mx > 0 ? mx : 1)));
    PD_TRY(tile_translate(h, md->tg, md->ntiles, md->csR.as<unsigned int>(), md->csI.as<unsigned int>(), md->tnbr,
                          md->tnn, md->tstride, mx, out.as<int>(), 0));
    std::vector<int> col((size_t)md->tstride * mx);
    if (mx > 0) PD_CUDA(cudaMemcpy(col.data(), out.p, sizeof(int) * col.size(), cudaMemcpyDeviceToHost));
    out.release();
    long o = 0;
    for (long i = 0; i < n; ++i)
        for (int k = 0; k < counts[i]; ++k) idx[o++] = col[(size_t)k * md->tstride + i];
    return PD_OK;
}

int pd_md_list_stats(pd_md md, long* n_dom, double* mean_nn, int* max_nn) {
    if (!md || !n_dom || !mean_nn || !max_nn) return PD_EINVAL;
    *n_dom = 0;
    *mean_nn = 0;
    *max_nn = 0;
    if (!md->vl) return PD_OK;
    long nd = md->tiles_active ? md->h->n_real : md->vl->n_dom;
    if (nd == 0) return PD_OK;
    std::vector<int> c(nd);
    PD_CUDA(cudaMemcpy(c.data(), md->tiles_active ? md->tnn.p : md->vl->nn.p, sizeof(int) * c.size(),
                       cudaMemcpyDeviceToHost));
    double s = 0;
    int m = 0;
    for (int x : c) {
        s += x;
        m = std::max(m, x);
    }
    *n_dom = (long)c.size();
    *mean_nn = s / (double)c.size();
    *max_nn = m;
    return PD_OK;
}

int pd_md_stats(pd_md md, long* builds, long* steps, int* err) {
    if (!md) return PD_EINVAL;
    if (builds) *builds = md->builds;
    if (steps) *steps = md->steps;
    if (err) {
        PD_TRY(read_ctrl(md->h, 0));
        *err = (int)md->h->ctrl_h->err;
    }
    return PD_OK;
}

}  // extern "C"
