// pd_mixed.cu -- precision form of the LJ integrator: FP32 cell-local positions,
// FP32 pair math with compensated (Kahan) sums, FP64 only for the periodic wrap
// at rebuilds and for the global energy / virial reductions.
//
// State between rebuilds (all particles, images included, in the tiled order):
//   off[k] = (x - c, y - c, z - c, cell id) : FP32 offset from the centre of the
//            particle's cell at the last rebuild (cell grid of side r_cut+skin);
//   v, f   : FP32 properties of the vector.
// A pair displacement is formed from the offsets and the cell difference
// (dx = (o_i - o_j) + (c_i - c_j) * s), so its rounding error is set by the
// offset magnitude (<= 1.5 s), not by the box size.  Offsets are kept on a grid
// of quantum q = 2^e with every value of the pair loop below 2^24 q
// (mixed_set_quantum): differences and cell shifts of grid values are then exact in
// FP32, so a pair displacement equals the FP64 displacement of the represented
// positions exactly, and r2 carries only its own roundings.  The cutoff is
// decided in FP64 for the few pairs within that rounding of it (in_cut_exact).
// Centres use the cell side rounded to the grid; an image offset is its source's
// offset plus a constant of the rebuild, exact when the box length is a multiple
// of q (else rounded to the grid once).  In a tile, staged records
// are rewritten once in shared memory: y and z are shifted by the row's cell
// difference to the tile's centre row (|.| <= 2.5 s) and w holds the record's
// cell column in the tile, so the pair loop forms
//   dx = fma(col_i - col_j, s_x, x_i - x_j), dy = y_i - y_j, dz = z_i - z_j.
// Per-particle force, energy and virial sums are accumulated in FP32 over the
// two entries of a row word and added to a Kahan-compensated FP32 accumulator
// (Kahan 1965); lanes sharing a particle combine in FP64; block energies in FP64.
#include "pd_device.cuh"
#include "pd_internal.cuh"
#include "pd_lj.cuh"
#include "pd_mixed.cuh"
#include "pd_mixed_dev.cuh"
#include "pd_tile.cuh"

#include <algorithm>
#include <cmath>

namespace pd {

// positions -> offsets from the cell centre (all n particles)
__global__ void k_x64_to_off(const double4* __restrict__ pos, long n, Grid<double> G, CellGeom C,
                             float4* __restrict__ off, unsigned int* __restrict__ err) {
    unsigned int bad = 0;
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        double4 r = ld4(pos, k);
        unsigned int c = (unsigned int)G.cell(r.x, r.y, r.z, bad);
        double cx, cy, cz;
        C.centre(c, cx, cy, cz);
        off[k] = make_float4(C.qd(r.x - cx), C.qd(r.y - cy), C.qd(r.z - cz), __uint_as_float(c));
    }
    if (bad) atomicOr(err, ERR_CELL_RANGE);
}

// offsets -> positions (real particles)
__global__ void k_off_to_x64(const float4* __restrict__ off, long n, CellGeom C, double4* __restrict__ pos) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        float4 o = off[k];
        double cx, cy, cz;
        C.centre(__float_as_uint(o.w), cx, cy, cz);
        st4(pos, k, make_double4(cx + (double)o.x, cy + (double)o.y, cz + (double)o.z, 0.0));
    }
}

// offsets -> positions written in id order as x,y,z triples (a finished
// system's result, ready for one contiguous copy to the host)
__global__ void k_off_to_x64_by_id(const float4* __restrict__ off, long n, CellGeom C, const int* __restrict__ gid,
                                   double* __restrict__ out) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        float4 o = off[k];
        double cx, cy, cz;
        C.centre(__float_as_uint(o.w), cx, cy, cz);
        const long g = gid[k];
        if (g < 0 || g >= n) continue;
        out[3 * g] = cx + (double)o.x;
        out[3 * g + 1] = cy + (double)o.y;
        out[3 * g + 2] = cz + (double)o.z;
    }
}

// image offset = source offset + K, K formed in FP64 at the rebuild
__global__ void k_image_k(const double4* __restrict__ pos, const float4* __restrict__ off, long n_real, long m,
                          const int* __restrict__ src, CellGeom C, float4* __restrict__ K) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < m; k += (long)gridDim.x * blockDim.x) {
        int s = src[k];
        double4 xi = ld4(pos, n_real + k), xs = ld4(pos, s);
        double ci[3], cs[3];
        C.centre(__float_as_uint(off[n_real + k].w), ci[0], ci[1], ci[2]);
        C.centre(__float_as_uint(off[s].w), cs[0], cs[1], cs[2]);
        K[k] = make_float4(C.qd((xi.x - ci[0]) - (xs.x - cs[0])), C.qd((xi.y - ci[1]) - (xs.y - cs[1])),
                           C.qd((xi.z - ci[2]) - (xs.z - cs[2])), 0.f);
    }
}

__global__ void k_replay32(float4* __restrict__ off, long n_real, long m, const int* __restrict__ src,
                           const float4* __restrict__ K) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < m; k += (long)gridDim.x * blockDim.x) {
        float4 o = off[src[k]], q = K[k];
        float4 r = off[n_real + k];
        r.x = o.x + q.x;
        r.y = o.y + q.y;
        r.z = o.z + q.z;
        off[n_real + k] = r;
    }
}

// v += h f ; o += dt v ; largest |o - o_build|^2
__global__ void __launch_bounds__(256) k_kick_drift32(float4* __restrict__ off, const float4* __restrict__ ob,
                                                      float* __restrict__ v, const float* __restrict__ f, long cap,
                                                      long n, float half, float dt, CellGeom C,
                                                      unsigned long long* __restrict__ maxd2) {
    double mx = 0;
    for (long i = blockIdx.x * 256L + threadIdx.x; i < n; i += (long)gridDim.x * 256) {
        float4 o = off[i];
        float vx = v[i] + half * f[i];
        float vy = v[cap + i] + half * f[cap + i];
        float vz = v[2 * cap + i] + half * f[2 * cap + i];
        o.x = C.qf(o.x + dt * vx);
        o.y = C.qf(o.y + dt * vy);
        o.z = C.qf(o.z + dt * vz);
        v[i] = vx;
        v[cap + i] = vy;
        v[2 * cap + i] = vz;
        off[i] = o;
        float4 b = ob[i];
        float dx = o.x - b.x, dy = o.y - b.y, dz = o.z - b.z;
        mx = fmax(mx, (double)dist2(dx, dy, dz));
    }
    mx = warp_max(mx);
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(maxd2, mx);
}

// k_kick32 of one step and k_kick_drift32 of the next in one pass (the same
// operations in the same order; kinetic energy partials of the closing kick)
__global__ void __launch_bounds__(256) k_kick_kick_drift32(float4* __restrict__ off, const float4* __restrict__ ob,
                                                           float* __restrict__ v, const float* __restrict__ f,
                                                           long cap, long n, float half, float dt, double mass,
                                                           CellGeom C, unsigned long long* __restrict__ maxd2,
                                                           double* __restrict__ part) {
    double mx = 0, ke = 0;
    for (long i = blockIdx.x * 256L + threadIdx.x; i < n; i += (long)gridDim.x * 256) {
        const float fx = f[i], fy = f[cap + i], fz = f[2 * cap + i];
        float vx = v[i] + half * fx;
        float vy = v[cap + i] + half * fy;
        float vz = v[2 * cap + i] + half * fz;
        ke += 0.5 * mass * ((double)vx * vx + (double)vy * vy + (double)vz * vz);
        vx = vx + half * fx;
        vy = vy + half * fy;
        vz = vz + half * fz;
        float4 o = off[i];
        o.x = C.qf(o.x + dt * vx);
        o.y = C.qf(o.y + dt * vy);
        o.z = C.qf(o.z + dt * vz);
        v[i] = vx;
        v[cap + i] = vy;
        v[2 * cap + i] = vz;
        off[i] = o;
        float4 b = ob[i];
        float dx = o.x - b.x, dy = o.y - b.y, dz = o.z - b.z;
        mx = fmax(mx, (double)dist2(dx, dy, dz));
    }
    mx = warp_max(mx);
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(maxd2, mx);
    ke = block_sum<double, 256>(ke);
    if (threadIdx.x == 0) part[blockIdx.x] = ke;
}

__global__ void __launch_bounds__(256) k_kick32(float* __restrict__ v, const float* __restrict__ f, long cap, long n,
                                                float half, double mass, double* __restrict__ part) {
    double ke = 0;
    for (long i = blockIdx.x * 256L + threadIdx.x; i < n; i += (long)gridDim.x * 256) {
        float vx = v[i] + half * f[i];
        float vy = v[cap + i] + half * f[cap + i];
        float vz = v[2 * cap + i] + half * f[2 * cap + i];
        v[i] = vx;
        v[cap + i] = vy;
        v[2 * cap + i] = vz;
        ke += 0.5 * mass * ((double)vx * vx + (double)vy * vy + (double)vz * vz);
    }
    ke = block_sum<double, 256>(ke);
    if (threadIdx.x == 0) part[blockIdx.x] = ke;
}

template <int P, int BLOCK>
__global__ void __launch_bounds__(BLOCK, 5 * FBLOCK_T / BLOCK) k_vtile_lj_mixed(const float4* __restrict__ off, long n_real,
                                                             TileGeom tg, const unsigned int* __restrict__ csR,
                                                             const unsigned int* __restrict__ csI, unsigned int cap,
                                                             const unsigned int* __restrict__ nbr,
                                                             const int* __restrict__ nn, long stride, float sx,
                                                             float sy, float sz, LJP<float> Pr, float* __restrict__ f,
                                                             long fcap, double* __restrict__ part,
                                                             unsigned int* __restrict__ err) {
    extern __shared__ __align__(128) unsigned char tile_raw[];
    float4* sm = reinterpret_cast<float4*>(tile_raw);
    __shared__ TileShM S;
    __shared__ unsigned long long bar;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    unsigned int uses = 0;
    double pe = 0, vir = 0;
    mixed_tile<P, BLOCK>(blockIdx.x, off, n_real, tg, csR, csI, cap, nbr, nn, stride, sx, sy, sz, Pr, f, fcap, err, sm,
                         S, &bar, uses, pe, vir);
    pe = block_sum<double, BLOCK>(pe);
    vir = block_sum<double, BLOCK>(vir);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = pe;
        part[2 * blockIdx.x + 1] = vir;
    }
}

// ---------------------------------------------------------------------------
double mixed_set_quantum(pd_cl cl, double skin) {
    double s = 0;
    for (int d = 0; d < 3; ++d) s = std::max(s, cl->spacing[d]);
    int e = 0;
    std::frexp(2.0 * s + (skin > 0 ? skin : 0.0), &e);  // 2^e > 2 s + skin
    cl->mq = std::ldexp(1.0, e - 24);
    return cl->mq;
}

CellGeom mixed_cell_geom(pd_cl cl) {
    if (!(cl->mq > 0)) mixed_set_quantum(cl, 0.5 * cl->spacing[0]);  // a skin of half a cell bounds any list
    CellGeom C;
    C.q = cl->mq;
    C.iq = 1.0 / cl->mq;
    for (int d = 0; d < 3; ++d) {
        C.lo[d] = cl->box_lo[d];
        C.sp[d] = std::rint(cl->spacing[d] * C.iq) * C.q;  // the cell side on the grid
        C.gs[d] = cl->gs[d];
    }
    C.pad = cl->pad;
    return C;
}

int mixed_from_positions(pd_vd h, pd_cl cl, Buf& off, Buf& K, cudaStream_t st) {
    long nt = h->n_total, m = h->n_img;
    PD_TRY(off.ensure(sizeof(float4) * (size_t)(h->cap > 0 ? h->cap : 1)));
    PD_TRY(K.ensure(sizeof(float4) * (size_t)(m > 0 ? m : 1)));
    Grid<double> G;
    for (int d = 0; d < 3; ++d) {
        G.lo[d] = cl->box_lo[d];
        G.sp[d] = cl->spacing[d];
        G.gs[d] = cl->gs[d];
    }
    G.pad = cl->pad;
    CellGeom C = mixed_cell_geom(cl);
    if (nt > 0)
        pd::launch(k_x64_to_off, grid_for(nt, 256), 256, 0, st, (const double4*)h->pos, nt, G, C, off.as<float4>(),
                   &h->ctrl->err);
    if (m > 0)
        pd::launch(k_image_k, grid_for(m, 256), 256, 0, st, (const double4*)h->pos, (const float4*)off.as<float4>(),
                   h->n_real, m, (const int*)h->img_src.as<int>(), C, K.as<float4>());
    PD_LAUNCH_CHECK();
    return PD_OK;
}

int mixed_to_positions(pd_vd h, pd_cl cl, const Buf& off, cudaStream_t st) {
    long n = h->n_real;
    if (n > 0)
        pd::launch(k_off_to_x64, grid_for(n, 256), 256, 0, st, (const float4*)off.as<float4>(), n, mixed_cell_geom(cl),
                   (double4*)h->pos);
    PD_LAUNCH_CHECK();
    return PD_OK;
}

int mixed_to_positions_by_id(pd_vd h, pd_cl cl, const Buf& off, double* out, cudaStream_t st) {
    long n = h->n_real;
    if (n > 0)
        pd::launch(k_off_to_x64_by_id, grid_for(n, 256), 256, 0, st, (const float4*)off.as<float4>(), n,
                   mixed_cell_geom(cl), (const int*)h->gid, out);
    PD_LAUNCH_CHECK();
    return PD_OK;
}

int mixed_replay(pd_vd h, Buf& off, const Buf& K, cudaStream_t st) {
    long m = h->n_img;
    if (m > 0)
        pd::launch(k_replay32, grid_for(m, 256), 256, 0, st, off.as<float4>(), h->n_real, m,
                   (const int*)h->img_src.as<int>(), (const float4*)K.as<float4>());
    PD_LAUNCH_CHECK();
    return PD_OK;
}

int mixed_kick_drift(pd_vd h, pd_cl cl, Buf& off, const Buf& ob, int vel_prop, int force_prop, int nblk,
                     double half, double dt, cudaStream_t st) {
    Prop& V = h->props[vel_prop];
    Prop& F = h->props[force_prop];
    pd::launch(k_kick_drift32, nblk, 256, 0, st, off.as<float4>(), (const float4*)ob.as<float4>(), (float*)V.d,
               (const float*)F.d, h->cap, h->n_real, (float)half, (float)dt, mixed_cell_geom(cl), &h->ctrl->maxdisp2);
    PD_LAUNCH_CHECK();
    return PD_OK;
}

int mixed_kick_kick_drift(pd_vd h, pd_cl cl, Buf& off, const Buf& ob, int vel_prop, int force_prop, int nblk,
                          double half, double dt, double mass, double* kpart, cudaStream_t st) {
    Prop& V = h->props[vel_prop];
    Prop& F = h->props[force_prop];
    pd::launch(k_kick_kick_drift32, nblk, 256, 0, st, off.as<float4>(), (const float4*)ob.as<float4>(), (float*)V.d,
               (const float*)F.d, h->cap, h->n_real, (float)half, (float)dt, mass, mixed_cell_geom(cl),
               &h->ctrl->maxdisp2, kpart);
    PD_LAUNCH_CHECK();
    return PD_OK;
}

int mixed_kick(pd_vd h, int vel_prop, int force_prop, int nblk, double half, double mass, double* kpart,
               cudaStream_t st) {
    Prop& V = h->props[vel_prop];
    Prop& F = h->props[force_prop];
    pd::launch(k_kick32, nblk, 256, 0, st, (float*)V.d, (const float*)F.d, h->cap, h->n_real, (float)half, mass,
               kpart);
    PD_LAUNCH_CHECK();
    return PD_OK;
}

template <int P, int BLOCK>
static int launch_mixed(pd_vd h, const TileGeom& tg, long ntiles, const unsigned int* csR, const unsigned int* csI,
                        unsigned int cap, const Buf& off, const Buf& nbr, const Buf& nn, long stride, float sx,
                        float sy, float sz, const LJP<float>& LP, float* f, double* part, cudaStream_t st) {
    int smem = (int)(cap * sizeof(float4));
    if (smem < 16) smem = 16;
    PD_CUDA(cudaFuncSetAttribute(k_vtile_lj_mixed<P, BLOCK>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    pd::launch(k_vtile_lj_mixed<P, BLOCK>, (unsigned)ntiles, BLOCK, (size_t)smem, st, (const float4*)off.as<float4>(),
               h->n_real, tg, csR, csI, cap, (const unsigned int*)nbr.as<unsigned int>(), (const int*)nn.as<int>(),
               stride, sx, sy, sz, LP, f, h->cap, part, &h->ctrl->err);
    PD_LAUNCH_CHECK();
    return PD_OK;
}

void mixed_cutoff(const pd_lj_params_t& lj, LJP<float>& P) {
    const float rc = (float)lj.r_cut;
    P.rc2 = rc * rc;
    P.rc2d = lj.r_cut * lj.r_cut;
    // |r2_f32 - r2| <= 3 u r2 (u = 2^-24) for exact dx, dy, dz: a band of 16 u r2 on each side
    P.rc2lo = (float)(P.rc2d * (1.0 - std::ldexp(1.0, -20)));
    P.rc2hi = (float)(P.rc2d * (1.0 + std::ldexp(1.0, -20)));
    P.rclose2 = (float)(0.95 * 0.95 * lj.sigma * lj.sigma);
    P.eps24d = 24.0 * lj.eps;
    P.eps4d = 4.0 * lj.eps;
    P.sig2d = lj.sigma * lj.sigma;
}

int mixed_lj(pd_vd h, pd_cl cl, const TileGeom& tg, long ntiles, const unsigned int* csR, const unsigned int* csI,
             unsigned int cap, const Buf& off, const Buf& nbr, const Buf& nn, long stride, const pd_lj_params_t& lj,
             int force_prop, double* part, int P, int block, cudaStream_t st) {
    LJP<float> LP{};
    LP.eps24 = (float)(24.0 * lj.eps);
    LP.eps4 = (float)(4.0 * lj.eps);
    LP.sig2 = (float)(lj.sigma * lj.sigma);
    mixed_cutoff(lj, LP);
    float* f = (float*)h->props[force_prop].d;
    const CellGeom C = mixed_cell_geom(cl);
    const float sx = (float)C.sp[0], sy = (float)C.sp[1], sz = (float)C.sp[2];  // exact: multiples of q
#define PD_MIXED_CASE(PP, BB)                                                                                   \
    if (P == PP && block == BB)                                                                                 \
        return launch_mixed<PP, BB>(h, tg, ntiles, csR, csI, cap, off, nbr, nn, stride, sx, sy, sz, LP, f, part, st);
    PD_MIXED_CASE(1, FBLOCK_T)
    PD_MIXED_CASE(2, FBLOCK_T)
    PD_MIXED_CASE(4, FBLOCK_T)
    PD_MIXED_CASE(1, FBLOCK_T / 2)
    PD_MIXED_CASE(2, FBLOCK_T / 2)
    PD_MIXED_CASE(4, FBLOCK_T / 2)
#undef PD_MIXED_CASE
    set_error("precision form: lanes per particle 1, 2 or 4 and CTAs of %d or %d threads", FBLOCK_T, FBLOCK_T / 2);
    return PD_EINVAL;
}

}  // namespace pd
