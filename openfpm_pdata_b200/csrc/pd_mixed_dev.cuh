// pd_mixed_dev.cuh -- device code of the mixed-form LJ tile kernel, shared by the
// single-system kernel (pd_mixed.cu) and the batched kernels (pd_serve.cu).
#pragma once
#include "pd_device.cuh"
#include "pd_internal.cuh"
#include "pd_lj.cuh"
#include "pd_tile.cuh"
#include "pd_tile_dev.cuh"

namespace pd {

struct TileShM {
    unsigned int cR[9][TXMAX + 3];
    unsigned int cI[9][TXMAX + 3];
    unsigned int oR[9], oI[9];
    unsigned int total;
    int ncol;
    unsigned int segb[18][TXMAX + 3];
};

// Cell centres of the precision form and the quantum of its offsets.  Centres are
// lo + (i - pad + 1/2) * sp with sp the cell side rounded to a multiple of the
// quantum q (a power of two, mixed_set_quantum in pd_mixed.cu); every offset is a
// multiple of q below 2^24 q in magnitude, so the FP32 differences and the cell
// shifts of the pair loop are exact (FP32 holds every multiple of q in that range).
struct CellGeom {
    double lo[3], sp[3];
    int gs[3], pad;
    double q, iq;  // quantum and its reciprocal (powers of two)
    // an FP64 offset rounded to the nearest multiple of q (exact in FP32)
    __device__ __forceinline__ float qd(double o) const { return (float)(rint(o * iq) * q); }
    // an FP32 value rounded to the nearest multiple of q (scalings by powers of two are exact)
    __device__ __forceinline__ float qf(float o) const { return rintf(o * (float)iq) * (float)q; }
    __device__ __forceinline__ void centre(unsigned int c, double& cx, double& cy, double& cz) const {
        int i0 = (int)(c % (unsigned)gs[0]);
        int i1 = (int)((c / (unsigned)gs[0]) % (unsigned)gs[1]);
        int i2 = (int)(c / ((unsigned)gs[0] * (unsigned)gs[1]));
        cx = lo[0] + ((double)(i0 - pad) + 0.5) * sp[0];
        cy = lo[1] + ((double)(i1 - pad) + 0.5) * sp[1];
        cz = lo[2] + ((double)(i2 - pad) + 0.5) * sp[2];
    }
};

// host: the centres and quantum of the precision form on the grid of `cl`
CellGeom mixed_cell_geom(pd_cl cl);
// host: the cutoff of the precision form (FP32 threshold and FP64 re-decision band)
void mixed_cutoff(const pd_lj_params_t& lj, LJP<float>& P);

// Pairs closer than Pr.rclose2 (0.95 sigma: the repulsive wall, where a relative
// rounding error of r2 grows about sevenfold in the force) are evaluated in FP64
// from the exact FP32 displacement: up to MIXED_KDEF per thread and round of a
// tile (more such contacts than that within one thread's share of a row stay in
// FP32).
static constexpr int MIXED_KDEF = 8;

struct Kahan {
    float s, c;
    __device__ __forceinline__ void add(float x) {
        float y = x - c;
        float t = s + y;
        c = (t - s) - y;
        s = t;
    }
    __device__ __forceinline__ double value() const { return (double)s - (double)c; }
};

// One tile of the mixed-form LJ kernel, shared by the single-system kernel and
// the batched persistent kernels of the serving loop; P lanes per particle, CTAs
// of BLOCK threads.  The mbarrier `bar` is
// initialised by the caller; `uses` counts its completed phases (the parity of
// the next wait).  Adds the thread's partial potential energy and virial to
// pe / vir.  A tile whose staging exceeds `cap` sets ERR_TILE_CAP, or, with an
// overflow list, is appended to it (item `ovf_item`) for a kernel with more
// shared memory; the return value is then true (nothing computed).
template <int P, int BLOCK = FBLOCK_T>
__device__ __forceinline__ bool mixed_tile(long tile, const float4* __restrict__ off, long n_real, const TileGeom& tg,
                                           const unsigned int* __restrict__ csR,
                                           const unsigned int* __restrict__ csI, unsigned int cap,
                                           const unsigned int* __restrict__ nbr, const int* __restrict__ nn,
                                           long stride, float sx, float sy, float sz, const LJP<float>& Pr,
                                           float* __restrict__ f, long fcap, unsigned int* __restrict__ err,
                                           float4* sm, TileShM& S, unsigned long long* bar, unsigned int& uses,
                                           double& pe, double& vir, unsigned int* ovf_cnt = nullptr,
                                           long* ovf_list = nullptr, long ovf_item = 0) {
    {
        long t = tile;
        int tx = (int)(t % tg.ntx);
        long rest = t / tg.ntx;
        int y = (int)(rest % tg.ny) + tg.pad;
        int z = (int)(rest / tg.ny) + tg.pad;
        int x0 = tg.pad + tx * tg.TX;
        int x1 = min(x0 + tg.TX, tg.gs0 - tg.pad);
        int ncol = x1 - x0 + 3;
        for (int e = threadIdx.x; e < 18 * ncol; e += blockDim.x) {
            int img = e >= 9 * ncol;
            int ee = img ? e - 9 * ncol : e;
            int r = ee / ncol, j = ee % ncol;
            int dz = r / 3 - 1, dy = r % 3 - 1;
            long c = (long)(x0 - 1 + j) + (long)tg.gs0 * ((y + dy) + (long)tg.gs1 * (z + dz));
            if (img) S.cI[r][j] = csI[c];
            else S.cR[r][j] = csR[c];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned int o = 0;
            for (int r = 0; r < 9; ++r) {
                S.oR[r] = o;
                o += S.cR[r][ncol - 1] - S.cR[r][0];
                S.oI[r] = o;
                o += S.cI[r][ncol - 1] - S.cI[r][0];
            }
            S.total = o;
            S.ncol = ncol;
        }
        __syncthreads();
    }
    const int ncol = S.ncol;
    const unsigned int ib = S.cR[4][1], ie = S.cR[4][ncol - 2];
    const float c24 = Pr.eps24 / Pr.sig2;
    bool ok = ib != ie && S.total <= cap;
    if (ib != ie && S.total > cap) {
        if (ovf_cnt) {
            if (threadIdx.x == 0) ovf_list[atomicAdd(ovf_cnt, 1u)] = ovf_item;
            return true;
        }
        if (threadIdx.x == 0) atomicOr(err, ERR_TILE_CAP);
    }
    if (ok) {
        for (int e = threadIdx.x; e < 18 * ncol; e += blockDim.x) {
            int sg = e / ncol, j = e % ncol, r = sg >> 1;
            S.segb[sg][j] = (sg & 1) ? S.oI[r] + (S.cI[r][j] - S.cI[r][0]) : S.oR[r] + (S.cR[r][j] - S.cR[r][0]);
        }
        __syncthreads();
        if (threadIdx.x < 32)
            stage_ranges_warp(S, 0, 9, sm, 0u, off, off + n_real, S.total * (unsigned int)sizeof(float4), bar);
        bool waited = mbar_wait_bounded(bar, uses & 1u, 1u << 24);
        if (!waited) {
            atomicOr(err, ERR_TIMEOUT);
            mbar_wait_bounded(bar, uses & 1u, 1u << 24);
        }
        ++uses;
        ok = __syncthreads_and(waited ? 1 : 0) != 0;
    }
    if (ok) {
        // rewrite the staged records: y/z relative to the centre row, w = cell column
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (int sg = warp; sg < 18; sg += BLOCK / 32) {
            const int r = sg >> 1;
            const float shy = (float)(r % 3 - 1) * sy, shz = (float)(r / 3 - 1) * sz;
            for (unsigned int k = S.segb[sg][0] + lane; k < S.segb[sg][ncol - 1]; k += 32) {
                int j = 0;
                while (j < ncol - 2 && S.segb[sg][j + 1] <= k) ++j;
                float4 q = sm[k];
                q.y += shy;
                q.z += shz;
                q.w = (float)j;
                sm[k] = q;
            }
        }
        __syncthreads();
        const unsigned int base = S.oR[4] - S.cR[4][0];
        // staged indices of the pairs a thread sets aside for FP64, column per thread
        __shared__ unsigned short defer[MIXED_KDEF][BLOCK];
        // rounds of the whole CTA over the tile's particles: P lanes per row while a
        // round is full, more lanes per row (up to a warp) in the last, partial round;
        // every thread takes part in every round (the shuffles need whole warps)
        unsigned int first = ib;
        while (first < ie) {
            const unsigned int left = ie - first;
            unsigned int q = P;
            while (q < 32u && left * (q << 1) <= (unsigned int)BLOCK) q <<= 1;
            const unsigned int cnt = min(left, (unsigned int)BLOCK / q);
            const int sub = (int)(threadIdx.x % q);
            const int Q = (int)q;
            const bool active = threadIdx.x / q < cnt;
            const unsigned int i = first + (active ? threadIdx.x / q : 0u);
            const unsigned int li = base + i;
            const float4 xi = sm[li];
            const int words = active ? (nn[i] + 1) >> 1 : 0;
            Kahan kx = {0.f, 0.f}, ky = {0.f, 0.f}, kz = {0.f, 0.f}, ke = {0.f, 0.f}, kw = {0.f, 0.f};
            int nd = 0;  // wall pairs set aside in defer[][threadIdx.x]
            const unsigned int* row = nbr + i;
            // row words read four iterations ahead (register shift ring) to cover the memory latency
            unsigned int q0 = sub < words ? __ldg(row + (long)sub * stride) : 0u;
            unsigned int q1 = sub + Q < words ? __ldg(row + (long)(sub + Q) * stride) : 0u;
            unsigned int q2 = sub + 2 * Q < words ? __ldg(row + (long)(sub + 2 * Q) * stride) : 0u;
            unsigned int q3 = sub + 3 * Q < words ? __ldg(row + (long)(sub + 3 * Q) * stride) : 0u;
#pragma unroll 2
            for (int k = sub; k < words; k += Q) {
                const unsigned int pair = q0;
                q0 = q1;
                q1 = q2;
                q2 = q3;
                q3 = k + 4 * Q < words ? __ldg(row + (long)(k + 4 * Q) * stride) : 0u;
                float fx = 0.f, fy = 0.f, fz = 0.f, e = 0.f, w = 0.f;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const unsigned int l = h ? (pair >> 16) : (pair & 0xffffu);
                    const float4 xq = sm[l];
                    const float dx = fmaf(xi.w - xq.w, sx, xi.x - xq.x);
                    const float dy = xi.y - xq.y, dz = xi.z - xq.z;
                    const float r2 = dist2(dx, dy, dz);
                    // every pair through the same instructions; pairs outside select zero;
                    // pairs within FP32 rounding of the cutoff decided in FP64; pairs on the
                    // repulsive wall set aside for FP64 (while this thread's list has room)
                    const bool in = in_cut_exact(r2, dx, dy, dz, Pr) && l != li;
                    const bool wall = in && r2 < Pr.rclose2 && nd < MIXED_KDEF;
                    if (wall) defer[nd++][threadIdx.x] = (unsigned short)l;
                    const bool in32 = in && !wall;
                    // s2 zero outside (NaN for the particle itself, selected away) zeroes
                    // the force, energy and virial terms; 1 / r2 enters as s2 / sig2
                    const float s2v = div_by(Pr.sig2, r2);
                    const float s2 = in32 ? s2v : 0.f;
                    const float s6 = s2 * s2 * s2;
                    const float ff = s2 * s6 * fmaf(2.f * c24, s6, -c24);  // 24 eps (2 s12 - s6) / r2
                    fx += ff * dx;
                    fy += ff * dy;
                    fz += ff * dz;
                    e = fmaf(s6, fmaf(Pr.eps4, s6, -Pr.eps4), e);  // 4 eps (s12 - s6)
                    w += ff * r2;
                }
                kx.add(fx);
                ky.add(fy);
                kz.add(fz);
                ke.add(e);
                kw.add(w);
            }
            double Fx = kx.value(), Fy = ky.value(), Fz = kz.value(), Ee = ke.value(), Ww = kw.value();
            // the set-aside wall pairs in FP64: the displacement is exact in FP32, so it
            // converts exactly; r2 and the pair terms then carry FP64 rounding only
            for (int k = 0; k < nd; ++k) {
                const float4 xq = sm[defer[k][threadIdx.x]];
                const double dx = fmaf(xi.w - xq.w, sx, xi.x - xq.x);
                const double dy = xi.y - xq.y, dz = xi.z - xq.z;
                const double r2 = dist2(dx, dy, dz);
                const double ir2 = recip(r2);
                const double s2 = Pr.sig2d * ir2;
                const double s6 = s2 * s2 * s2;
                const double ff = Pr.eps24d * ir2 * s6 * (2.0 * s6 - 1.0);
                Fx += ff * dx;
                Fy += ff * dy;
                Fz += ff * dz;
                Ee += Pr.eps4d * s6 * (s6 - 1.0);
                Ww += ff * r2;
            }
            for (unsigned int o = 1; o < q; o <<= 1) {
                Fx += __shfl_xor_sync(0xffffffffu, Fx, o);
                Fy += __shfl_xor_sync(0xffffffffu, Fy, o);
                Fz += __shfl_xor_sync(0xffffffffu, Fz, o);
                Ee += __shfl_xor_sync(0xffffffffu, Ee, o);
                Ww += __shfl_xor_sync(0xffffffffu, Ww, o);
            }
            if (active && sub == 0) {
                f[i] = (float)Fx;
                f[fcap + i] = (float)Fy;
                f[2 * fcap + i] = (float)Fz;
                pe += 0.5 * Ee;
                vir += 0.5 * Ww;
            }
            first += cnt;
        }
    }
    return false;
}

}  // namespace pd
