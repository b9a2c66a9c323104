// pd_tile_dev.cuh -- device code of the tiled Verlet structure shared by the
// single-system kernels (pd_tile.cu) and the batched kernels of the serving loop
// (pd_serve.cu): tile layout, TMA staging of the 18 neighbour ranges, row build.
#pragma once
#include "pd_device.cuh"
#include "pd_internal.cuh"
#include "pd_tile.cuh"

namespace pd {

// Rows hold two 16-bit entries per 32-bit word: entries 2w and 2w+1 of particle
// i share word w*stride + i (column-major over words).
__device__ __forceinline__ long pair_slot(int k, long stride, unsigned int i) {
    return (((long)(k >> 1) * stride + i) << 1) | (k & 1);
}

struct TileSh {
    unsigned int cR[9][TXMAX + 3];
    unsigned int cI[9][TXMAX + 3];
    unsigned int oR[9], oI[9];
    unsigned int total;
    int ncol;
    unsigned long long bar;
};

__device__ __forceinline__ void tile_layout(const TileGeom& tg, long t, const unsigned int* __restrict__ csR,
                                            const unsigned int* __restrict__ csI, TileSh& S) {
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
    // staging offsets of the 18 ranges (row r's real range, then its images, r = 0..8):
    // an exclusive scan of their lengths across the first warp
    if (threadIdx.x < 32) {
        const int s = (int)threadIdx.x, r = s >> 1;
        unsigned int len = 0;
        if (s < 18) len = (s & 1) ? S.cI[r][ncol - 1] - S.cI[r][0] : S.cR[r][ncol - 1] - S.cR[r][0];
        unsigned int inc = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned int v = __shfl_up_sync(0xffffffffu, inc, o);
            if (s >= o) inc += v;
        }
        if (s < 18) {
            if (s & 1) S.oI[r] = inc - len;
            else S.oR[r] = inc - len;
        }
        if (s == 17) S.total = inc;
        if (s == 0) S.ncol = ncol;
    }
    __syncthreads();
}

// The bulk copies of a tile's staged ranges of rows [r0, r0 + nrow), issued by the
// first warp, one lane a range (lane 2k: row r0 + k's real range, 2k + 1: its
// images), into dst at the ranges' staging offsets less `base`; lane 0 first sets the
// barrier's expected bytes.  Called by the whole first warp.
template <class TS, class T4>
__device__ __forceinline__ void stage_ranges_warp(const TS& S, int r0, int nrow, T4* dst, unsigned int base,
                                                  const T4* __restrict__ preal, const T4* __restrict__ pimg,
                                                  unsigned int bytes, unsigned long long* bar) {
    const unsigned int lane = threadIdx.x & 31u;
    if (lane == 0) mbar_arrive_expect_tx(bar, bytes);
    __syncwarp();
    if (lane < 2u * (unsigned int)nrow) {
        const int r = r0 + (int)(lane >> 1), nc = S.ncol - 1;
        const bool img = lane & 1u;
        const unsigned int c0 = img ? S.cI[r][0] : S.cR[r][0];
        const unsigned int len = (img ? S.cI[r][nc] : S.cR[r][nc]) - c0;
        if (len)
            bulk_g2s(dst + ((img ? S.oI[r] : S.oR[r]) - base), (img ? pimg : preal) + c0,
                     len * (unsigned int)sizeof(T4), bar);
    }
}

// Stage the tile's 18 ranges; false (uniformly) if the tile does not fit or the
// bounded wait gave up (error bit set).
template <class T>
__device__ __forceinline__ bool tile_stage(const typename V4<T>::type* __restrict__ preal,
                                           const typename V4<T>::type* __restrict__ pimg, TileSh& S,
                                           typename V4<T>::type* sm, unsigned int cap, unsigned int* err) {
    typedef typename V4<T>::type T4;
    if (S.total > cap) {
        if (threadIdx.x == 0) atomicOr(err, ERR_TILE_CAP);
        return false;
    }
    if (S.total == 0) return true;
    if (threadIdx.x == 0) mbar_init(&S.bar, 1);
    __syncthreads();
    if (threadIdx.x < 32) stage_ranges_warp(S, 0, 9, sm, 0u, preal, pimg, S.total * (unsigned int)sizeof(T4), &S.bar);
    bool ok = mbar_wait_bounded(&S.bar, 0, 1u << 24);
    if (!ok) {
        atomicOr(err, ERR_TIMEOUT);
        mbar_wait_bounded(&S.bar, 0, 1u << 24);  // let copies in flight land before the CTA exits
    }
    return __syncthreads_and(ok ? 1 : 0) != 0;
}

// staging with a caller-owned mbarrier (persistent CTAs): `parity` is the phase the
// wait expects; returns 1 if copies were issued (the caller flips its parity), 0 if
// none were needed, -1 if the tile does not fit or the bounded wait gave up.
template <class T>
__device__ __forceinline__ int tile_stage_bar(const typename V4<T>::type* __restrict__ preal,
                                              const typename V4<T>::type* __restrict__ pimg, const TileSh& S,
                                              typename V4<T>::type* sm, unsigned int cap, unsigned int* err,
                                              unsigned long long* bar, unsigned int parity) {
    typedef typename V4<T>::type T4;
    if (S.total > cap) {
        if (threadIdx.x == 0) atomicOr(err, ERR_TILE_CAP);
        return -1;
    }
    if (S.total == 0) return 0;
    if (threadIdx.x < 32) stage_ranges_warp(S, 0, 9, sm, 0u, preal, pimg, S.total * (unsigned int)sizeof(T4), bar);
    bool ok = mbar_wait_bounded(bar, parity, 1u << 24);
    if (!ok) {
        atomicOr(err, ERR_TIMEOUT);
        mbar_wait_bounded(bar, parity, 1u << 24);  // let copies in flight land
    }
    return __syncthreads_and(ok ? 1 : 0) ? 1 : -1;
}

// exact predicate for the rare candidates inside the FP32 uncertainty band
template <class T>
__device__ __noinline__ bool exact_in(const typename V4<T>::type* __restrict__ pos, unsigned int i, int q, T r2) {
    typename V4<T>::type a = ld4(pos, (long)i), b = ld4(pos, (long)q);
    return dist2(a.x - b.x, a.y - b.y, a.z - b.z) < r2;
}

// absolute staging index of every cell start, per segment
__device__ __forceinline__ void tile_segb(const TileSh& S, unsigned int (*segb)[TXMAX + 3]) {
    const int ncol = S.ncol;
    for (int e = threadIdx.x; e < 18 * ncol; e += blockDim.x) {
        int sg = e / ncol, j = e % ncol, r = sg >> 1;
        segb[sg][j] = (sg & 1) ? S.oI[r] + (S.cI[r][j] - S.cI[r][0]) : S.oR[r] + (S.cR[r][j] - S.cR[r][0]);
    }
}

// Accept mask of one chunk of n <= 32 staged candidates (c4[0..n)) for the
// particle at x: the sign of t = d2 - lo_thr (surely in) shifted in, the first
// candidate ending in the highest bit: bit n-1-k stands for c4[k] (fl(a - b) < 0
// exactly when a < b for finite a, b).  Candidates possibly in (lo_thr <= d2 <
// hi_thr) have 0 <= t <= fl(hi_thr - lo_thr); non-negative floats order like
// their bit patterns and negative ones have the sign bit, so a running unsigned
// minimum of the patterns flags them, one instruction a candidate.  The rare
// flagged chunk is walked again and its band candidates decided exactly in the
// position type.
template <class T>
__device__ __forceinline__ unsigned int chunk_mask(const float4* __restrict__ c4, unsigned int n, const float4 x,
                                                   unsigned int i, const typename V4<T>::type* __restrict__ pos,
                                                   T r2, float lo_thr, float hi_thr) {
    unsigned int m = 0, umin = 0xffffffffu;
#pragma unroll 4
    for (unsigned int k = 0; k < n; ++k) {
        const float4 xq = c4[k];
        const float d2 = dist2(x.x - xq.x, x.y - xq.y, x.z - xq.z);
        const unsigned int t = __float_as_uint(d2 - lo_thr);
        m = __funnelshift_l(t, m, 1);
        umin = min(umin, t);
    }
    if (umin <= __float_as_uint(hi_thr - lo_thr)) {
        for (unsigned int k = 0; k < n; ++k) {
            const float4 xq = c4[k];
            const float d2 = dist2(x.x - xq.x, x.y - xq.y, x.z - xq.z);
            if (!(d2 < lo_thr) && d2 < hi_thr && exact_in<T>(pos, i, __float_as_int(xq.w), r2))
                m |= 1u << (n - 1 - k);
        }
    }
    return m;
}

// Row entries of particle i (global index; FP32 copy x) from the staged candidates
// [qb, qe), staging indices, candidate q at sm[q - base], appended in ascending q
// (the entries of the candidate-by-candidate walk, in its order).  Up to three
// chunks of 32 are tested into masks first; their accepted candidates then leave
// as one stream, two entries (one 32-bit word) at a time, so a lane's loop runs
// about half its accept count rather than the sum of the chunks' largest counts
// over the warp.  c counts the row's entries, pend holds the first half of an
// unfinished word.
template <class T>
__device__ __forceinline__ void seg_rows(const float4* __restrict__ sm, unsigned int base, unsigned int qb,
                                         unsigned int qe, const float4 x, unsigned int i,
                                         const typename V4<T>::type* __restrict__ pos, T r2, float lo_thr,
                                         float hi_thr, unsigned int* __restrict__ out, long stride, int max_nn,
                                         int& c, unsigned int& pend) {
#pragma unroll 1
    for (unsigned int q0 = qb; q0 < qe; q0 += 96) {
        const unsigned int n = min(96u, qe - q0);
        const unsigned int na = min(32u, n), nb = min(32u, n - na), nc = n - na - nb;
        const float4* c4 = sm + (q0 - base);
        unsigned int ma = chunk_mask<T>(c4, na, x, i, pos, r2, lo_thr, hi_thr);
        unsigned int mb = chunk_mask<T>(c4 + 32, nb, x, i, pos, r2, lo_thr, hi_thr);
        unsigned int mc = chunk_mask<T>(c4 + 64, nc, x, i, pos, r2, lo_thr, hi_thr);
        // candidate of bit b of a mask: qt - 31 + clz position, qt = last q of the chunk
        unsigned int qa = q0 + na - 32, qb_ = q0 + 32 + nb - 32, qc = q0 + 64 + nc - 32;
        int rem = __popc(ma) + __popc(mb) + __popc(mc);
        if (rem == 0) continue;
        // the stream: ma first; an emptied mask takes the next one's place
        if (ma == 0) { ma = mb; qa = qb_; mb = mc; qb_ = qc; mc = 0; }
        if (ma == 0) { ma = mb; qa = qb_; mb = 0; }
        if (mb == 0) { mb = mc; qb_ = qc; mc = 0; }
        auto next = [&]() -> unsigned int {
            const int z = __clz(ma);
            const unsigned int q = qa + (unsigned int)z;
            ma ^= 0x80000000u >> z;
            if (ma == 0) { ma = mb; qa = qb_; mb = mc; qb_ = qc; mc = 0; }
            return q;
        };
        if (c & 1) {  // complete the pending word
            const unsigned int q = next();
            if (c < max_nn) out[(long)(c >> 1) * stride] = pend | (q << 16);
            ++c;
            --rem;
        }
        for (; rem >= 2; rem -= 2, c += 2) {
            const unsigned int q1 = next();
            const unsigned int q2 = next();
            if (c < max_nn) out[(long)(c >> 1) * stride] = q1 | (q2 << 16);
        }
        if (rem) {
            pend = next();
            ++c;
        }
    }
}

// List build of one staged tile.  The candidates are staged as FP32 copies; d2
// in FP32 decides every pair farther than `band` from r^2 (|d2_f32 - d2_exact| <
// band by the error bound computed on the host), the few inside the band are
// decided exactly in the position type T from global memory -- so the rows equal
// the exact predicate d2 < r^2.  Entries are stored a 32-bit word (two entries)
// at a time.
template <class T>
__device__ __forceinline__ void tile_rows(const TileSh& S, const unsigned int (*segb)[TXMAX + 3], const float4* sm,
                                          const typename V4<T>::type* __restrict__ pos, T r2, float lo_thr,
                                          float hi_thr, unsigned int* __restrict__ nbr, int* __restrict__ nn,
                                          long stride, int max_nn, unsigned int* __restrict__ err,
                                          unsigned int* __restrict__ nn_max) {
    const unsigned int ib = S.cR[4][1], ie = S.cR[4][S.ncol - 2];
    const int ncol = S.ncol;
    const unsigned int self_base = S.oR[4] - S.cR[4][0];
    for (unsigned int i = ib + threadIdx.x; i < ie; i += blockDim.x) {
        const float4 xi = sm[self_base + i];
        int j = 1;
        while (j < ncol - 2 && S.cR[4][j + 1] <= i) ++j;
        int cnt = 0;
        unsigned int pend = 0;
        unsigned int* out = nbr + i;
#pragma unroll 1
        for (int sg = 0; sg < 18; ++sg)
            seg_rows<T>(sm, 0, segb[sg][j - 1], segb[sg][j + 2], xi, i, pos, r2, lo_thr, hi_thr, out, stride, max_nn,
                        cnt, pend);
        // odd rows end with the particle itself, which the pair kernel skips
        if ((cnt & 1) && cnt < max_nn) out[(long)(cnt >> 1) * stride] = pend | ((self_base + i) << 16);
        if (cnt > max_nn) {
            atomicOr(err, ERR_NN_OVERFLOW);
            atomicMax(nn_max, (unsigned int)cnt);
            cnt = max_nn;
        }
        nn[i] = cnt;
    }
}

// Row build of one tile in three passes of one z-layer each (rows 0-2, 3-5, 6-8:
// segments 0-5, 6-11, 12-17), staged one after the other into the same shared
// memory of `pcap` records.  A particle's entry count and pending half-word carry
// over the passes, so its row holds the entries in the same order as the
// single-pass walk (tile_rows); entries index the full staging layout, which the
// pair kernels stage.  The caller owns the mbarrier; `ph` counts its completed
// phases.  Returns false (uniformly) if the tile does not fit (ERR_TILE_CAP: a
// layer beyond pcap) or a wait gave up.
template <class T>
__device__ __forceinline__ bool tile_rows_layers(const TileSh& S, const unsigned int (*segb)[TXMAX + 3],
                                                 const float4* __restrict__ preal, const float4* __restrict__ pimg,
                                                 float4* sm, unsigned int pcap,
                                                 const typename V4<T>::type* __restrict__ pos, T r2, float lo_thr,
                                                 float hi_thr, unsigned int* __restrict__ nbr, int* __restrict__ nn,
                                                 long stride, int max_nn, unsigned int* __restrict__ err,
                                                 unsigned int* __restrict__ nn_max, unsigned long long* bar,
                                                 unsigned int& ph) {
    const unsigned int ib = S.cR[4][1], ie = S.cR[4][S.ncol - 2];
    const int ncol = S.ncol;
    const unsigned int self_base = S.oR[4] - S.cR[4][0];
    // each thread: up to MAXI domain particles of a sweep, one per blockDim.x of the
    // tile's particles in order; a tile of more than MAXI * blockDim.x particles (a
    // dense column) takes further sweeps, each staging the three layers again
    constexpr int MAXI = 2;
    const unsigned int sweep = (unsigned int)MAXI * blockDim.x;
    for (unsigned int sb = ib; sb < ie; sb += sweep) {
        float4 xi[MAXI];
        int jcol[MAXI], cnt[MAXI];
        unsigned int pend[MAXI];
        int nmine = 0;
        for (unsigned int i = sb + threadIdx.x; i < ie && nmine < MAXI; i += blockDim.x, ++nmine) {
            xi[nmine] = preal[i];
            int j = 1;
            while (j < ncol - 2 && S.cR[4][j + 1] <= i) ++j;
            jcol[nmine] = j;
            cnt[nmine] = 0;
            pend[nmine] = 0;
        }
        for (int pass = 0; pass < 3; ++pass) {
            const unsigned int base = S.oR[3 * pass];
            const unsigned int end = pass < 2 ? S.oR[3 * pass + 3] : S.total;
            const unsigned int tot = end - base;
            if (tot > pcap) {
                if (threadIdx.x == 0) atomicOr(err, ERR_TILE_CAP);
                return false;
            }
            bool ok = true;
            if (tot > 0) {
                if (threadIdx.x < 32)
                    stage_ranges_warp(S, 3 * pass, 3, sm, base, preal, pimg, tot * (unsigned int)sizeof(float4), bar);
                ok = mbar_wait_bounded(bar, ph & 1u, 1u << 24);
                if (!ok) {
                    atomicOr(err, ERR_TIMEOUT);
                    mbar_wait_bounded(bar, ph & 1u, 1u << 24);
                }
                ++ph;
            }
            if (!__syncthreads_and(ok ? 1 : 0)) return false;
            for (int m = 0; m < nmine; ++m) {
                const unsigned int i = sb + threadIdx.x + (unsigned int)m * blockDim.x;
                const int j = jcol[m];
                const float4 x = xi[m];
                int c = cnt[m];
                unsigned int pd_ = pend[m];
                unsigned int* out = nbr + i;
#pragma unroll 1
                for (int sg = 6 * pass; sg < 6 * pass + 6; ++sg)
                    seg_rows<T>(sm, base, segb[sg][j - 1], segb[sg][j + 2], x, i, pos, r2, lo_thr, hi_thr, out,
                                stride, max_nn, c, pd_);
                cnt[m] = c;
                pend[m] = pd_;
            }
            // every thread is done with this layer before the next one is copied over it
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
        }
        for (int m = 0; m < nmine; ++m) {
            const unsigned int i = sb + threadIdx.x + (unsigned int)m * blockDim.x;
            int c = cnt[m];
            unsigned int* out = nbr + i;
            // odd rows end with the particle itself, which the pair kernel skips
            if ((c & 1) && c < max_nn) out[(long)(c >> 1) * stride] = pend[m] | ((self_base + i) << 16);
            if (c > max_nn) {
                atomicOr(err, ERR_NN_OVERFLOW);
                atomicMax(nn_max, (unsigned int)c);
                c = max_nn;
            }
            nn[i] = c;
        }
    }
    return true;
}

}  // namespace pd
