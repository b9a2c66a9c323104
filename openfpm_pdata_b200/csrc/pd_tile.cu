// pd_tile.cu -- tiled neighbour structure of the integrator: Verlet rows as
// tile-local 16-bit indices into a shared-memory staging of the neighbour cells.
//
// Layout after a rebuild (cell grid of side r_cut + skin):
//   real particles [0, n_real)        sorted by cell, cell starts csR[ncells+1]
//   periodic images [n_real, n_total) sorted by cell, cell starts csI (relative)
// A tile is TX consecutive cells along x of one cell row (y, z).  Its
// neighbourhood is 9 rows (dy, dz in {-1,0,1}) x cells x0-1 .. x0+TX, i.e. 9
// contiguous ranges of real particles and 9 of images.  One CTA per tile copies
// those 18 ranges into shared memory with 1-D TMA bulk copies
// (cp.async.bulk global -> shared, mbarrier completion, no multicast), in the
// order R0, I0, R1, I1, ... R8, I8.  The Verlet row of a domain particle of the
// tile stores positions in that staging (uint16), column-major
// nbr[k*stride + i]; the force kernel stages the same ranges and reads every
// neighbour from shared memory.  Compared with global int32 indices this halves
// the list bytes and replaces dependent global gathers by shared-memory loads.
// Walk order per row: the real cells x-1..x+1, then the image cells x-1..x+1.
#include "pd_device.cuh"
#include "pd_internal.cuh"
#include "pd_lj.cuh"
#include "pd_tile.cuh"
#include "pd_tile_dev.cuh"

#include <cmath>

namespace pd {

// largest staged neighbourhood and largest centre count over the tiles
__global__ void k_tile_sizes(TileGeom tg, long ntiles, const unsigned int* __restrict__ csR,
                             const unsigned int* __restrict__ csI, unsigned int* __restrict__ tmax,
                             unsigned int* __restrict__ cmax, unsigned int* __restrict__ pmax) {
    unsigned int mt = 0, mc = 0, mp = 0;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < ntiles; t += (long)gridDim.x * blockDim.x) {
        int tx = (int)(t % tg.ntx);
        long rest = t / tg.ntx;
        int y = (int)(rest % tg.ny) + tg.pad;
        int z = (int)(rest / tg.ny) + tg.pad;
        int x0 = tg.pad + tx * tg.TX;
        int x1 = min(x0 + tg.TX, tg.gs0 - tg.pad);
        unsigned int tot = 0, pass = 0;
        for (int r = 0; r < 9; ++r) {
            int dz = r / 3 - 1, dy = r % 3 - 1;
            long rb = (long)tg.gs0 * ((y + dy) + (long)tg.gs1 * (z + dz));
            const unsigned int rt = (csR[rb + x1 + 1] - csR[rb + x0 - 1]) + (csI[rb + x1 + 1] - csI[rb + x0 - 1]);
            tot += rt;
            pass += rt;
            if (r % 3 == 2) {
                mp = max(mp, pass);
                pass = 0;
            }
            if (r == 4) mc = max(mc, csR[rb + x1] - csR[rb + x0]);
        }
        mt = max(mt, tot);
    }
    mt = warp_max(mt);
    mc = warp_max(mc);
    mp = warp_max(mp);
    if ((threadIdx.x & 31) == 0) {
        atomicMax(tmax, mt);
        atomicMax(cmax, mc);
        atomicMax(pmax, mp);
    }
}

// pos32[k] = (float)pos[k] (x, y, z) with the slot index in w: the staged copy of
// the list build, half the bytes of the FP64 records
template <class T>
__global__ void k_pos32(const typename V4<T>::type* __restrict__ pos, long n, float4* __restrict__ out) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        typename V4<T>::type r = ld4(pos, k);
        out[k] = make_float4((float)r.x, (float)r.y, (float)r.z, __int_as_float((int)k));
    }
}

// List build: one CTA per tile (rows: tile_rows in pd_tile_dev.cuh).
template <class T>
__global__ void __launch_bounds__(TBLOCK) k_vtile_build(const typename V4<T>::type* __restrict__ pos,
                                                        const float4* __restrict__ pos32, long n_real,
                                                        TileGeom tg, const unsigned int* __restrict__ csR,
                                                        const unsigned int* __restrict__ csI, unsigned int cap, T r2,
                                                        float lo_thr, float hi_thr, unsigned int* __restrict__ nbr,
                                                        int* __restrict__ nn, long stride, int max_nn,
                                                        unsigned int* __restrict__ err,
                                                        unsigned int* __restrict__ nn_max) {
    extern __shared__ __align__(128) unsigned char tile_raw[];
    float4* sm = reinterpret_cast<float4*>(tile_raw);
    __shared__ TileSh S;
    __shared__ unsigned int segb[18][TXMAX + 3];
    tile_layout(tg, blockIdx.x, csR, csI, S);
    const unsigned int ib = S.cR[4][1], ie = S.cR[4][S.ncol - 2];
    if (ib == ie) return;
    tile_segb(S, segb);
    if (!tile_stage<float>(pos32, pos32 + n_real, S, sm, cap, err)) return;  // (its barrier also covers segb)
    tile_rows<T>(S, segb, sm, pos, r2, lo_thr, hi_thr, nbr, nn, stride, max_nn, err, nn_max);
}

// List build in three passes of one z-layer each (tile_rows_layers in
// pd_tile_dev.cuh): a third of the full staging, more resident CTAs.
template <class T>
__global__ void __launch_bounds__(TBLOCK, 9) k_vtile_build3(const typename V4<T>::type* __restrict__ pos,
                                                         const float4* __restrict__ pos32, long n_real,
                                                         TileGeom tg, const unsigned int* __restrict__ csR,
                                                         const unsigned int* __restrict__ csI, unsigned int pcap,
                                                         T r2, float lo_thr, float hi_thr,
                                                         unsigned int* __restrict__ nbr, int* __restrict__ nn,
                                                         long stride, int max_nn, unsigned int* __restrict__ err,
                                                         unsigned int* __restrict__ nn_max) {
    extern __shared__ __align__(128) unsigned char tile_raw[];
    float4* sm = reinterpret_cast<float4*>(tile_raw);
    __shared__ TileSh S;
    __shared__ unsigned int segb[18][TXMAX + 3];
    tile_layout(tg, blockIdx.x, csR, csI, S);
    const unsigned int ib = S.cR[4][1], ie = S.cR[4][S.ncol - 2];
    if (ib == ie) return;
    tile_segb(S, segb);
    if (threadIdx.x == 0) mbar_init(&S.bar, 1);
    __syncthreads();
    unsigned int ph = 0;
    tile_rows_layers<T>(S, segb, pos32, pos32 + n_real, sm, pcap, pos, r2, lo_thr, hi_thr, nbr, nn, stride, max_nn,
                        err, nn_max, &S.bar, ph);
}

// P threads per domain particle split its row (words w = sub, sub+P, ...; two
// entries per word) -- more in a tile's last, partial round; partial sums meet
// through shuffles.  Energies: one FP64
// partial per block (fixed-order tree), reduced in fixed order afterwards.
template <class T, bool ENERGY, int P>
__global__ void __launch_bounds__(FBLOCK_T) k_vtile_lj(const typename V4<T>::type* __restrict__ pos, long n_real,
                                                       TileGeom tg, const unsigned int* __restrict__ csR,
                                                       const unsigned int* __restrict__ csI, unsigned int cap,
                                                       const unsigned int* __restrict__ nbr,
                                                       const int* __restrict__ nn, long stride, LJP<T> Pr,
                                                       T* __restrict__ f, long fcap, double* __restrict__ part,
                                                       unsigned int* __restrict__ err) {
    typedef typename V4<T>::type T4;
    extern __shared__ __align__(128) unsigned char tile_raw[];
    T4* sm = reinterpret_cast<T4*>(tile_raw);
    __shared__ TileSh S;
    tile_layout(tg, blockIdx.x, csR, csI, S);
    const unsigned int ib = S.cR[4][1], ie = S.cR[4][S.ncol - 2];
    double pe = 0, vir = 0;
    bool staged = ib != ie && tile_stage<T>(pos, pos + n_real, S, sm, cap, err);
    if (staged) {
        const unsigned int base = S.oR[4] - S.cR[4][0];
        // Rounds of the whole CTA over the tile's domain particles: P lanes share a
        // row while a round is full; the last, partial round spreads its particles
        // over more lanes (up to a warp each) so that it ends about as soon as the
        // full ones instead of leaving most warps idle at the block's barrier.
        // Every thread takes part in every round (the shuffles need whole warps).
        unsigned int first = ib;
        while (first < ie) {
            const unsigned int left = ie - first;
            unsigned int q = P;
            while (q < 32u && left * (q << 1) <= (unsigned int)FBLOCK_T) q <<= 1;
            const unsigned int cnt = min(left, (unsigned int)FBLOCK_T / q);
            const int sub = (int)(threadIdx.x % q);
            const bool active = threadIdx.x / q < cnt;
            const unsigned int i = first + (active ? threadIdx.x / q : 0u);
            const unsigned int li = base + i;
            T4 xi = sm[li];
            const int words = active ? (nn[i] + 1) >> 1 : 0;
            const int Q = (int)q;
            T fx = 0, fy = 0, fz = 0, e = 0, w = 0;
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
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const unsigned int l = h ? (pair >> 16) : (pair & 0xffffu);
                    T4 xq = sm[l];
                    T dx = xi.x - xq.x, dy = xi.y - xq.y, dz = xi.z - xq.z;
                    T r2 = dist2(dx, dy, dz);
                    // every pair through the same instructions (most lanes of a warp have a
                    // pair inside the cutoff at every step); the others contribute zero
                    const bool in = r2 < Pr.rc2 && l != li;
                    const T ir2 = recip(in ? r2 : T(1));
                    const T s2 = Pr.sig2 * ir2;
                    const T s6 = s2 * s2 * s2;
                    const T ff = in ? Pr.eps24 * ir2 * s6 * (T(2) * s6 - T(1)) : T(0);
                    fx += ff * dx;
                    fy += ff * dy;
                    fz += ff * dz;
                    if (ENERGY) {
                        e += in ? Pr.eps4 * s6 * (s6 - T(1)) : T(0);
                        w += ff * r2;
                    }
                }
            }
            for (unsigned int o = 1; o < q; o <<= 1) {
                fx += __shfl_xor_sync(0xffffffffu, fx, o);
                fy += __shfl_xor_sync(0xffffffffu, fy, o);
                fz += __shfl_xor_sync(0xffffffffu, fz, o);
                if (ENERGY) {
                    e += __shfl_xor_sync(0xffffffffu, e, o);
                    w += __shfl_xor_sync(0xffffffffu, w, o);
                }
            }
            if (active && sub == 0) {
                f[i] = fx;
                f[fcap + i] = fy;
                f[2 * fcap + i] = fz;
                if (ENERGY) {
                    pe += 0.5 * (double)e;
                    vir += 0.5 * (double)w;
                }
            }
            first += cnt;
        }
    }
    if (ENERGY) {
        pe = block_sum<double, FBLOCK_T>(pe);
        vir = block_sum<double, FBLOCK_T>(vir);
        if (threadIdx.x == 0) {
            part[2 * blockIdx.x] = pe;
            part[2 * blockIdx.x + 1] = vir;
        }
    }
}

// The same pair loop on split staging: (x, y) as 16-byte records through the bulk
// copies and z as 8-byte values loaded by the CTA (their ranges need not start on
// a 16-byte boundary), 24 bytes a record instead of 32; (x, y) records of
// consecutive slots fall on all eight 16-byte bank groups.
template <bool ENERGY, int P, int MINB, bool DRIFT>
__global__ void __launch_bounds__(FBLOCK_T, MINB) k_vtile_lj_xyz(const double2* __restrict__ xy,
                                                           const double* __restrict__ zz, long n_real, TileGeom tg,
                                                           const unsigned int* __restrict__ csR,
                                                           const unsigned int* __restrict__ csI, unsigned int cap,
                                                           const unsigned int* __restrict__ nbr,
                                                           const int* __restrict__ nn, long stride, int mwords,
                                                           LJP<double> Pr,
                                                           double* __restrict__ f, long fcap,
                                                           double* __restrict__ part, unsigned int* __restrict__ err,
                                                           DriftArgs D) {
    static_assert(ENERGY || !DRIFT, "the drift's kinetic energy partials ride on the energy partials");
    extern __shared__ __align__(128) unsigned char tile_raw[];
    double2* sxy = reinterpret_cast<double2*>(tile_raw);
    double* sz = reinterpret_cast<double*>(tile_raw + (size_t)cap * sizeof(double2));
    __shared__ TileSh S;
    tile_layout(tg, blockIdx.x, csR, csI, S);
    const unsigned int ib = S.cR[4][1], ie = S.cR[4][S.ncol - 2];
    const double c24 = Pr.eps24 / Pr.sig2;
    double pe = 0, vir = 0, ke = 0, md2 = 0;
    // (x, y) by bulk copies; the CTA loads z while they are in flight
    bool staged = false;
    if (ib != ie) {
        if (S.total > cap) {
            if (threadIdx.x == 0) atomicOr(err, ERR_TILE_CAP);
        } else {
            const int nc = S.ncol - 1;
            const unsigned int lane = threadIdx.x & 31u;
            if (threadIdx.x < 32) {
                if (lane == 0) mbar_init(&S.bar, 1);
                __syncwarp();
                stage_ranges_warp(S, 0, 9, sxy, 0u, xy, xy + n_real, S.total * (unsigned int)sizeof(double2), &S.bar);
            }
            // z of the same ranges, a warp a range, while the copies are in flight
            for (int sg = (int)(threadIdx.x >> 5); sg < 18; sg += FBLOCK_T / 32) {
                const int r = sg >> 1;
                const bool img = sg & 1;
                const unsigned int c0 = img ? S.cI[r][0] : S.cR[r][0];
                const unsigned int len = (img ? S.cI[r][nc] : S.cR[r][nc]) - c0;
                const double* src = zz + (img ? n_real : 0L) + c0;
                double* dst = sz + (img ? S.oI[r] : S.oR[r]);
#pragma unroll 4
                for (unsigned int k = lane; k < len; k += 32u) dst[k] = __ldg(src + k);
            }
            // every thread waits on the barrier only after the first lane initialised it
            __syncthreads();
            bool ok = mbar_wait_bounded(&S.bar, 0, 1u << 24);
            if (!ok) {
                atomicOr(err, ERR_TIMEOUT);
                mbar_wait_bounded(&S.bar, 0, 1u << 24);  // let copies in flight land before the CTA exits
            }
            staged = __syncthreads_and(ok ? 1 : 0) != 0;
        }
    }
    if (staged) {
        const unsigned int base = S.oR[4] - S.cR[4][0];
        unsigned int first = ib;
        while (first < ie) {
            const unsigned int left = ie - first;
            unsigned int q = P;
            while (q < 32u && left * (q << 1) <= (unsigned int)FBLOCK_T) q <<= 1;
            const unsigned int cnt = min(left, (unsigned int)FBLOCK_T / q);
            const int sub = (int)(threadIdx.x % q);
            const bool active = threadIdx.x / q < cnt;
            const unsigned int i = first + (active ? threadIdx.x / q : 0u);
            const unsigned int li = base + i;
            const double2 xyi = sxy[li];
            const double zi = sz[li];
            const int Q = (int)q;
            const unsigned int* row = nbr + i;
            // the first row words are read together with the row length (within the
            // buffer's mwords words per particle), not after it
            unsigned int q0 = sub < mwords ? __ldg(row + (long)sub * stride) : 0u;
            unsigned int q1 = sub + Q < mwords ? __ldg(row + (long)(sub + Q) * stride) : 0u;
            unsigned int q2 = sub + 2 * Q < mwords ? __ldg(row + (long)(sub + 2 * Q) * stride) : 0u;
            unsigned int q3 = sub + 3 * Q < mwords ? __ldg(row + (long)(sub + 3 * Q) * stride) : 0u;
            const int words = active ? (nn[i] + 1) >> 1 : 0;
            if (DRIFT && active && sub == 0) {
                // the drift's operands into L2 while the row is computed
                prefetch_l2(D.v + i);
                prefetch_l2(D.v + D.vcap + i);
                prefetch_l2(D.v + 2 * D.vcap + i);
                prefetch_l2(D.pos + i);
                prefetch_l2(D.xb + i);
            }
            double fx = 0, fy = 0, fz = 0, e = 0, w = 0;
            // one pair (rows hold the particle itself, as the reference's full list
            // does): outside the cutoff or self, s2 is zero and with it the force,
            // energy and virial terms -- one select; 1 / r2 enters the force as
            // s2 / sig2 (c24 = 24 eps / sig2)
            auto pair_term = [&](unsigned int l) {
                const double2 xyq = sxy[l];
                const double dx = xyi.x - xyq.x, dy = xyi.y - xyq.y, dz = zi - sz[l];
                const double r2 = dist2(dx, dy, dz);
                const bool in = r2 < Pr.rc2 && l != li;
                const double s2v = div_by(Pr.sig2, r2);  // NaN for the particle itself, selected away
                const double s2 = in ? s2v : 0.0;
                const double s6 = s2 * s2 * s2;
                const double ff = s2 * s6 * fma(2.0 * c24, s6, -c24);  // 24 eps (2 s12 - s6) / r2
                fx = fma(ff, dx, fx);
                fy = fma(ff, dy, fy);
                fz = fma(ff, dz, fz);
                if (ENERGY) {
                    e = fma(s6, fma(Pr.eps4, s6, -Pr.eps4), e);  // 4 eps (s12 - s6)
                    w = fma(ff, r2, w);
                }
            };
#pragma unroll 2
            for (int k = sub; k < words; k += Q) {
                const unsigned int pair = q0;
                q0 = q1;
                q1 = q2;
                q2 = q3;
                q3 = k + 4 * Q < words ? __ldg(row + (long)(k + 4 * Q) * stride) : 0u;
                pair_term(pair & 0xffffu);
                pair_term(pair >> 16);
            }
            for (unsigned int o = 1; o < q; o <<= 1) {
                fx += __shfl_xor_sync(0xffffffffu, fx, o);
                fy += __shfl_xor_sync(0xffffffffu, fy, o);
                fz += __shfl_xor_sync(0xffffffffu, fz, o);
                if (ENERGY) {
                    e += __shfl_xor_sync(0xffffffffu, e, o);
                    w += __shfl_xor_sync(0xffffffffu, w, o);
                }
            }
            if (active && sub == 0) {
                if (DRIFT) {
                    const long vc = D.vcap;
                    double vx = D.v[i] + D.half * fx;
                    double vy = D.v[vc + i] + D.half * fy;
                    double vz = D.v[2 * vc + i] + D.half * fz;
                    ke += 0.5 * D.mass * (vx * vx + vy * vy + vz * vz);
                    vx = vx + D.half * fx;
                    vy = vy + D.half * fy;
                    vz = vz + D.half * fz;
                    double4 x = ld4(D.pos, i);
                    x.x += D.dt * vx;
                    x.y += D.dt * vy;
                    x.z += D.dt * vz;
                    D.v[i] = vx;
                    D.v[vc + i] = vy;
                    D.v[2 * vc + i] = vz;
                    st4(D.pos, i, x);
                    D.sxy_next[i] = make_double2(x.x, x.y);
                    D.sz_next[i] = x.z;
                    const double4 b = ld4(D.xb, i);
                    md2 = fmax(md2, dist2(x.x - b.x, x.y - b.y, x.z - b.z));
                } else {
                    f[i] = fx;
                    f[fcap + i] = fy;
                    f[2 * fcap + i] = fz;
                }
                if (ENERGY) {
                    pe += 0.5 * e;
                    vir += 0.5 * w;
                }
            }
            first += cnt;
        }
    }
    if (ENERGY) {
        pe = block_sum<double, FBLOCK_T>(pe);
        vir = block_sum<double, FBLOCK_T>(vir);
        if (DRIFT) ke = block_sum<double, FBLOCK_T>(ke);
        if (threadIdx.x == 0) {
            if (DRIFT) {
                part[3 * blockIdx.x] = pe;
                part[3 * blockIdx.x + 1] = vir;
                part[3 * blockIdx.x + 2] = ke;
            } else {
                part[2 * blockIdx.x] = pe;
                part[2 * blockIdx.x + 1] = vir;
            }
        }
    }
    if (DRIFT) {
        md2 = block_max<double, FBLOCK_T>(md2);
        if (threadIdx.x == 0) atomic_max_nonneg(D.maxd2, md2);
    }
}

// (x, y) and z of the slots [first, first + n) from the 32-byte records
__global__ void k_split_xyz(const double4* __restrict__ pos, long first, long n, double2* __restrict__ xy,
                            double* __restrict__ zz) {
    for (long k = first + blockIdx.x * (long)blockDim.x + threadIdx.x; k < first + n;
         k += (long)gridDim.x * blockDim.x) {
        const double4 r = ld4(pos, k);
        xy[k] = make_double2(r.x, r.y);
        zz[k] = r.z;
    }
}

// tile-local rows -> global particle indices (for checks and downloads)
__global__ void __launch_bounds__(TBLOCK) k_vtile_translate(long n_real, TileGeom tg,
                                                            const unsigned int* __restrict__ csR,
                                                            const unsigned int* __restrict__ csI,
                                                            const unsigned short* __restrict__ nbr,
                                                            const int* __restrict__ nn, long stride,
                                                            int* __restrict__ out) {
    __shared__ TileSh S;
    tile_layout(tg, blockIdx.x, csR, csI, S);
    const unsigned int ib = S.cR[4][1], ie = S.cR[4][S.ncol - 2];
    const int nc = S.ncol - 1;
    for (unsigned int i = ib + threadIdx.x; i < ie; i += blockDim.x) {
        int m = nn[i];
        for (int k = 0; k < m; ++k) {
            unsigned int l = nbr[pair_slot(k, stride, i)];
            int g = -1;
            for (int r = 0; r < 9; ++r) {
                unsigned int lr = S.cR[r][nc] - S.cR[r][0], li = S.cI[r][nc] - S.cI[r][0];
                if (l >= S.oR[r] && l < S.oR[r] + lr) g = (int)(S.cR[r][0] + (l - S.oR[r]));
                if (l >= S.oI[r] && l < S.oI[r] + li) g = (int)(n_real + S.cI[r][0] + (l - S.oI[r]));
            }
            out[(long)k * stride + i] = g;
        }
    }
}

// ---------------------------------------------------------------------------
// host side

static const int SMEM_LIMIT = 200 * 1024;

int tile_plan(pd_cl cl, long n_real, int TX_req, TileGeom& tg, long& ntiles) {
    tg.gs0 = cl->gs[0];
    tg.gs1 = cl->gs[1];
    tg.gs2 = cl->gs[2];
    tg.pad = cl->pad;
    int nxi = tg.gs0 - 2 * tg.pad;
    int TX = TX_req;
    if (TX <= 0) {
        double cells = (double)cl->div[0] * cl->div[1] * cl->div[2];
        double occ = cells > 0 ? (double)n_real / cells : 1.0;
        TX = (int)(140.0 / (occ > 1e-3 ? occ : 1e-3) + 0.5);
    }
    if (TX < 1) TX = 1;
    if (TX > TXMAX) TX = TXMAX;
    if (TX > nxi) TX = nxi;
    tg.TX = TX;
    tg.ntx = (nxi + TX - 1) / TX;
    tg.ny = tg.gs1 - 2 * tg.pad;
    tg.nz = tg.gs2 - 2 * tg.pad;
    ntiles = (long)tg.ntx * tg.ny * tg.nz;
    if (cl->pad != 1) {
        set_error("tile plan: the tiled list needs one padding layer");
        return PD_EINVAL;
    }
    return PD_OK;
}

int tile_sizes(pd_vd h, const TileGeom& tg, long ntiles, const unsigned int* csR, const unsigned int* csI,
               unsigned int& tmax, unsigned int& cmax, cudaStream_t st) {
    PD_CUDA(cudaMemsetAsync(&h->ctrl->tile_max, 0, 3 * sizeof(unsigned int), st));
    pd::launch(k_tile_sizes, grid_for(ntiles, 256), 256, 0, st, tg, ntiles, csR, csI, &h->ctrl->tile_max,
               &h->ctrl->tile_center_max, &h->ctrl->tile_pass_max);
    PD_LAUNCH_CHECK();
    PD_TRY(read_ctrl(h, st));
    tmax = h->ctrl_h->tile_max;
    cmax = h->ctrl_h->tile_center_max;
    return PD_OK;
}

template <class K> static int allow_smem(K kernel, int bytes) {
    PD_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    return PD_OK;
}

bool tile_fits(pd_vd h, unsigned int tmax) {
    return (long)tmax * h->pos_bytes <= SMEM_LIMIT && tmax <= 65535u;
}

// |d2_f32 - d2| for pairs near r: coordinates rounded to FP32 (relative 2^-24)
// at magnitude <= X, differences and the 3-term sum rounded once more each.
double fp32_band(pd_vd h, double r) {
    double X = 0;
    for (int d = 0; d < 3; ++d)
        X = std::max(X, std::max(std::fabs(h->lo[d] - 2 * h->g[d]), std::fabs(h->hi[d] + 2 * h->g[d])));
    const double u = std::ldexp(1.0, -24);
    double D = 2 * u * X + u * r;                       // per-component error of the FP32 difference
    double e = 2 * std::sqrt(3.0) * r * D + 3 * D * D + 4 * u * (r * r + 1.0);
    return 4 * e;                                       // safety factor 4
}

int tile_build(pd_vd h, const TileGeom& tg, long ntiles, const unsigned int* csR, const unsigned int* csI,
               unsigned int cap, double r_list, Buf& pos32, Buf& nbr, Buf& nn, long& stride, int& max_nn,
               cudaStream_t st) {
    long n = h->n_real;
    stride = ((n + 31) / 32) * 32;
    if (stride < 32) stride = 32;
    long nt = h->n_total;
    PD_TRY(pos32.ensure(sizeof(float4) * (size_t)(nt > 0 ? nt : 1)));
    if (h->dtype == PD_F64)
        pd::launch(k_pos32<double>, grid_for(nt, 256), 256, 0, st, (const double4*)h->pos, nt, pos32.as<float4>());
    else
        pd::launch(k_pos32<float>, grid_for(nt, 256), 256, 0, st, (const float4*)h->pos, nt, pos32.as<float4>());
    PD_LAUNCH_CHECK();
    double band = fp32_band(h, r_list);
    float lo_thr = (float)(r_list * r_list - band), hi_thr = (float)(r_list * r_list + band);
    if (max_nn <= 0) {
        double vol = (h->hi[0] - h->lo[0]) * (h->hi[1] - h->lo[1]) * (h->hi[2] - h->lo[2]);
        double mean = (double)n / vol * 4.18879 * r_list * r_list * r_list;
        max_nn = (int)(mean * 1.5 + 32);
    }
    max_nn = (max_nn + 1) & ~1;  // whole 32-bit words
    // three z-layer passes with a third of the staging (more resident CTAs) when
    // the largest layer is well below the whole tile (the sizes of the tile_sizes
    // call before); a tile of more than two domain particles a thread takes the
    // passes again for the rest
    const unsigned int pcap = h->ctrl_h->tile_pass_max;
    const bool layers = pcap > 0 && 2 * pcap < cap;
    for (int attempt = 0; attempt < 3; ++attempt) {
        int smem = (int)((layers ? pcap : cap) * sizeof(float4));
        if (smem < 16) smem = 16;
        PD_TRY(nbr.ensure(sizeof(unsigned short) * (size_t)stride * max_nn));
        PD_TRY(nn.ensure(sizeof(int) * (size_t)stride));
        PD_CUDA(cudaMemsetAsync(nn.p, 0, sizeof(int) * (size_t)stride, st));
        if (layers && h->dtype == PD_F64) {
            PD_TRY(allow_smem(k_vtile_build3<double>, smem));
            pd::launch(k_vtile_build3<double>, (unsigned)ntiles, TBLOCK, (size_t)smem, st, (const double4*)h->pos,
                       (const float4*)pos32.as<float4>(), n, tg, csR, csI, pcap, r_list * r_list, lo_thr, hi_thr,
                       nbr.as<unsigned int>(), nn.as<int>(), stride, max_nn, &h->ctrl->err, &h->ctrl->nn_max);
        } else if (layers) {
            float rl = (float)r_list;
            PD_TRY(allow_smem(k_vtile_build3<float>, smem));
            pd::launch(k_vtile_build3<float>, (unsigned)ntiles, TBLOCK, (size_t)smem, st, (const float4*)h->pos,
                       (const float4*)pos32.as<float4>(), n, tg, csR, csI, pcap, rl * rl, lo_thr, hi_thr,
                       nbr.as<unsigned int>(), nn.as<int>(), stride, max_nn, &h->ctrl->err, &h->ctrl->nn_max);
        } else if (h->dtype == PD_F64) {
            PD_TRY(allow_smem(k_vtile_build<double>, smem));
            pd::launch(k_vtile_build<double>, (unsigned)ntiles, TBLOCK, (size_t)smem, st, (const double4*)h->pos,
                       (const float4*)pos32.as<float4>(), n, tg, csR, csI, cap, r_list * r_list, lo_thr, hi_thr,
                       nbr.as<unsigned int>(), nn.as<int>(), stride, max_nn, &h->ctrl->err, &h->ctrl->nn_max);
        } else {
            float rl = (float)r_list;
            PD_TRY(allow_smem(k_vtile_build<float>, smem));
            pd::launch(k_vtile_build<float>, (unsigned)ntiles, TBLOCK, (size_t)smem, st, (const float4*)h->pos,
                       (const float4*)pos32.as<float4>(), n, tg, csR, csI, cap, rl * rl, lo_thr, hi_thr,
                       nbr.as<unsigned int>(), nn.as<int>(), stride, max_nn, &h->ctrl->err, &h->ctrl->nn_max);
        }
        PD_LAUNCH_CHECK();
        PD_TRY(read_ctrl(h, st));
        if (h->ctrl_h->err & (ERR_TILE_CAP | ERR_TIMEOUT)) {
            set_error("tiled Verlet build failed (err=0x%x)", h->ctrl_h->err);
            return PD_EOVERFLOW;
        }
        if (!(h->ctrl_h->err & ERR_NN_OVERFLOW)) return PD_OK;
        max_nn = ((int)(h->ctrl_h->nn_max * 1.15 + 8) + 1) & ~1;
        h->ctrl_h->err &= ~ERR_NN_OVERFLOW;
        h->ctrl_h->nn_max = 0;
        PD_CUDA(cudaMemcpyAsync(&h->ctrl->err, &h->ctrl_h->err, sizeof(unsigned int) * 2, cudaMemcpyHostToDevice, st));
    }
    set_error("tiled Verlet build: row capacity did not converge");
    return PD_EOVERFLOW;
}

int tile_split(pd_vd h, Buf& sxy, Buf& sz, long first, long n, cudaStream_t st) {
    const size_t cap = (size_t)(h->cap > 0 ? h->cap : 1);
    PD_TRY(sxy.ensure(cap * sizeof(double2)));
    PD_TRY(sz.ensure(cap * sizeof(double)));
    if (n <= 0) return PD_OK;
    pd::launch(k_split_xyz, grid_for(n, 256), 256, 0, st, (const double4*)h->pos, first, n, sxy.as<double2>(),
               sz.as<double>());
    PD_LAUNCH_CHECK();
    return PD_OK;
}

template <bool E, int P, int MINB, bool DRIFT>
static int launch_lj_xyz_k(pd_vd h, const TileGeom& tg, long ntiles, const unsigned int* csR, const unsigned int* csI,
                           unsigned int cap, const Buf& nbr, const Buf& nn, long stride, const LJP<double>& LP,
                           double* f, double* part, const Buf& sxy, const Buf& sz, const DriftArgs& D,
                           cudaStream_t st) {
    int smem = (int)(cap * 24);
    if (smem < 32) smem = 32;
    const int mwords = (int)std::min<long>((long)(nbr.bytes / (4 * (size_t)stride)), 1L << 30);
    PD_TRY(allow_smem(k_vtile_lj_xyz<E, P, MINB, DRIFT>, smem));
    pd::launch(k_vtile_lj_xyz<E, P, MINB, DRIFT>, (unsigned)ntiles, FBLOCK_T, (size_t)smem, st,
               (const double2*)sxy.as<double2>(), (const double*)sz.as<double>(), h->n_real, tg, csR, csI, cap,
               nbr.as<unsigned int>(), nn.as<int>(), stride, mwords, LP, f, h->cap, part, &h->ctrl->err, D);
    PD_LAUNCH_CHECK();
    return PD_OK;
}

template <bool E, int P, int MINB>
static int launch_lj_xyz(pd_vd h, const TileGeom& tg, long ntiles, const unsigned int* csR, const unsigned int* csI,
                         unsigned int cap, const Buf& nbr, const Buf& nn, long stride, const LJP<double>& LP, double* f,
                         double* part, const Buf& sxy, const Buf& sz, const DriftArgs* drift, cudaStream_t st) {
    if (!sxy.p || !sz.p) {
        set_error("tile_lj: the FP64 staging copies were not made");
        return PD_ESTATE;
    }
    if (!drift) return launch_lj_xyz_k<E, P, MINB, false>(h, tg, ntiles, csR, csI, cap, nbr, nn, stride, LP, f, part,
                                                          sxy, sz, DriftArgs{}, st);
    if (!E || !drift->sxy_next || !drift->sz_next || drift->sxy_next == sxy.as<double2>()) {
        set_error("tile_lj: a drift needs the energy partials and a second pair of staging copies");
        return PD_EINVAL;
    }
    return launch_lj_xyz_k<E, P, MINB, E>(h, tg, ntiles, csR, csI, cap, nbr, nn, stride, LP, f, part, sxy, sz, *drift,
                                          st);
}

// FP32 storage: the 16-byte records
template <class T, bool E, int P>
struct LjLaunch {
    static int run(pd_vd h, const TileGeom& tg, long ntiles, const unsigned int* csR, const unsigned int* csI,
                   unsigned int cap, const Buf& nbr, const Buf& nn, long stride, const LJP<T>& LP, T* f, double* part,
                   const Buf& sxy, const Buf& sz, int smem, const DriftArgs* drift, cudaStream_t st) {
        (void)sxy;
        (void)sz;
        if (drift) {
            set_error("tile_lj: the fused drift is the FP64 path's");
            return PD_EINVAL;
        }
        PD_TRY(allow_smem(k_vtile_lj<T, E, P>, smem));
        pd::launch(k_vtile_lj<T, E, P>, (unsigned)ntiles, FBLOCK_T, (size_t)smem, st,
                   (const typename V4<T>::type*)h->pos, h->n_real, tg, csR, csI, cap, nbr.as<unsigned int>(),
                   nn.as<int>(), stride, LP, f, h->cap, part, &h->ctrl->err);
        PD_LAUNCH_CHECK();
        return PD_OK;
    }
};
// FP64: the split staging (k_vtile_lj_xyz, at most 64 registers: four CTAs per SM)
template <bool E, int P>
struct LjLaunch<double, E, P> {
    static int run(pd_vd h, const TileGeom& tg, long ntiles, const unsigned int* csR, const unsigned int* csI,
                   unsigned int cap, const Buf& nbr, const Buf& nn, long stride, const LJP<double>& LP, double* f,
                   double* part, const Buf& sxy, const Buf& sz, int smem, const DriftArgs* drift, cudaStream_t st) {
        (void)smem;
        return launch_lj_xyz<E, P, 4>(h, tg, ntiles, csR, csI, cap, nbr, nn, stride, LP, f, part, sxy, sz, drift, st);
    }
};

template <class T>
static int tile_lj_t(pd_vd h, const TileGeom& tg, long ntiles, const unsigned int* csR, const unsigned int* csI,
                     unsigned int cap, const Buf& nbr, const Buf& nn, long stride, const pd_lj_params_t& lj, T* f,
                     double* part, bool energy, int P, const Buf& sxy, const Buf& sz, int smem,
                     const DriftArgs* drift, cudaStream_t st) {
    LJP<T> LP{};
    LP.eps24 = (T)(24.0 * lj.eps);
    LP.eps4 = (T)(4.0 * lj.eps);
    LP.sig2 = (T)(lj.sigma * lj.sigma);
    T rc = (T)lj.r_cut;
    LP.rc2 = rc * rc;
#define PD_LJ_CASE(E, PP)                                                                                         \
    if (energy == E && P == PP)                                                                                   \
        return LjLaunch<T, E, PP>::run(h, tg, ntiles, csR, csI, cap, nbr, nn, stride, LP, f, part, sxy, sz, smem, \
                                       drift, st);
    PD_LJ_CASE(true, 1)
    PD_LJ_CASE(true, 2)
    PD_LJ_CASE(true, 4)
    PD_LJ_CASE(false, 1)
    PD_LJ_CASE(false, 2)
    PD_LJ_CASE(false, 4)
#undef PD_LJ_CASE
    set_error("tile_lj: threads per particle must be 1, 2 or 4");
    return PD_EINVAL;
}

int tile_lj(pd_vd h, const TileGeom& tg, long ntiles, const unsigned int* csR, const unsigned int* csI,
            unsigned int cap, const Buf& nbr, const Buf& nn, long stride, const pd_lj_params_t& lj, int force_prop,
            double* part, bool energy, int P, const Buf& sxy, const Buf& sz, cudaStream_t st,
            const DriftArgs* drift) {
    Prop& F = h->props[force_prop];
    int smem = (int)(cap * h->pos_bytes);
    if (smem < 16) smem = 16;
    if (h->dtype == PD_F64)
        return tile_lj_t<double>(h, tg, ntiles, csR, csI, cap, nbr, nn, stride, lj, (double*)F.d, part, energy, P,
                                 sxy, sz, smem, drift, st);
    return tile_lj_t<float>(h, tg, ntiles, csR, csI, cap, nbr, nn, stride, lj, (float*)F.d, part, energy, P, sxy,
                            sz, smem, drift, st);
}

int tile_translate(pd_vd h, const TileGeom& tg, long ntiles, const unsigned int* csR, const unsigned int* csI,
                   const Buf& nbr, const Buf& nn, long stride, int max_nn, int* out_dev, cudaStream_t st) {
    pd::launch(k_vtile_translate, (unsigned)ntiles, TBLOCK, 0, st, h->n_real, tg, csR, csI, nbr.as<unsigned short>(),
               nn.as<int>(), stride, out_dev);
    PD_LAUNCH_CHECK();
    (void)max_nn;
    return PD_OK;
}

}  // namespace pd
