// pd_tile.cuh -- tiled Verlet structure shared by the integrator (see pd_tile.cu).
#pragma once
#include "pd_internal.cuh"

namespace pd {

static constexpr int TXMAX = 32;   // cells per tile along x, at most
static constexpr int TBLOCK = 128;   // threads per tile CTA of the list build
static constexpr int FBLOCK_T = 256; // threads per tile CTA of the pair kernels

struct TileGeom {
    int gs0, gs1, gs2, pad;
    int TX, ntx, ny, nz;
};

int tile_plan(pd_cl cl, long n_real, int TX_req, TileGeom& tg, long& ntiles);
int tile_sizes(pd_vd h, const TileGeom& tg, long ntiles, const unsigned int* csR, const unsigned int* csI,
               unsigned int& tmax, unsigned int& cmax, cudaStream_t st);
bool tile_fits(pd_vd h, unsigned int tmax);
// bound on |d2_f32 - d2| for pairs near r in the vector's box (FP32 prefilter band of the build)
double fp32_band(pd_vd h, double r);  // FP64/FP32 staging of the pair kernel fits
int tile_build(pd_vd h, const TileGeom& tg, long ntiles, const unsigned int* csR, const unsigned int* csI,
               unsigned int cap, double r_list, Buf& pos32, Buf& nbr, Buf& nn, long& stride, int& max_nn,
               cudaStream_t st);
// The FP64 pair kernel stages (x, y) and z from copies of the positions: those of
// the slots [first, first + n) refreshed from the records (room for the vector's capacity)
int tile_split(pd_vd h, Buf& sxy, Buf& sz, long first, long n, cudaStream_t st);
// The velocity-Verlet update a plain FP64 step makes after its forces, done by the
// pair kernel for each domain particle while the particle's force is in registers:
// the closing half kick of this step (kinetic energy partial), the next step's
// opening half kick and drift (the operations of the separate kick-kick-drift
// kernel, in its order), the drifted position into the vector and into the other
// pair of staging copies (the pair kernel still reads the current ones), and the
// largest |x - x_build|^2 into *maxd2.  The force itself is not stored: the next
// step recomputes it before anything reads it.
struct DriftArgs {
    double4* pos;
    const double4* xb;
    double* v;
    long vcap;
    double half, dt, mass;
    double2* sxy_next;
    double* sz_next;
    unsigned long long* maxd2;
};
// LJ forces from the tiled rows (FP64: from the staging copies sxy / sz, which must be
// current).  Per tile, part receives (pe, vir), or (pe, vir, ke) with a drift.
int tile_lj(pd_vd h, const TileGeom& tg, long ntiles, const unsigned int* csR, const unsigned int* csI,
            unsigned int cap, const Buf& nbr, const Buf& nn, long stride, const pd_lj_params_t& lj, int force_prop,
            double* part, bool energy, int P, const Buf& sxy, const Buf& sz, cudaStream_t st,
            const DriftArgs* drift = nullptr);
int tile_translate(pd_vd h, const TileGeom& tg, long ntiles, const unsigned int* csR, const unsigned int* csI,
                   const Buf& nbr, const Buf& nn, long stride, int max_nn, int* out_dev, cudaStream_t st);

}  // namespace pd
