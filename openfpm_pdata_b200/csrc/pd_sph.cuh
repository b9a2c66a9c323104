// pd_sph.cuh -- weakly compressible SPH on the tiled neighbour structure (see pd_sph.cu).
#pragma once
#include "pd_internal.cuh"
#include "pd_tile.cuh"

namespace pd {

int sph_pack(pd_vd h, const pd_sph_params_t& sp, int vel_prop, Buf& aux, cudaStream_t st);
int sph_kick_drift(pd_vd h, const pd_sph_params_t& sp, int vel_prop, int acc_prop, const Buf& xb, Buf& aux,
                   int nblk, double dt, cudaStream_t st);
int sph_kick(pd_vd h, const pd_sph_params_t& sp, int vel_prop, int acc_prop, int nblk, double dt, double* kpart,
             double* rpart, cudaStream_t st);
// sph_kick of one step and sph_kick_drift of the next in one pass
int sph_kick_kick_drift(pd_vd h, const pd_sph_params_t& sp, int vel_prop, int acc_prop, const Buf& xb, Buf& aux,
                        int nblk, double dt, double* kpart, double* rpart, cudaStream_t st);
int sph_rates(pd_vd h, const TileGeom& tg, long ntiles, const unsigned int* csR, unsigned int cap, const Buf& nbr,
              const Buf& nn, long stride, const Buf& aux, const pd_sph_params_t& sp, int acc_prop, int P,
              cudaStream_t st);
bool sph_tile_fits(pd_vd h, unsigned int tmax);

}  // namespace pd
