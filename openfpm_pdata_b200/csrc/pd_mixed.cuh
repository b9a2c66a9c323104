// pd_mixed.cuh -- precision form of the LJ integrator (see pd_mixed.cu).
#pragma once
#include "pd_internal.cuh"
#include "pd_tile.cuh"

namespace pd {

// quantum of the offsets for the grid of `cl` and a list skin (stored in cl->mq):
// the largest power of two q with every value of the pair loop (at most
// 2 * cell side + skin in magnitude) below 2^24 q
double mixed_set_quantum(pd_cl cl, double skin);
int mixed_from_positions(pd_vd h, pd_cl cl, Buf& off, Buf& K, cudaStream_t st);
int mixed_to_positions(pd_vd h, pd_cl cl, const Buf& off, cudaStream_t st);
// positions of the real particles in id order, x,y,z per particle, into `out` (3 n doubles)
int mixed_to_positions_by_id(pd_vd h, pd_cl cl, const Buf& off, double* out, cudaStream_t st);
int mixed_replay(pd_vd h, Buf& off, const Buf& K, cudaStream_t st);
int mixed_kick_drift(pd_vd h, pd_cl cl, Buf& off, const Buf& ob, int vel_prop, int force_prop, int nblk,
                     double half, double dt, cudaStream_t st);
// mixed_kick of one step and mixed_kick_drift of the next in one pass
int mixed_kick_kick_drift(pd_vd h, pd_cl cl, Buf& off, const Buf& ob, int vel_prop, int force_prop, int nblk,
                          double half, double dt, double mass, double* kpart, cudaStream_t st);
int mixed_kick(pd_vd h, int vel_prop, int force_prop, int nblk, double half, double mass, double* kpart,
               cudaStream_t st);
int mixed_lj(pd_vd h, pd_cl cl, const TileGeom& tg, long ntiles, const unsigned int* csR, const unsigned int* csI,
             unsigned int cap, const Buf& off, const Buf& nbr, const Buf& nn, long stride, const pd_lj_params_t& lj,
             int force_prop, double* part, int P, int block, cudaStream_t st);

}  // namespace pd
