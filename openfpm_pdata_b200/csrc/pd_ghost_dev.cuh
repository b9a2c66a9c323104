// pd_ghost_dev.cuh -- the local periodic ghost boxes in device memory, shared by
// ghost_get (pd_ghost.cu) and the batched rebuild of the serving loop (pd_serve.cu).
#pragma once
#include "pd_device.cuh"
#include "pd_internal.cuh"

namespace pd {

static constexpr int MAXBOX = 64;

template <class T> struct BoxSet {
    T lo[MAXBOX][3];
    T hi[MAXBOX][3];
    int sv[MAXBOX];
    int nb;
    // core [clo, chi): a region every box misses on some axis (checked on the host
    // when core is set), so a particle inside it has no image
    T clo[3], chi[3];
    int core;
};

// the particle lies in the core: no box contains it (a box missing the core on
// axis d has hi <= clo[d] or lo >= chi[d] there, which excludes every core point)
template <class T> __device__ __forceinline__ bool in_core(const BoxSet<T>& B, T x, T y, T z) {
    return B.core && x >= B.clo[0] && x < B.chi[0] && y >= B.clo[1] && y < B.chi[1] && z >= B.clo[2] &&
           z < B.chi[2];
}

template <class T> __device__ __forceinline__ bool inside_np(const BoxSet<T>& B, int i, T x, T y, T z) {
    return !(x < B.lo[i][0] || x >= B.hi[i][0] || y < B.lo[i][1] || y >= B.hi[i][1] || z < B.lo[i][2] ||
             z >= B.hi[i][2]);
}

// host computation of the domain ghost boxes (pd_ghost.cu)
int ghost_boxes_host(pd_vd h, BoxSet<double>* B, double* shifts27);

}  // namespace pd
