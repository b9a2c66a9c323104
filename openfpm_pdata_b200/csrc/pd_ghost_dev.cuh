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
};

template <class T> __device__ __forceinline__ bool inside_np(const BoxSet<T>& B, int i, T x, T y, T z) {
    return !(x < B.lo[i][0] || x >= B.hi[i][0] || y < B.lo[i][1] || y >= B.hi[i][1] || z < B.lo[i][2] ||
             z >= B.hi[i][2]);
}

// host computation of the domain ghost boxes (pd_ghost.cu)
int ghost_boxes_host(pd_vd h, BoxSet<double>* B, double* shifts27);

}  // namespace pd
