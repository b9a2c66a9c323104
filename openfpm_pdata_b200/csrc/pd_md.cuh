// pd_md.cuh -- the integrator handle, shared by the single-system driver
// (pd_md.cu) and the serving loop (pd_serve.cu).
#pragma once
#include <cstdint>
#include <vector>
#include "pd_internal.cuh"
#include "pd_tile.cuh"

struct pd_md_s {
    pd_vd h = nullptr;
    // the rebuild's reorder swaps the vector's spare storage in (single-system driver;
    // off where device pointers are kept in tables, the serving loop)
    bool swap_reorder = true;
    pd_lj_params_t lj;
    pd_md_params_t mp;
    pd_vl vl = nullptr;   // Verlet list (r_cut + skin)
    pd_cl cl = nullptr;   // cell list of side r_cut (cell-list mode)
    pd::Buf xb, fpart, kpart, E;
    int nblk = 0;
    bool ready = false;
    // tiled neighbour structure (pd_tile.cu)
    bool use_tiles = true;
    int tile_tx = 0;  // cells per tile along x (0: from the mean occupancy)
    int tile_p = 2;   // threads per domain particle in the pair kernel
    int tile_block = pd::FBLOCK_T;  // threads per CTA of the precision form's pair kernel
    bool tiles_active = false;
    pd::TileGeom tg;
    long ntiles = 0;
    unsigned int tcap = 0;
    long tstride = 0;
    int tmax_nn = 0;
    pd::Buf csR, csI, tnbr, tnn, tpart, pos32;
    pd::Buf sxy, sz;  // FP64 tiled path: the pair kernel's (x, y) / z copies of the positions
    pd::Buf sxy2, sz2;  // the second pair, written by a pair kernel that also drifts
    bool drifted = false;  // the last pair kernel made the next step's kick and drift
    // precision form: FP32 cell-local offsets (all particles), their value at the
    // last build (real particles) and the constant parts of the image offsets
    int physics = 0;  // 0: Lennard-Jones, 1: WCSPH
    pd_sph_params_t sp;
    pd::Buf aux, rpart;
    bool mixed = false;
    bool off_valid = false;  // `off` holds the authoritative state (after the first build)
    pd::Buf off, offb, offK;
    long builds = 0, steps = 0;
    // cell-list mode: the captured step graph, its image capacity, the step counter
    cudaGraphExec_t gcl = nullptr;
    cudaStream_t gst = nullptr;
    long gcl_img_cap = 0;
    std::vector<uintptr_t> gcl_key;  // the buffers and sizes the graph captured
    unsigned long long gcl_kernels = 0;
    pd::Buf eidx;
    int cluster_ctas = 0;  // CTAs of the last one-cluster run (0: none so far)
    // optional per-phase device timing (CUDA events on the run's stream)
    bool timing = false;
    std::vector<cudaEvent_t> evp;  // six per step of a timed run, recorded without synchronising
    double ms[4] = {0, 0, 0, 0};   // integrate, rebuild, images, force
    long cnt[4] = {0, 0, 0, 0};
    // the last timed run's events, read when the times are asked for or before the
    // next run records them again (not inside the run)
    std::vector<unsigned char> ev_rebuilt;  // per step of that run: rebuilt or not
};

namespace pd {
int force_blocks(long n);
// wrap, sort, periodic images, neighbour structure (and the mixed-form offsets)
int md_rebuild(pd_md md, cudaStream_t st);
// forces of the current state into the force property (with `drift`, the plain FP64
// tiled path's pair kernel also makes the next step's kick and drift instead)
int md_forces(pd_md md, cudaStream_t st, const DriftArgs* drift = nullptr);
// cell-list mode of a small system: every step of a run in one thread-block cluster (pd_cluster.cu)
bool md_cluster_eligible(pd_md md);
int md_run_cluster(pd_md md, int steps, cudaStream_t st, double* E);
}  // namespace pd
