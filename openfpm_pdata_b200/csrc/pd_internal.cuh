// pd_internal.cuh -- shared internals of libpdgpu.so (host structures, device helpers).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pdgpu.h"

namespace pd {

void set_error(const char* fmt, ...);
// PD_OK when p is device (or managed) memory of the current device; else PD_EINVAL
// with a message naming `who` and `what`.  Neither allocates nor synchronises.
int check_device_ptr(const void* p, const char* who, const char* what);

#define PD_CUDA(call)                                                                                   \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess) {                                                                        \
            pd::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_));           \
            return e_ == cudaErrorMemoryAllocation ? PD_ENOMEM : PD_ECUDA;                              \
        }                                                                                               \
    } while (0)

#define PD_LAUNCH_CHECK() PD_CUDA(cudaGetLastError())

#define PD_TRY(expr)             \
    do {                         \
        int r_ = (expr);         \
        if (r_ != PD_OK) return r_; \
    } while (0)

// Device-side error bits (Ctrl::err)
enum : unsigned int {
    ERR_IMG_OVERFLOW = 1u,  // more periodic images than the image capacity
    ERR_NN_OVERFLOW = 2u,   // a Verlet row longer than the list capacity
    ERR_CELL_RANGE = 4u,    // a particle outside the cell grid (clamped)
    ERR_CAP_OVERFLOW = 8u,  // real + images beyond the particle capacity
    ERR_TIMEOUT = 16u,      // a bounded wait on a bulk copy gave up
    ERR_TILE_CAP = 32u,     // a tile's staged neighbourhood exceeded the shared-memory capacity
};

// Control block resident in device memory: sizes that change on the device and
// reductions read back by the host.
struct Ctrl {
    unsigned int n_img;          // periodic images currently stored after the real particles
    unsigned int err;            // ERR_* bits
    unsigned int nn_max;         // longest Verlet row seen by the last build
    unsigned int rebuild;        // rebuild flag of the integrator
    unsigned long long maxdisp2; // bits of the largest squared displacement (non-negative double)
    unsigned long long steps;
    unsigned long long builds;
    unsigned int tile_max;         // largest staged neighbourhood of a tile (records)
    unsigned int tile_center_max;  // largest number of domain particles of a tile
    unsigned int tile_pass_max;    // largest staged z-layer (3 rows) of a tile (records)
    unsigned int n_keep;           // count of the last compaction / index selection
};

// Allocation context: inside an AllocScope, device allocations of the library are
// stream-ordered on `st` from `pool` (see dev_alloc in pd_core.cu).
struct AllocCtx {
    cudaStream_t st;
    cudaMemPool_t pool;
};
extern thread_local AllocCtx* g_alloc_ctx;
extern thread_local bool g_capturing;  // the library is capturing a stream on this thread
struct AllocScope {
    AllocCtx ctx;
    AllocCtx* prev;
    AllocScope(cudaStream_t st, cudaMemPool_t pool) : ctx{st, pool}, prev(g_alloc_ctx) { g_alloc_ctx = &ctx; }
    ~AllocScope() { g_alloc_ctx = prev; }
};
cudaError_t dev_alloc(void** p, size_t b);
void dev_free(void* p);

// Growable device buffer
struct Buf {
    void* p = nullptr;
    size_t bytes = 0;
    int ensure(size_t b);
    void release();
    template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

struct Prop {
    int type = 0;
    int ncomp = 0;
    int esize = 0;
    char* d = nullptr;  // component-major [ncomp][cap]
};

inline int type_size(int t) {
    switch (t) {
        case PD_F32: case PD_I32: case PD_U32: return 4;
        case PD_F64: case PD_I64: return 8;
        default: return 0;
    }
}

// exclusive scan, in place, of nb per-block partial counts (one block); the total to *total_dev
int scan_partials(unsigned int* part, long nb, unsigned int* total_dev, cudaStream_t st);
// exclusive scan of n uint32 values (in may equal out); writes the total to *total_dev
int scan_u32(const unsigned int* in, unsigned int* out, long n, unsigned int* total_dev, Buf& scratch,
             cudaStream_t st);

inline unsigned int grid_for(long n, int block, long cap_blocks = 148L * 64) {
    long g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > cap_blocks) g = cap_blocks;
    return (unsigned int)g;
}

inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Every kernel launch of the library goes through launch(): it counts launches
// (pd_launch_count) so a caller can verify how many native kernels ran.
extern unsigned long long g_launches;
template <typename... KArgs, typename... Args>
inline void launch(void (*k)(KArgs...), dim3 g, dim3 b, size_t smem, cudaStream_t st, Args... args) {
    k<<<g, b, smem, st>>>(args...);
    __atomic_fetch_add(&g_launches, 1ull, __ATOMIC_RELAXED);
}

}  // namespace pd

// ---------------------------------------------------------------------------
// handles
struct pd_vd_s {
    int dtype = PD_F64;
    int pos_bytes = 32;  // per record
    double lo[3], hi[3], g[3];
    int bc[3];
    long n_real = 0;   // ghostMarker
    long n_total = 0;  // real + ghosts
    long cap = 0;      // capacity in particles
    void* pos = nullptr;
    int* gid = nullptr;  // original index of the particle in each slot
    std::vector<pd::Prop> props;
    // periodic images (o_part_loc): source slot and shift id of each ghost
    pd::Buf img_src, img_shift, img_cnt, img_start;
    pd::Buf boxes, box_sv, shifts;  // device copies of the local ghost boxes
    int nbox = 0;
    long n_img = 0;
    bool img_valid = false;
    bool img_gen_order = false;  // images in generation order (ghost_put can fold them)
    bool ghost_pending = false;  // an Ighost_get waits for its ghost_wait
    bool pend_replay = false;
    unsigned long pend_mask = 0;
    int pend_opt = 0;
    pd::Ctrl* ctrl = nullptr;    // device
    pd::Ctrl* ctrl_h = nullptr;  // pinned host mirror
    pd::Buf scan_scratch, tmp, tmp2, red;
    // spare storage of the same capacity: a reorder gathers into it and swaps it in
    // (cl_reorder with swap); allocated on first use, freed with the storage
    void* spare_pos = nullptr;
    int* spare_gid = nullptr;
    std::vector<char*> spare_props;
    long spare_cap = 0;
    long epoch = 0;
    // slab decomposition (pd_slab.cu): the rows of the last labelling, in send
    // order (slot of each row, shift code of each halo row), and the halo
    // received last (from slot halo_base on, while the epoch is halo_epoch)
    pd::Buf slab_idx, slab_shift, slab_flag, slab_off, slab_tot;
    long slab_rows = 0;
    int slab_kind = 0;  // 0 none, 1 map, 2 halo
    double slab_L = 0;
    int slab_axis = 0;
    long halo_base = 0, halo_epoch = -1;
};

struct pd_cl_s {
    pd_vd owner = nullptr;
    double r_cut = 0;
    int opt = 0;
    int nn_box = 1;
    double enlarge = 1.013f;
    int pad = 1;
    int div[3], gs[3];
    double box_lo[3], spacing[3];
    long ncells = 0;
    pd::Buf cell_start, cell_cnt, sorted, sorted_tmp, cell_of, slot, dom_sort, flags;
    long n_part = 0;
    long ghost_marker = 0;
    bool reordered = false;  // the vector holds cell-ordered data until restore_order
    unsigned long reordered_mask = 0;
    long epoch = -1;
    double mq = 0;  // quantum of the precision form's offsets on this grid (mixed_set_quantum; 0: unset)
};

struct pd_vl_s {
    pd_vd owner = nullptr;
    double r_cut = 0;
    pd_cl cl = nullptr;  // internal cell list (side r_cut)
    pd::Buf nbr, nn;     // nbr[k*stride + i], nn[i]
    long stride = 0;
    int max_nn = 0;
    long n_dom = 0;
    long epoch = -1;
    bool sym = false;  // half list (VL_SYMMETRIC): each pair once, see verlet_build
};

// ---------------------------------------------------------------------------
// internal host API shared between translation units
namespace pd {
int ensure_capacity(pd_vd h, long need, cudaStream_t st);
// storage of `cap` particles in the vector's layout (positions, ids, every property);
// PD_ENOMEM (nothing held) on failure
int alloc_storage(pd_vd h, long cap, void** pos, int** gid, std::vector<char*>& props);
void free_storage(void* pos, int* gid, const std::vector<char*>& props);
int set_ctrl_n_img(pd_vd h, long n_img, cudaStream_t st);
int read_ctrl(pd_vd h, cudaStream_t st);
int cl_geometry(pd_cl cl, pd_vd h, double r_cut, double enlarge, int nn_box);
// counting sort of the particles [first, first + n_part) (ids relative to `first`)
int cl_build(pd_vd h, pd_cl cl, long n_part, const unsigned int* n_part_dev, cudaStream_t st, long first = 0);
// gather src[ids[k]] -> dst[k] for k < n of 4/8/16/32-byte elements (dst may not alias src)
int gather_bytes(const void* src, void* dst, const int* ids, long n, int esize, cudaStream_t st);
// Further outputs of the reorder of FP64 positions into spare storage: the reordered
// records also to `xb` and as (x, y) / z copies to `sxy` / `sz` (room for n_part);
// *done tells whether they were written (not by the in-place reorder)
struct ReorderExtra {
    double4* xb;
    double2* sxy;
    double* sz;
};
int cl_reorder(pd_vd h, pd_cl cl, long n_part, unsigned long prop_mask, bool with_pos, bool with_gid,
               cudaStream_t st, bool swap = false, const ReorderExtra* extra = nullptr, bool* done = nullptr);
int ghost_boxes_upload(pd_vd h, cudaStream_t st);
int ghost_generate(pd_vd h, long img_cap, bool sync_count, cudaStream_t st);
int ghost_replay(pd_vd h, unsigned long prop_mask, bool with_pos, const unsigned int* n_img_dev, long n_img_bound,
                 cudaStream_t st);
int verlet_build(pd_vd h, pd_vl vl, long n_dom, const unsigned int* n_img_dev, cudaStream_t st, bool check);
int wrap_positions(pd_vd h, long n, cudaStream_t st);
}  // namespace pd
