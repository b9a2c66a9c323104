/*
 * pdgpu.h -- C ABI of libpdgpu.so, a B200-native (sm_100a) drop-in for the
 * single-process GPU particle path of OpenFPM pdata's vector_dist.
 *
 * Every entry point takes plain pointers and sizes, returns an int status
 * (PD_OK or a negative PD_E* code, never throws across the ABI) and, where it
 * launches GPU work, a caller-provided CUDA stream passed as `void*`
 * (NULL = the legacy default stream).  Host buffers are caller-owned; device
 * storage is owned by the handles.  Each declaration names the reference
 * interface it replaces (file:line inside the openfpm_pdata project).
 *
 * Positions cross the ABI as AoS xyz triples (Point<3,St>); properties as
 * component-major arrays (component c of particle i at [c*n + i]).
 */
#ifndef PDGPU_H
#define PDGPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define PD_OK 0
#define PD_EINVAL (-1)    /* bad argument (the reference: ACTION_ON_ERROR under SE_CLASS1) */
#define PD_ENOMEM (-2)    /* device allocation failed */
#define PD_ECUDA (-3)     /* a CUDA call failed; pd_last_error() has the text */
#define PD_ESTALE (-4)    /* handle built for an older decomposition / particle set */
#define PD_ETIMEOUT (-5)  /* a bounded device wait gave up */
#define PD_EOVERFLOW (-6) /* a device-side capacity was exceeded; the result is void */
#define PD_ESTATE (-7)    /* call out of order (e.g. restore_order without a reorder) */
#define PD_EIO (-8)       /* a file could not be written / read, or is not of the expected format */

/* ---- value types -------------------------------------------------------- */
#define PD_F32 1
#define PD_F64 2
#define PD_I32 3
#define PD_U32 4
#define PD_I64 5

/* boundary conditions: same values as the reference (NON_PERIODIC, PERIODIC) */
#define PD_NON_PERIODIC 0
#define PD_PERIODIC 1

/* ghost_get / map options, same values as the reference
 * (Vector/cuda/vector_dist_comm_util_funcs.cuh:13-15, util/common_pdata.hpp:12-13) */
#define PD_NO_POSITION 1
#define PD_WITH_POSITION 2
#define PD_NO_CHANGE_ELEMENTS 4
#define PD_SKIP_LABELLING 512
#define PD_KEEP_PROPERTIES 512
#define PD_RUN_ON_DEVICE 1024

/* cell-list options (CL_* of openfpm_data; values are this library's own).
 * PD_CL_SYMMETRIC: getCellListSym (vector_dist.hpp:1062-1066) -- pair kernels
 * through it visit each pair once and put the reaction on the partner, ghosts
 * included; pd_ghost_put(PD_PUT_ADD) folds the ghosts' share onto the sources. */
#define PD_CL_SYMMETRIC 1
#define PD_CL_NON_SYMMETRIC 2
#define PD_CL_GPU_REORDER_POSITION 64
#define PD_CL_GPU_REORDER_PROPERTY 128
#define PD_CL_GPU_REORDER (PD_CL_GPU_REORDER_POSITION | PD_CL_GPU_REORDER_PROPERTY)

/* ghost_put merge operations (add_, max_, replace_ of the reference) */
#define PD_PUT_ADD 1
#define PD_PUT_MAX 2
#define PD_PUT_REPLACE 3

/* writer options of pd_write / pd_write_frame (VTK_WRITER, CSV_WRITER, FORMAT_BINARY
 * of the reference; values are this library's own) */
#define PD_VTK_WRITER 0
#define PD_CSV_WRITER 1
#define PD_FORMAT_BINARY 2

/* comparisons of pd_get_indexes_by_type (the functor::check of the reference) */
#define PD_CMP_EQ 0
#define PD_CMP_NE 1
#define PD_CMP_LT 2
#define PD_CMP_LE 3
#define PD_CMP_GT 4
#define PD_CMP_GE 5

/* reductions (reduce_local<prp,_add_/_max_>) */
#define PD_RED_ADD 1
#define PD_RED_MAX 2

typedef struct pd_vd_s* pd_vd; /* vector_dist_gpu<3,St,aggregate<...>>          */
typedef struct pd_cl_s* pd_cl; /* CellList_gpu<3,St,CudaMemory,shift_only<3,St>> */
typedef struct pd_vl_s* pd_vl; /* VerletList<3,St,VL_NON_SYMMETRIC,...>         */
typedef struct pd_md_s* pd_md; /* velocity-Verlet LJ driver bound to a vector   */

/* Kernel view of a vector (vector_dist_ker, Vector/vector_dist_kernel.hpp:57-305):
 * non-owning device pointers, invalid after any call that can reallocate
 * (map, ghost_get, resize); `epoch` increments on every such call. */
typedef struct {
    void* pos;          /* float4 / double4 records (x, y, z, unused)       */
    void* prop[16];     /* component-major property arrays, stride `stride` */
    int prop_type[16];
    int prop_ncomp[16];
    int n_prop;
    int dtype;
    long stride;        /* allocated capacity in particles                  */
    long size_local;    /* ghostMarker: real particles are [0, size_local)  */
    long size;          /* real + ghost particles                           */
    long epoch;
} pd_view_t;

/* Kernel view of a cell list (CellList_gpu::toKernel): the grid and the
 * counting-sort result. */
typedef struct {
    const int* cell_start;  /* ncells + 1 offsets into sorted_ids            */
    const int* sorted_ids;  /* particle index of each sorted slot            */
    const int* dom_sort_ids;/* sorted slot of each domain particle, in order  */
    long ncells;
    int gs[3];              /* cells per dimension including padding         */
    int div[3];
    int pad;
    int nn_box;             /* NNIteratorBox layers                          */
    double box_lo[3];
    double spacing[3];
    long ghost_marker;
    long n_part;
} pd_cl_view_t;

/* launch shape of getDomainIteratorGPU (vector_dist.hpp:1958-1965) */
typedef struct {
    unsigned int wthr[3];
    unsigned int thr[3];
} pd_launch_t;

/* LJ 12-6 parameters */
typedef struct {
    double eps, sigma, r_cut;
} pd_lj_params_t;

/* integrator precision */
#define PD_PREC_FP64 0  /* positions, velocities, forces in the vector's dtype */
#define PD_PREC_MIXED 1 /* FP32 cell-local positions and pair math, Kahan sums, FP64 wrap and energies */

/* velocity-Verlet parameters */
typedef struct {
    double dt, mass, skin;
    int vel_prop;   /* property id holding velocities (3 comps; PD_F32 in the mixed form) */
    int force_prop; /* property id receiving forces   (3 comps; PD_F32 in the mixed form) */
    int use_cell_list; /* 1: force from the cell list every step (no Verlet list) */
    int precision;     /* PD_PREC_FP64 or PD_PREC_MIXED (the vector must then be PD_F64) */
} pd_md_params_t;

/* weakly compressible SPH parameters (cubic spline of support 2h, Tait EOS,
 * Monaghan artificial viscosity, gravity along z); property ids of the vector */
typedef struct {
    double h, mass, c0, rho0, alpha, gz;
    int rho_prop;  /* density (1 comp, dtype of the vector)            */
    int drho_prop; /* density rate (1 comp, dtype of the vector)       */
    int type_prop; /* PD_I32: 0 fluid, 1 fixed wall particle           */
} pd_sph_params_t;

/* ---- library ------------------------------------------------------------ */
const char* pd_last_error(void);
/* number of CUDA kernels this library has launched so far (all handles) */
unsigned long long pd_launch_count(void);
/* Device blocks freed by the library (outside the serving loop) are cached for
 * reuse up to a limit (4 GiB by default): pd_empty_cache returns them to the
 * driver; pd_set_cache_limit sets the limit (bytes < 0: unchanged) and reports
 * the bytes held.  No counterpart in the reference package (its device memory
 * comes from a dependency's allocator). */
int pd_empty_cache(void);
/* Halo selection of a slab decomposition (one sub-domain per rank): of the n
 * positions x [n][3] (double, device memory), the ascending indices i with
 * x[i][axis] < lo_thr (to the lower neighbour) and with x[i][axis] >= hi_thr (to
 * the upper one), written to idx_lo / idx_hi (device or host, room for n each),
 * their counts to *n_lo / *n_hi.  The reference selects the particles of each
 * neighbouring sub-domain's ghost box (vector_dist_comm.hpp:1398-1596). */
int pd_slab_halo(const double* x, long n, int axis, double lo_thr, double hi_thr, int* idx_lo, int* idx_hi,
                 long* n_lo, long* n_hi, void* stream);
int pd_set_cache_limit(long bytes, long* held);
int pd_device_info(int* sm_count, long* free_bytes, long* total_bytes);

/* ---- vector_dist -------------------------------------------------------- */
/* vector_dist(size_t np, Box<dim,St> box, const size_t (&bc)[dim], const Ghost<dim,St>& g)
 * -- Vector/vector_dist.hpp:498-518.  dim must be 3; ghost is per dimension. */
int pd_create(int dim, int dtype, long n, const double* lo, const double* hi, const int* bc,
              const double* ghost, int opts, pd_vd* out);
int pd_destroy(pd_vd h);
/* aggregate<...> property list: append one property of `ncomp` components */
int pd_add_prop(pd_vd h, int type, int ncomp, int* prop_id);
/* size_local / size_local_with_ghost -- vector_dist.hpp:559-572 */
int pd_size(pd_vd h, long* size_local, long* size_with_ghost);
/* resize of the local part (drops ghosts) -- vector_dist.hpp:923-984 add/resize */
int pd_resize(pd_vd h, long n);
/* hostToDevicePos / deviceToHostPos -- vector_dist.hpp:2984-3030; host AoS xyz in
 * the vector's dtype, particles [offset, offset+count).  These four copies also
 * take a device pointer (unified addressing picks the direction), so device
 * arrays of another library are read and written without a host round trip. */
int pd_h2d_pos(pd_vd h, const void* host_xyz, long offset, long count, void* stream);
int pd_d2h_pos(pd_vd h, void* host_xyz, long offset, long count, void* stream);
/* hostToDeviceProp<prp> / deviceToHostProp<prp>; host component-major [ncomp][count] */
int pd_h2d_prop(pd_vd h, int prop, const void* host, long offset, long count, void* stream);
int pd_d2h_prop(pd_vd h, int prop, void* host, long offset, long count, void* stream);
/* map(RUN_ON_DEVICE) on one process -- vector_dist.hpp:2158-2176 ->
 * vector_dist_comm.hpp:1405-1437 -> apply_bc_each_part (vector_dist_cuda_funcs.cuh:45-53):
 * drops the ghost and wraps every periodic coordinate with periodic_l. */
int pd_map(pd_vd h, int opt, void* stream);
/* ghost_get<prp...>(opt) on one process -- vector_dist.hpp:2203-2231 ->
 * vector_dist_comm.hpp:1754-1829, 734-795: periodic images of the real particles,
 * appended after ghostMarker, particle-major with shift ids ascending, all
 * properties copied.  opt & PD_SKIP_LABELLING replays the stored image list
 * (process_ghost_particles_local, vector_dist_cuda_funcs.cuh:133-155); with
 * PD_NO_POSITION only properties are refreshed.  prop_mask selects the
 * properties copied on a replay (bit p = property p; ~0 = all). */
int pd_ghost_get(pd_vd h, unsigned long prop_mask, int opt, void* stream);
/* Ighost_get<prp...>(opt) / ghost_wait() -- vector_dist.hpp:2241-2291: the ghost
 * exchange enqueued on `stream` without a host synchronisation (images written
 * into the storage's spare room, sized from the previous count with a margin);
 * ghost_wait reads the image count (one synchronisation) and, if the room was too
 * small, redoes the exchange synchronously.  Between the two calls the vector's
 * sizes are not final: make no other call on it. */
int pd_ighost_get(pd_vd h, unsigned long prop_mask, int opt, void* stream);
int pd_ghost_wait(pd_vd h, void* stream);
/* the (source, shift id) record of every ghost (o_part_loc) */
int pd_ghost_records(pd_vd h, int* src, int* shift_id, long cap, long* n_img);
/* ghost_put<op, prp...>(opt) on one process -- vector_dist.hpp:2304-2310 ->
 * vector_dist_comm.hpp:2086-2182 (local part merge_prp_v): the values of every
 * ghost are merged onto its source with op (PD_PUT_ADD / _MAX / _REPLACE), the
 * ghosts of a source in image order.  Needs the images of the last ghost_get
 * (PD_ESTATE otherwise).  prop_mask: bit p = property p. */
int pd_ghost_put(pd_vd h, unsigned long prop_mask, int op, void* stream);
/* explicit box-list image kernels, the reference's num_shift_ghost_each_part +
 * scan + shift_ghost_each_part (vector_dist_cuda_funcs.cuh:157-233) on caller
 * data: boxes [nb][2][3] (lo, hi), sv[nb] shift ids sorted ascending, shifts[..][3].
 * Device pointers; counts[n] out; images written after `n` in pos/prop arrays. */
int pd_ghost_count_boxes(pd_vd h, const double* boxes_host, const int* sv_host, int nb, int* counts_host,
                         void* stream);
int pd_ghost_get_boxes(pd_vd h, const double* boxes_host, const int* sv_host, int nb,
                       const double* shifts_host, int n_shifts, void* stream);
/* toKernel() -- vector_dist.hpp:2961-2966 */
int pd_view(pd_vd h, pd_view_t* out);
/* getDomainIteratorGPU(n_thr) / getDomainAndGhostIteratorGPU -- vector_dist.hpp:1958-1979 */
int pd_domain_iterator(pd_vd h, int n_thr, int with_ghost, pd_launch_t* out);
/* reduce_local<prp,_add_/_max_> -- vector_dist_cuda_funcs.cuh:247-270 (component `comp`) */
int pd_reduce(pd_vd h, int prop, int comp, int op, void* stream, double* out);
/* remove_marked<prp>(vd) -- vector_dist_cuda_funcs.cuh:333-412: removes the
 * domain particles whose property `prop` (component 0; int, unsigned, float,
 * double or int64) is non-zero, keeping the order of the others, and drops the
 * ghosts.  Destructive on `prop` like the reference: it holds 1 on the kept
 * particles afterwards (and on every particle when none was marked). */
int pd_remove_marked(pd_vd h, int prop, void* stream);
/* get_indexes_by_type<prp, functor>(vd, ids, end, ctx) -- vector_dist_cuda_funcs.cuh:449-481:
 * the ascending indexes p < end (end < 0: the domain size) whose property `prop`
 * (component 0) compares `cmp` (PD_CMP_*) to `value` -- the functor::check of the
 * reference as a comparison.  `ids` (device or host memory, room for `cap`)
 * receives them; *n_out their count (PD_EOVERFLOW if above cap). */
int pd_get_indexes_by_type(pd_vd h, int prop, int cmp, long long value, long end, unsigned int* ids, long cap,
                           long* n_out, void* stream);
/* Failure detection of the bounded device waits (no reference counterpart): runs
 * the tile kernels' staging pattern -- an mbarrier armed for one 16-byte
 * cp.async.bulk copy, then a wait of at most `limit` polls -- on one CTA.  With
 * issue_copy the copy completes the phase: PD_OK and out4 = in4.  Without it
 * nothing completes the phase: the wait gives up, the kernel records the timeout
 * and returns, and the call returns PD_ETIMEOUT with the context still usable. */
int pd_selftest_wait(long limit, int issue_copy, const float* in4, float* out4);
/* Measured vector FMA throughput of this GPU in TFLOP/s (an FMA counts two flops),
 * FP32 or FP64: the denominator of the pair kernels' arithmetic roofline. */
int pd_measure_fma_rate(int dtype, double* tflops);
/* save(filename) / load(filename) -- vector_dist.hpp:2459-2476: the domain
 * particles (positions, global ids, properties) in this library's own binary
 * checkpoint format (checksummed); load replaces the particles of a vector of
 * the same dtype whose property list is the file's or empty (then added).
 * Synchronous; PD_EIO on a file error or a corrupt/foreign file. */
int pd_save(pd_vd h, const char* path);
int pd_load(pd_vd h, const char* path);
/* write(out, meta_info, opt) / write_frame(out, iteration, meta_info, opt) --
 * vector_dist.hpp:2498-2721: VTK XML PolyData `<out>_0.vtp` (`<out>_0_<it>.vtp`;
 * PD_FORMAT_BINARY for base64 binary arrays) or CSV `<out>_0.csv` with
 * PD_CSV_WRITER.  meta "name = value" becomes a FieldData value.  Domain only. */
int pd_write(pd_vd h, const char* out, const char* meta, int opt);
int pd_write_frame(pd_vd h, const char* out, long iteration, const char* meta, int opt);
/* the original index of every particle in its current storage slot */
int pd_d2h_gid(pd_vd h, long* host, long offset, long count, void* stream);

/* ---- cell list ---------------------------------------------------------- */
/* getCellListGPU<CellList_gpu<...>>(r_cut, opt, NNIteratorBox, no_se3, ghostEnlargeFactor)
 * -- vector_dist.hpp:1222-1260 (geometry only; nothing is binned yet) */
int pd_celllist_create(pd_vd h, double r_cut, int opt, int nn_box, double enlarge_factor, pd_cl* out);
int pd_celllist_destroy(pd_cl cl);
/* updateCellListGPU<prp...>(cl) -- vector_dist.hpp:1334-1401: cell hash, warp-aggregated
 * counting sort (stable), and with PD_CL_GPU_REORDER a coalesced reorder of the
 * positions / the properties in prop_mask into cell order. */
int pd_celllist_update(pd_vd h, pd_cl cl, unsigned long prop_mask, void* stream);
/* restoreOrder<prp...>(cl) -- vector_dist.hpp:3042-3049: positions, the properties
 * in prop_mask and every property the update reordered return to the original order */
int pd_restore_order(pd_vd h, pd_cl cl, unsigned long prop_mask, void* stream);
int pd_celllist_view(pd_cl cl, pd_cl_view_t* out);
/* download: cell_start[ncells+1], sorted_ids[n] (NULL to skip either) */
int pd_celllist_get(pd_cl cl, int* cell_start, int* sorted_ids, void* stream);
/* the reference's test functor calculate_force / calculate_force_sort
 * (Vector/cuda/vector_dist_gpu_unit_tests.cu:46-119) as a device kernel:
 * out_prop(p) = sum over getNNIteratorBox q != p of in_prop(q)*(xq-xp)/|xq-xp| */
int pd_test_force(pd_vd h, pd_cl cl, int in_prop, int out_prop, int sorted, void* stream);

/* No counterpart in the reference.  The counting sort of pd_celllist_update for
 * callers that cannot allocate device memory: plugins in hosts whose device
 * memory belongs to the host's own pool, and callers that must not let
 * cudaMalloc/cudaFree synchronise the device under running work.  It
 * calls no allocator; its only scratch is a fixed static device array (about
 * 8.4 MB, held on every GPU that loads the library until exit).  Inputs and
 * outputs are caller-owned device buffers: pos_xyz [n][3] in dtype, cell_start
 * [gs0*gs1*gs2 + 1], sorted_ids [n]; the results equal pd_celllist_update's
 * for the same positions and grid (box_lo, spacing, gs including `pad`
 * padding layers).  Limits: n <= 524288 particles and gs0*gs1*gs2 <= 524288
 * cells, else PD_EINVAL.  The first call on each device looks up the scratch
 * address (cudaGetSymbolAddress) and should come before any stream capture.
 * All calls share the scratch: calls that overlap on the GPU race.  The three
 * buffers must be device memory of the current device (else PD_EINVAL, before
 * any launch).  A NaN or out-of-grid position is clamped into a border cell, as
 * pd_celllist_update does (which reports it as PD_EOVERFLOW); here the optional
 * device word `status` (NULL to skip) is cleared and then receives
 * PD_STATIC_OUT_OF_GRID, readable once the stream's work is done. */
#define PD_STATIC_OUT_OF_GRID 1u
int pd_celllist_build_static(int dtype, const void* pos_xyz, long n, const double* box_lo, const double* spacing,
                             const int* gs, int pad, int* cell_start, int* sorted_ids, unsigned int* status,
                             void* stream);

/* ---- Verlet list -------------------------------------------------------- */
/* getVerlet(r_cut) -- vector_dist.hpp:1514-1547: full list of every domain particle
 * over domain + ghost within r_cut (self included), built from a cell list of
 * side r_cut on the domain enlarged by the ghost magnified 1.013. */
int pd_verlet_create(pd_vd h, double r_cut, pd_vl* out);
/* getVerletSym(r_cut) -- vector_dist.hpp:1412-1416: symmetric (half) list, each
 * interacting pair once: a domain partner q of p iff q > p, a ghost iff it lies
 * after p in (x, y, z) lexicographic order (the mirror pair across the periodic
 * boundary is then kept by the other particle).  Forces from it (pd_lj_forces)
 * land on ghosts too; pd_ghost_put(PD_PUT_ADD) folds them onto their sources. */
int pd_verlet_create_sym(pd_vd h, double r_cut, pd_vl* out);
int pd_verlet_destroy(pd_vl vl);
/* updateVerlet(vl, r_cut) -- vector_dist.hpp:1556-1620 */
int pd_verlet_update(pd_vd h, pd_vl vl, void* stream);
/* download as CSR: counts[n] (and idx[sum counts] if non-NULL) */
int pd_verlet_get(pd_vl vl, int* counts, int* idx, long idx_cap, void* stream);

/* ---- pair kernels ------------------------------------------------------- */
/* LJ forces of the domain particles from a Verlet list (vl) or a cell list (cl);
 * writes force_prop (3 comps); returns sum PE and sum virial in energy[2] (FP64). */
int pd_lj_forces(pd_vd h, pd_vl vl, pd_cl cl, const pd_lj_params_t* lj, int force_prop, void* stream,
                 double* energy);

/* the reciprocal used by the pair kernels (Newton-Raphson on the hardware
 * approximation), evaluated on n host values -- a self-test of its error bound */
int pd_selftest_recip(int dtype, const void* x_host, void* out_host, long n);

/* ---- velocity-Verlet LJ driver ------------------------------------------ */
/* Binds a vector holding real particles (no ghost) to an integrator that keeps
 * the particles in cell order, periodic images and a skin Verlet list on the
 * device; rebuilds when the largest displacement since the last build exceeds
 * skin/2 (skin <= 0: every step). */
int pd_md_create(pd_vd h, const pd_lj_params_t* lj, const pd_md_params_t* md, pd_md* out);
int pd_md_destroy(pd_md md);
/* WCSPH driver on the same integrator (no reference counterpart; the reference's
 * pair-functor pattern is vector_dist_gpu_unit_tests.cu:46-119): kick-drift-kick
 * of velocity and density, fluid particles move, wall particles are fixed and
 * their density evolves.  mp: dt, skin, vel_prop, force_prop (= acceleration);
 * the box must be non-periodic.  pd_md_run's E then holds KE of the fluid,
 * sum of densities, 0, rebuilt. */
int pd_sph_create(pd_vd h, const pd_sph_params_t* sp, const pd_md_params_t* mp, pd_md* out);
/* run `steps` steps; E (if non-NULL) receives [steps][4] = KE, PE, virial, rebuilt */
int pd_md_run(pd_md md, int steps, void* stream, double* E);
/* statistics: builds so far, steps so far, device-side error word */
int pd_md_stats(pd_md md, long* builds, long* steps, int* err);
/* per-phase device time (CUDA events on the run's stream, recorded without a
 * synchronisation and read when pd_md_timers is called or the next run starts):
 * ms/counts[4] = integrate, rebuild, image refresh, force (on the plain FP64 tiled
 * path the pair kernel also makes the next step's kick and drift, so "force" holds
 * them and "integrate" the energies); enabling resets them */
int pd_md_set_timing(pd_md md, int on);
/* neighbour structure of the driver: tiled shared-memory rows (on, default) or
 * global-index rows; tx = cells per tile along x (0 = from the mean occupancy),
 * threads_per_particle = 1, 2 or 4 lanes sharing one row (0 = 2) */
int pd_md_set_tiles(pd_md md, int on, int tx, int threads_per_particle);
/* threads per CTA (256 or 128) of the precision form's pair kernel (no reference counterpart) */
int pd_md_set_block(pd_md md, int threads);
/* the driver's Verlet rows as CSR of global particle indices (current storage
 * order: real particles then images); *tiled tells which structure is active */
int pd_md_verlet_get(pd_md md, int* counts, int* idx, long idx_cap, int* tiled);
/* Verlet rows of the last build: domain particles, mean and longest row */
int pd_md_list_stats(pd_md md, long* n_dom, double* mean_nn, int* max_nn);
int pd_md_timers(pd_md md, double* ms, long* counts);
/* launch shape of the driver's kernels: CTAs of the one-cluster run of a small
 * cell-list system (16, or 8 where the GPU cannot place 16; 0 before such a run),
 * and the tile width in cells and lanes per particle of the tiled rows of the last
 * build (0 and 0 without them) */
int pd_md_launch_shape(pd_md md, int* cluster_ctas, int* tile_tx, int* threads_per_particle);

/* ---- serving loop -------------------------------------------------------- */
/* Many independent periodic LJ systems (precision form, FP32 forces / FP64
 * energies) resident on one GPU and stepped together by persistent batched
 * kernels captured as CUDA graphs.  No reference counterpart: the reference's
 * many-systems idiom is an array of kernel views passed to one kernel
 * (Vector/cuda/vector_dist_gpu_MP_tests.cu:427-781).  Requests are admitted in
 * FIFO order as slots and HBM (budget and free memory) allow; each tick advances
 * every admitted system by one velocity-Verlet step and retires finished ones. */
typedef struct pd_srv_s* pd_srv;
int pd_srv_create(long hbm_budget_bytes, int max_slots, const pd_lj_params_t* lj, double dt, double skin,
                  pd_srv* out);
int pd_srv_destroy(pd_srv s);
/* autotune != 0: the force kernel's launch shape (tile width, lanes per particle
 * 1/2/4, threads per CTA 256/128) chosen per size bucket (floor(log2 N)) by timing
 * the single-system kernel on the first system of the bucket; else the fixed shape
 * (tx 0: the width from the occupancy) */
int pd_srv_set_tuning(pd_srv s, int autotune, int tx, int lanes, int block);
/* the shape of one size bucket set by the caller (used as if tuned, with or without autotune) */
int pd_srv_set_shape(pd_srv s, int bucket, int tx, int lanes, int block);
/* queue a system: n particles in a periodic cube of side `box`, host AoS x, v */
int pd_srv_submit(pd_srv s, long n, double box, const double* x_host, const double* v_host, int steps,
                  long* ticket);
int pd_srv_tick(pd_srv s, int* n_active, int* n_queued);
/* 0 queued, 1 running, 2 done, 3 failed */
int pd_srv_state(pd_srv s, long ticket, int* state);
/* final positions (submission order), E[steps][4] = KE, PE, virial, rebuilt;
 * times[3] = submit, admit, done (seconds since the server was created) */
int pd_srv_result(pd_srv s, long ticket, double* x_out, double* E_out, double* times);
int pd_srv_release(pd_srv s, long ticket);
int pd_srv_stats(pd_srv s, long* particle_steps, long* systems_done, long* ticks, long* rebuilds, double* tune_ms);
/* autotuner table: size bucket (floor(log2 N)) -> tile width, lanes per particle, threads per CTA */
int pd_srv_tuned(pd_srv s, int* buckets, int* widths, int* lanes, int* blocks, int cap, int* n);
/* tickets finished (done or failed) since the last call, oldest first, at most
   `cap`; the rest stay for the next call */
int pd_srv_completed(pd_srv s, long* tickets, int cap, int* n);
/* host wall time (ms) spent in: admission, the slot reset part of admission, the
   batched step graphs (launch to completion), retirement */
int pd_srv_timers(pd_srv s, double ms[4]);

/* ---- slab decomposition over ranks (one sub-domain per rank) -------------
 * The reference decomposes the box into sub-domains (Decomposition/
 * CartDecomposition.hpp), sends every particle to the sub-domain owning it
 * (map, vector_dist_comm.hpp:1957-2014) and copies to each neighbouring
 * sub-domain the particles in its ghost (ghost_get, vector_dist_comm.hpp:
 * 1398-1596), over MPI.  Here a sub-domain is the slab r of `nslabs` along
 * `axis` (rank r owns [lo + r w, lo + (r + 1) w), w = (hi - lo) / nslabs, the
 * last slab closed at hi); each rank's vector holds its slab, created with the
 * split axis NON_PERIODIC (its own periodic images cover the other axes).  The
 * library labels, packs and unpacks on the device; the caller moves the packed
 * rows between ranks (an all-to-all of NCCL, MPI, or any transport): rows to
 * rank d are contiguous, ranks ascending, send_counts[d] of them.  A row is
 * pd_slab_row_bytes bytes: the position in the vector's type, then the
 * properties of prop_mask in their own types (int32 stays int32). */
typedef struct {
    int axis;      /* split axis 0..2 */
    int nslabs;    /* slabs = ranks */
    int periodic;  /* the global box is periodic along the axis */
    double lo, hi; /* the global box along the axis */
    double ghost;  /* halo width (<= the slab width) */
} pd_slab_t;
/* map, labelling: positions wrapped (the split axis by the global box when
 * periodic, the other axes by the vector's box), the owner of every real particle
 * found, the rows grouped by destination rank (ascending index within a rank);
 * send_counts[nslabs] (host) receives the rows per rank.  Synchronises. */
int pd_slab_map_label(pd_vd h, const pd_slab_t* s, long* send_counts, void* stream);
/* ghost_get, labelling for rank `rank`: every real particle and local periodic
 * image within `ghost` of the slab's lower face goes to the lower neighbour,
 * within `ghost` of the upper face to the upper one, shifted by the box length
 * across a periodic face; nothing for one slab.  Synchronises. */
int pd_slab_halo_label(pd_vd h, const pd_slab_t* s, int rank, long* send_counts, void* stream);
/* bytes of one packed row for the properties in prop_mask (a multiple of 8) */
int pd_slab_row_bytes(pd_vd h, unsigned long prop_mask, long* bytes);
/* the rows of the last labelling into `send` (device memory, room for cap_rows rows) */
int pd_slab_pack(pd_vd h, unsigned long prop_mask, void* send, long cap_rows, void* stream);
/* map, unpacking: the vector's particles become the n_recv received rows (ghosts
 * dropped; ids 0..n_recv-1; properties not in prop_mask zeroed) */
int pd_slab_map_unpack(pd_vd h, unsigned long prop_mask, const void* recv, long n_recv, void* stream);
/* ghost_get, unpacking: the n_recv received rows are appended as ghosts after the
 * vector's local periodic images (id -1); a later ghost_get or map drops them */
int pd_slab_halo_unpack(pd_vd h, unsigned long prop_mask, const void* recv, long n_recv, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PDGPU_H */
