/* fluidisim_delta3d.h — C ABI of the B200 delta (δ) MAC-grid pressure projection.
 *
 * The drop-in boundary for water-core's `Volume3` projection API.  Each entry point names the
 * reference function it replaces (paths relative to the reference project, code/water-core/src/).
 * Plain C types only: no CUDA, no torch.  Link against libfluidisim_delta3d.so.
 *
 * Conventions
 *  - Layouts are the reference's (delta3d.rs:24-28, 187-206): cells c = (k*ny + j)*nx + i, x
 *    fastest; u faces (nx+1)*ny*nz, v faces nx*(ny+1)*nz, w faces nx*ny*(nz+1); columns j*nx + i;
 *    SDF nodes (nx+1)*(ny+1)*(nz+1), x fastest.
 *  - Every entry point returns an fd3_status.  Codes 1..8 are the reference's `Error`
 *    (delta_projection.rs:133-150) in declaration order; codes >= 100 are device-side failures.
 *  - Refusals are atomic, as in the reference: on any error the published fields (u, v, w, p,
 *    eta and its roundoff) keep their previous bits.
 *  - All device memory is allocated by fd3_configure* and fd3_enable_multigrid; projections and
 *    steps allocate nothing (the reference's I-06 after `seal()`).
 *  - One CUDA stream per handle (fd3_set_stream); calls on one handle are not thread-safe, as
 *    `&mut self` in the reference.
 */
#ifndef FLUIDISIM_DELTA3D_H
#define FLUIDISIM_DELTA3D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum fd3_status {
  FD3_OK = 0,
  FD3_ERR_DOMAIN = 1,             /* Error::Domain */
  FD3_ERR_NOT_FINITE = 2,         /* Error::NotFinite */
  FD3_ERR_SHAPE = 3,              /* Error::Shape */
  FD3_ERR_BUDGET = 4,             /* Error::Budget (never raised here) */
  FD3_ERR_CLOCK = 5,              /* Error::Clock (never raised here) */
  FD3_ERR_CONVERGENCE = 6,        /* Error::Convergence */
  FD3_ERR_BACKGROUND_CONTEXT = 7, /* Error::BackgroundContext (never raised here) */
  FD3_ERR_NON_PLANAR = 8,         /* Error::NonPlanar (never raised here) */
  FD3_ERR_CUDA = 100,             /* a CUDA runtime call failed; fd3_last_cuda_error() says which */
  FD3_ERR_NO_DEVICE = 101,        /* no CUDA device */
  FD3_ERR_INVALID_ARGUMENT = 102, /* null handle or pointer */
  FD3_ERR_OUT_OF_MEMORY = 103,    /* device allocation failed at configure/enable time */
  FD3_ERR_SCRATCH_LIMIT = 104     /* the volume exceeds the static scratch of a no-alloc entry point */
} fd3_status;

/* Domain3 (delta3d.rs:44-63): cubic cells of side dx; the lid is z0 = nz*dx. */
typedef struct fd3_domain {
  uint64_t nx, ny, nz;
  float dx;
} fd3_domain;

/* Report (delta_projection.rs:164-189). */
typedef struct fd3_report {
  uint32_t refinements;
  uint32_t iterations;
  uint8_t degraded;
  uint8_t floor;
  uint8_t pad[6];
  double residual;
  double divergence;
  double backward_error;
  double divergence_plain;
} fd3_report;

/* Arithmetic of the global reductions (dot products, norms).
 *  FD3_REDUCE_F64          FP64 accumulation, FP64 alpha/beta and residual tests (default).
 *  FD3_REDUCE_ORDERED_F32  the reference's own order and precision (host.rs:60-72,
 *                          delta3d.rs:860-876): f32 sums of 64-element chunks merged in index
 *                          order in f32.  With it the whole projection reproduces the reference
 *                          bit for bit; the in-order merge is serial, so it is a parity mode. */
typedef enum fd3_reduction { FD3_REDUCE_F64 = 0, FD3_REDUCE_ORDERED_F32 = 1 } fd3_reduction;

/* Storage of the multigrid V-cycle's vectors (no reference counterpart; the reference stores f32).
 *  FD3_STORAGE_F32  the reference's f32 (default).
 *  FD3_STORAGE_F16  FP16 storage with f32 arithmetic for the fine z and every coarse level's x, r
 *                   and residual; CG vectors stay f32, dots and the true residual f64.  The V-cycle
 *                   runs on r / sigma, sigma = rms(r) dx^2 / 6, which keeps its values well inside
 *                   the FP16 range whatever the pressure scale; PCG is unchanged by that positive
 *                   scale.  The reference's outer loop (true residual, restart from b - A p,
 *                   delta3d_mobile.rs:547-588) is the defect correction that restores the 1e-6
 *                   tolerance.  Needs FD3_REDUCE_F64, kernels = 0 or 3 and an even nx (it runs
 *                   on the two-cells-per-thread kernels). */
typedef enum fd3_storage { FD3_STORAGE_F32 = 0, FD3_STORAGE_F16 = 1 } fd3_storage;

typedef struct fd3_options {
  uint32_t reduction;     /* fd3_reduction */
  uint32_t mg_max_levels; /* coarse levels kept by fd3_enable_multigrid; 0 = every level the
                             reference's coarsening rule allows (delta3d_multigrid.rs:73-88) */
  uint32_t use_graphs;    /* 1 = run the inner PCG loop as a CUDA graph with a WHILE node */
  uint32_t kernels;       /* fine-level kernels in f64 mode: 0 = 2.5-D blocked (default): on volumes
                             of 2^23 cells or more with f32 storage the TMA-staged kernels (nx % 8 ==
                             0) or four cells per thread (nx % 4 == 0), else two cells per thread
                             (one when nx is odd); 1 = one cell per thread (the family the ordered
                             mode always uses); 2 = 2.5-D blocked with one cell per thread; 3 = 2.5-D
                             blocked with two cells per thread; 4 = 2.5-D blocked with four cells per
                             thread (nx % 4 == 0, f32 storage); 5 = 2.5-D blocked, two cells per
                             thread, layers staged in shared memory by TMA copies (nx % 8 == 0, f32
                             storage).  Every family gives the same cell values; only the order of
                             the f64 partial sums differs */
  uint32_t no_overlap;    /* 1 = launch each kernel only after the previous one completes; 0 (default)
                             = programmatic dependent launch: the next kernel is scheduled early and
                             waits on the device (results are identical either way) */
  uint32_t storage;       /* fd3_storage of the V-cycle vectors */
  uint32_t no_tile_skip;  /* 1 = the blocked fine kernels process the tiles of columns outside the
                             sparse set too; 0 (default) = they skip them (results are identical) */
  uint32_t reserved[1];
} fd3_options;

typedef struct fd3_volume fd3_volume;

/* SparseChange (delta3d_sparse.rs:85-99): what a change of the sparse column set did. */
typedef struct fd3_sparse_change {
  uint64_t activated;       /* columns that entered the set, at rest with zero velocities */
  uint64_t deactivated;     /* columns that left the set, put to rest */
  uint64_t active_columns;  /* columns of the set after the change */
  double volume_removed;    /* perturbation volume the leaving columns carried, m^3 (compensated
                               height, summed in column order in f64) */
  float height_removed;     /* largest |eta - rest| of a leaving column, m */
  float velocity_removed;   /* largest |velocity| of a face set to zero, m/s */
} fd3_sparse_change;

/* LevelChange (delta3d_levels.rs:29-36): what a level change did. */
typedef struct fd3_level_change {
  double volume_before;  /* perturbation volume of the source, m^3 */
  double volume_after;   /* perturbation volume of the destination, m^3: equal to roundoff, less
                            what the destination's sparse set does not cover of the source's */
} fd3_level_change;

/* Side of a block of the shared block lattice, in columns (domain_blocks.rs:18). */
#define FD3_BLOCK 8

/* Library and device. */
const char* fd3_version(void);
const char* fd3_last_cuda_error(void);
int fd3_status_name(int status, char* buf, size_t len);

/* Volume3::configure (delta3d.rs:210): flat bottom, lateral walls, open lid. */
int fd3_configure(const fd3_domain* domain, float rho, float g_eff, fd3_volume** out);
/* Volume3::configure_with_bottom (delta3d.rs:300): bottom heights at column centres (nx*ny). */
int fd3_configure_with_bottom(const fd3_domain* domain, float rho, float g_eff, const float* bottom,
                              size_t bottom_len, fd3_volume** out);
/* Volume3::configure_with_solid (delta3d.rs:327): plus a solid given by its signed distance at
 * the nodes (negative inside), cut exactly by 24 tetrahedra per cell (delta3d_cut.rs:429). */
int fd3_configure_with_solid(const fd3_domain* domain, float rho, float g_eff, const float* bottom,
                             size_t bottom_len, const float* solid, size_t solid_len, fd3_volume** out);
void fd3_destroy(fd3_volume* v);

/* Solver options; call before fd3_enable_multigrid for mg_max_levels to apply. */
int fd3_set_options(fd3_volume* v, const fd3_options* options);
int fd3_get_options(const fd3_volume* v, fd3_options* options);
/* The CUDA stream (a cudaStream_t) every call of this handle is ordered on; NULL = the handle's
 * own non-blocking stream, created at configure (the legacy default stream cannot be captured). */
int fd3_set_stream(fd3_volume* v, void* stream);

/* Volume3::enable_multigrid (delta3d_multigrid.rs:339): the V-cycle preconditioner. */
int fd3_enable_multigrid(fd3_volume* v);
/* Volume3::multigrid_levels (delta3d_multigrid.rs:353); -1 when not enabled. */
int fd3_multigrid_levels(const fd3_volume* v);

/* Volume3::set_solid_rigid (delta3d.rs:382-509): the solid of a volume configured with one moves
 * as a rigid body (translation `velocity`, rotation `angular` in rad/s about `center`).  `solid` is
 * its new signed distance at the nodes.  The cut is redone on the device from the bottom-only
 * geometry; a face that opens takes the wall's normal velocity at its centre, a face that closes
 * loses its own; the solid volume a column gains raises its surface (compensated).  Refusal is
 * atomic: FD3_ERR_SHAPE, FD3_ERR_NOT_FINITE, FD3_ERR_DOMAIN (no solid, or the solid shares a cell
 * or a face with the bottom cut or reaches the lid layer, delta3d_cut.rs:485). */
int fd3_set_solid_rigid(fd3_volume* v, const float* solid, size_t solid_len, const float velocity[3],
                        const float angular[3], const float center[3]);
/* Volume3::set_solid (delta3d.rs:376-378): set_solid_rigid without rotation. */
int fd3_set_solid(fd3_volume* v, const float* solid, size_t solid_len, const float velocity[3]);

/* Volume3::set_free_surface (delta3d_mobile.rs:9): eta per column and the rest level; p = 0. */
int fd3_set_free_surface(fd3_volume* v, const float* eta, size_t len, float rest);
/* Volume3::set_surface (delta3d.rs:614). */
int fd3_set_surface(fd3_volume* v, const float* eta, size_t len);
/* Volume3::set_velocity (delta3d.rs:631): closes walls and closed faces (close_walls, :666). */
int fd3_set_velocity(fd3_volume* v, const float* u, size_t nu, const float* vv, size_t nv,
                     const float* w, size_t nw);
/* The same with device pointers (inputs already resident in HBM). */
int fd3_set_velocity_device(fd3_volume* v, const float* d_u, const float* d_v, const float* d_w);
/* Zero the pressure (the state set_free_surface leaves), e.g. to repeat a first projection. */
int fd3_reset_pressure(fd3_volume* v);

/* The sparse column set (delta3d_sparse.rs).  The memory stays the box (the window); a column
 * outside the set is solid for every operator, the faces touching it are closed, and it stays at
 * rest.  The edge of the set reads as the box's edge in the advection.  A full set is the box, bit
 * for bit.  The linear path refuses a volume with a set (FD3_ERR_DOMAIN); set_free_surface and
 * set_surface refuse a surface that is not `rest`, to the bit, outside the set.
 *
 * Volume3::enable_sparse (delta3d_sparse.rs:105): reserves the set, every column in it.
 * FD3_ERR_DOMAIN if already reserved. */
int fd3_enable_sparse(fd3_volume* v);
/* Volume3::set_active_columns (delta3d_sparse.rs:147): mask[j*nx + i] != 0 puts column (i, j) in
 * the set.  A column that leaves goes to rest (surface, roundoff, pressure, every face); what it
 * carried is published in `change` (may be NULL).  FD3_ERR_DOMAIN without a set, FD3_ERR_SHAPE
 * when len != nx*ny; nothing is written then.  No allocation. */
int fd3_set_active_columns(fd3_volume* v, const uint8_t* mask, size_t len, fd3_sparse_change* change);
/* Volume3::set_active_blocks (delta3d_sparse.rs:163): the set from blocks of FD3_BLOCK x FD3_BLOCK
 * columns; `blocks` holds `count` (i, j) pairs of int32, and block (bi, bj) covers the columns
 * [(bi - origin_i)*FD3_BLOCK, +FD3_BLOCK) x [(bj - origin_j)*FD3_BLOCK, +FD3_BLOCK), clipped to the
 * window.  As fd3_set_active_columns. */
int fd3_set_active_blocks(fd3_volume* v, const int32_t* blocks, size_t count, int32_t origin_i, int32_t origin_j,
                          fd3_sparse_change* change);
/* Volume3::active_columns (delta3d_sparse.rs:129): the set, one byte per column.  FD3_ERR_DOMAIN
 * without a set. */
int fd3_active_columns(const fd3_volume* v, uint8_t* out, size_t len);
/* Volume3::sparse_cells (delta3d_sparse.rs:135): cells of the set's columns (every cell without
 * a set). */
uint64_t fd3_sparse_cells(const fd3_volume* v);

/* Volume3::resample_from (delta3d_levels.rs:43): `v` receives the state of `src`, which covers the
 * same window at another dx (a level change).  The surface by overlap of a conservative linear
 * reconstruction of each source column (centred slopes and the cross term; the perturbation volume
 * is kept exactly), the velocities trilinear at each destination face's centre on the source's
 * staggered grid, averaged over n x n sub-faces when the destination is coarser (n = ceil of the
 * ratio), the pressure zero, walls and faces outside the destination's sparse set closed.  Either
 * volume may carry a sparse set: the source's edge reads as the box's edge, and only the
 * destination's set receives the state.  Both volumes on the same device.  FD3_ERR_DOMAIN, nothing
 * written: different extent (1e-6 relative), rest, density or gravity, or a cut on either side. */
int fd3_resample_from(fd3_volume* v, fd3_volume* src, fd3_level_change* change);
/* Volume3::perturbation_volume (delta3d_balance.rs:105): sum over columns of the compensated height
 * minus rest, times dx^2, in f64 and in column order. */
int fd3_perturbation_volume(fd3_volume* v, double* out);

/* project_mobile3 (delta3d_mobile.rs:465) of the current velocity field: us = u, then the
 * projection with `scale` (-rho/dt) and `k1` (dt/rho), as tests_delta3d.rs:389-400 does. */
int fd3_project_mobile(fd3_volume* v, float scale, float k1, uint32_t max_iters, fd3_report* report);
/* refine_mobile3 (delta3d_coupling.rs:226-248), the reference's defect correction of a projection
 * that stopped at its floor: the current pressure is kept as the base, the current (corrected)
 * velocity field is projected again from p = 0 with homogeneous ghosts (ghost values 0,
 * delta3d_mobile.rs:130, 140), and the pressure increment is added to the base.  report is that
 * second projection's, with refinements = 1.  A refusal leaves u, v, w and p untouched. */
int fd3_refine_mobile(fd3_volume* v, float scale, float k1, uint32_t max_iters, fd3_report* report);
/* Volume3::step_surface_mobile (delta3d_mobile.rs:819): advect, project, extrapolate, transport. */
int fd3_step_surface_mobile(fd3_volume* v, uint64_t duration_us, uint32_t max_iters, fd3_report* report);
/* Volume3::enable_advection_correction (delta3d_advection.rs:19): the second-order term of the
 * advection, + (dt^2/2) sum V_a V_b d_a d_b u on the prediction (Lax-Wendroff at constant velocity),
 * for the mobile steps that follow.  Off by default: the step is then the reference's, bit for bit. */
int fd3_enable_advection_correction(fd3_volume* v);
/* Volume3::advection_correction (delta3d_advection.rs:24): 1 when the term is on. */
int fd3_advection_correction(const fd3_volume* v);
/* The predictor alone, as tests_delta3d.rs:2136-2160 runs it: advect_mobile3 over dt seconds, the
 * second-order term when on, then the prediction becomes the velocity.  No projection. */
int fd3_advect_for_tests(fd3_volume* v, float dt);
/* No reference counterpart: many independent volumes (patches), each projected as
 * fd3_project_mobile projects it, concurrently.  Every volume keeps its own stream and device-side
 * loop; `threads` host workers (0 = up to 16) issue them, largest first.  statuses[i] and
 * reports[i] are volume i's; the return value is FD3_OK unless the arguments are invalid (a null
 * pointer, or one volume listed twice). */
int fd3_project_batch(fd3_volume* const* volumes, size_t count, const float* scales, const float* k1s,
                      uint32_t max_iters, int threads, fd3_report* reports, int* statuses);
/* The persistent batch (no reference counterpart): many volumes (patches) projected by ONE kernel
 * launch.  Thread-block clusters of `cluster_size` CTAs (1, 2, 4 or 8) of 1024 threads are
 * independent solvers; the volumes are dealt, largest first, to the least loaded of the clusters
 * that fit the GPU at once, and each cluster runs its volumes' whole project_mobile3 (assembly,
 * hierarchy, multigrid PCG, outer checks, report) on the device, one volume after another.
 * fd3_batch_create validates and prepares (all of its allocations happen here): every volume on
 * the same device, listed once, with multigrid, f64 reductions and f32 storage (FD3_ERR_DOMAIN
 * otherwise).  The batch holds pointers into the volumes: destroy it before them.  Calls on one
 * batch are not thread-safe. */
typedef struct fd3_batch fd3_batch;
int fd3_batch_create(fd3_volume* const* volumes, size_t count, int cluster_size, fd3_batch** out);
void fd3_batch_destroy(fd3_batch* batch);
/* The clusters the volumes were dealt to and their size. */
int fd3_batch_clusters(const fd3_batch* batch, int* clusters, int* cluster_size);
uint64_t fd3_batch_kernel_launches(const fd3_batch* batch);
/* Projects every volume of the batch as fd3_project_mobile does (us = u), in one launch on the
 * batch's own stream, after each volume's stream has finished its earlier work; returns when all
 * are done.  reset_pressure = 1 starts every volume from p = 0 (fd3_reset_pressure).  in_u, in_v,
 * in_w (all or none; device pointers per volume, of the face counts) are copied into the volumes'
 * velocities first.  statuses[i] is volume i's result (FD3_OK, FD3_ERR_NOT_FINITE for a
 * non-finite input, ...); a refused volume keeps u, v, w and p as they were.  reports[i] is its
 * Report.  Allocates nothing. */
int fd3_batch_project(fd3_batch* batch, const float* scales, const float* k1s, uint32_t max_iters, int reset_pressure,
                      const float* const* in_u, const float* const* in_v, const float* const* in_w,
                      fd3_report* reports, int* statuses);
/* Volume3::last_refused_report (delta3d_mobile.rs:982); FD3_ERR_DOMAIN when none. */
int fd3_last_refused_report(const fd3_volume* v, fd3_report* report);

/* The linear (fixed-lid) path.  project (delta3d.rs:1060) of the current velocity field: us = u,
 * then CG (or Jacobi-PCG on a cut bottom with ny > 1) with the lid at eta - z0, as
 * tests_delta3d.rs:143-148 does.  The multigrid, when enabled, is not used on this path. */
int fd3_project_linear(fd3_volume* v, float scale, float k1, uint32_t max_iters, fd3_report* report);
/* Volume3::step_surface_linear (delta3d.rs:1209): project, then the heights from the column
 * fluxes (compensated).  Refusal is atomic, as for the mobile step. */
int fd3_step_surface_linear(fd3_volume* v, uint64_t duration_us, uint32_t max_iters, fd3_report* report);
/* Volume3::set_precondition_cut (delta3d.rs:526): Jacobi on the linear cut path (default on). */
int fd3_set_precondition_cut(fd3_volume* v, int on);

/* Accessors (delta3d.rs:647-661) into caller buffers. */
int fd3_get_pressure(const fd3_volume* v, float* out, size_t len);
int fd3_get_velocity(const fd3_volume* v, float* u, size_t nu, float* vv, size_t nv, float* w, size_t nw);
int fd3_get_surface(const fd3_volume* v, float* eta, float* roundoff, size_t len);
/* Device pointers of the published fields (p, u, v, w), valid until fd3_destroy. */
int fd3_device_fields(const fd3_volume* v, float** p, float** u, float** vv, float** w);
/* Cut geometry (delta3d.rs:595-602): frac, open_u/v/w, floor.  FD3_ERR_DOMAIN on a flat bottom. */
int fd3_get_geometry(const fd3_volume* v, float* frac, float* open_u, float* open_v, float* open_w, float* floor);
uint64_t fd3_wet_cells(const fd3_volume* v);

/* Volume3::apply_pressure_operator_for_trials (delta3d_mobile.rs:936). */
int fd3_apply_pressure_operator_for_trials(fd3_volume* v, const float* p, float* out, size_t len);
/* Volume3::assemble_pressure_problem_for_trials (delta3d_mobile.rs:960). */
int fd3_assemble_pressure_problem_for_trials(fd3_volume* v, const float* divergence, float scale,
                                             float* rhs, float* prec, size_t len);
/* The pressure-problem assembly for callers that cannot allocate device memory when they call:
 * a host whose memory arena is sealed once it is set up, or a real-time loop in which a cudaMalloc
 * would stall a frame.  It has no counterpart in the reference.
 * Inputs and outputs are device pointers of `len` cells on the volume's device: d_divergence in;
 * d_rhs (the right-hand side: scale times the divergence plus the surface-ghost terms of each wet
 * row, 0 on dry cells) and d_prec (1 / the row's diagonal, 0 on dry cells) out; |rhs|^2 in f64
 * written to *rhs_norm2 (host memory).  The volume's own buffers are not touched.
 * Ordering: the call runs on the volume's stream (fd3_set_stream) and does not wait for the
 * caller's other streams, so work that writes d_divergence must be complete before the call; the
 * call synchronises the volume's stream before it returns.  The volume's device is made current
 * for the call and the caller's current device is restored.
 * It allocates nothing: its scratch is a static device array of 128 KiB + 256 B in this library,
 * held on every GPU that loads it until the process exits, so volumes above 4,194,304 cells are
 * refused with FD3_ERR_SCRATCH_LIMIT.  The first call on a device looks the scratch's device
 * address up (cudaGetSymbolAddress) and should come before any stream capture.  All calls share
 * the one scratch array and it keeps the last call's contents: each call clears the parts that
 * must start at zero, and calls that overlap on the GPU (other streams, other threads) race.
 * A non-finite divergence gives FD3_ERR_NOT_FINITE (the outputs are then written anyway). */
int fd3_assemble_pressure_problem_noalloc(fd3_volume* v, const float* d_divergence, float scale, float* d_rhs,
                                          float* d_prec, size_t len, double* rhs_norm2);
/* v_cycle3 (delta3d_multigrid.rs:393) on `x`, set up as tests_delta3d.rs:1840-1873 does
 * (rhs = 0, rhs_mobile3(1), prepare_multigrid3, res = x).  Writes z = M^-1 x. */
int fd3_vcycle_for_tests(fd3_volume* v, const float* x, float* z, size_t len);
/* Coarse level l after prepare_multigrid3: kind, diag, open_u/v/w (Level3, delta3d_multigrid.rs:37). */
int fd3_level_geometry(const fd3_volume* v, uint32_t l, float* kind, float* diag, float* open_u,
                       float* open_v, float* open_w);

/* Kernel launches issued by this handle since creation (for launch accounting).  No reference
 * counterpart: instrumentation of this library. */
uint64_t fd3_kernel_launches(const fd3_volume* v);
/* Per-kernel timing (no reference counterpart): with on = 1, every launch of this handle is
 * bracketed by CUDA events on its stream and the durations are summed per kernel name at each
 * synchronisation; CUDA-graph replay is bypassed meanwhile.  on = 0 stops it. */
int fd3_profile(fd3_volume* v, int on);
int fd3_profile_count(const fd3_volume* v);
int fd3_profile_entry(const fd3_volume* v, int index, char* name, size_t name_len, uint64_t* launches,
                      double* total_ms);

/* ------------------------------------------------------------------ learned preconditioner
 * No reference counterpart: the learned part of the B200 build.  A 3-D U-Net (3 levels, 16/32/64
 * channels, 3x3x3 convolutions, BF16 with FP32 accumulation) used as the preconditioner of a
 * flexible CG, with the multigrid PCG of fd3_project_mobile as its fallback. */
typedef struct fd3_unet fd3_unet;

/* A network whose buffers hold max_batch samples of nz x ny x nx cells (each a multiple of 4; a
 * forward pass takes nx <= 512). */
int fd3_unet_create(int max_batch, int nz, int ny, int nx, fd3_unet** out);
void fd3_unet_destroy(fd3_unet* net);
int fd3_unet_set_stream(fd3_unet* net, void* stream);
/* Parameters, f32, per layer (e0, e1, b, d1, d0, head): w[27][cout][cin] then b[cout]. */
uint64_t fd3_unet_param_count(const fd3_unet* net);
int fd3_unet_set_params(fd3_unet* net, const float* params, size_t len);
int fd3_unet_get_params(const fd3_unet* net, float* params, size_t len);
/* The accumulated parameter gradient (then cleared). */
int fd3_unet_get_grads(fd3_unet* net, float* grads, size_t len);
/* y = out_scale[b] * net(x), x[b*cells + c][3] = (residual * in_scale[b], solid, liquid); device
 * pointers x and y, host arrays of B scales.  Stream-ordered. */
int fd3_unet_forward(fd3_unet* net, int batch, int nz, int ny, int nx, const float* d_in, const float* in_scale,
                     const float* out_scale, float* d_out);
/* Accumulates the parameter gradient of the last forward for dL/dy = d_gout (device). */
int fd3_unet_backward(fd3_unet* net, const float* d_gout);
/* Adam step on the accumulated gradient (consumed). */
int fd3_unet_adam(fd3_unet* net, float lr, float beta1, float beta2, float eps);
int fd3_unet_sync(fd3_unet* net);
/* Convolution kernels of the network: 1 = tcgen05.mma with tensor-memory accumulators, one phase at
 * a time per CTA (default); 2 = the same MMAs as a warp-specialised pipeline (producer warps staging
 * a ring of shared-memory slots, one MMA-issuing thread, epilogue warps draining one of two
 * tensor-memory accumulators while the other fills; the same bits as 1); 0 = mma.sync m16n8k16
 * (the earlier tensor-core path, kept to cross-check). */
int fd3_unet_set_conv_kernels(fd3_unet* net, int tcgen05);
/* Budget of 128-row output tiles per CTA of the tcgen05 convolutions, 1..5 (default 5; raised to
 * what one row of the layer needs): fewer tiles make smaller CTAs, more of them per SM. */
int fd3_unet_set_conv_tiles(fd3_unet* net, int tiles);
uint64_t fd3_unet_kernel_launches(const fd3_unet* net);

/* Device-side hooks of a training loop, on a volume: the rhs and row codes of project_mobile3 for
 * the current velocity (us = u), their device pointers, A x, the network input of a residual
 * (and its squared norm), and loss = w |A z - b|^2 with d_grad = 2 w A (A z - b). */
int fd3_assemble_device(fd3_volume* v, float scale);
int fd3_problem_device(fd3_volume* v, float** d_rhs, const unsigned short** d_codes);
int fd3_apply_device(fd3_volume* v, const float* d_x, float* d_out);
int fd3_learned_input(fd3_volume* v, const float* d_r, float* d_in3, double* rr);
/* How fd3_project_learned uses the network (no reference counterpart): 0 (default) = FCG's
 * preconditioner is the network alone; 1 = the multigrid V-cycle plus the network's approximation
 * of A^-1 applied to the residual the V-cycle leaves (a network trained on such residuals, see
 * fd3_vcycle_residual_device).  Mode 1 needs a volume with multigrid. */
int fd3_unet_set_mode(fd3_unet* net, int mode);
/* The residual a V-cycle leaves: rho = r - A V(r) for a device vector r of the last assembly's
 * problem (fd3_assemble_device), |rho|^2 into *rho2 (may be NULL).  Uses the volume's work buffers;
 * d_rho may equal d_r.  FD3_ERR_DOMAIN without multigrid.  No reference counterpart. */
int fd3_vcycle_residual_device(fd3_volume* v, const float* d_r, float* d_rho, double* rho2);
int fd3_residual_loss(fd3_volume* v, const float* d_z, const float* d_b, float weight, float* d_grad, double* loss);

/* project_mobile3 with the learned FCG in front (from the current p): FCG(1) with the network as
 * the preconditioner until the reference tolerance, max_fcg iterations or a stall, then the
 * reference acceptance loop.  When FCG reached the tolerance the loop starts from its p; when it
 * stalled (or hit max_fcg), its p is discarded and the loop's multigrid PCG, the fallback, starts
 * from the pressure the call started with.  report is that loop's (its iterations are the
 * fallback's); fcg_iterations and fell_back describe FCG. */
int fd3_project_learned(fd3_volume* v, fd3_unet* net, float scale, float k1, uint32_t max_iters, uint32_t max_fcg,
                        fd3_report* report, uint32_t* fcg_iterations, int* fell_back);

#ifdef __cplusplus
}
#endif

#endif /* FLUIDISIM_DELTA3D_H */
