/*
 * ppf.h -- C ABI of libppf, a B200-native (sm_100a) implementation of the
 * PaScaL_POISSON_FFT solve path: 2-D real FFT / DCT-II in x and y, batched
 * tridiagonal solves along z, inverse transforms, mean removal and the
 * ghost-cell update, all in hand-written CUDA kernels.
 *
 * Plain C types only: sizes are int, arrays are pointers, CUDA streams are
 * passed as `void*` (a cudaStream_t, NULL = legacy default stream).  Every
 * entry point returns an int status (PPF_OK = 0, negative on error) and
 * never aborts; ppf_last_error() returns a message for the calling thread.
 *
 * Array layouts are the reference's (Fortran column-major, first index
 * fastest):
 *   PRHS(1:n1m, 1:n2m, 1:n3m)            right-hand side, FP64, device
 *   P(0:n1m+1, 0:n2m+1, 0:n3m+1)          solution with ghost cells, FP64, device
 *   dmx1(0:n1m+1) dmx2(0:n2m+1) dmx3(0:n3m+1) dx3(0:n3m+1)   metrics, FP64, device
 * where n*m is the number of cells along an axis (the reference's n*m,
 * n* = n*m + 1 faces).
 */
#ifndef PPF_H
#define PPF_H

#if defined(__GNUC__)
#define PPF_API __attribute__((visibility("default")))
#else
#define PPF_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

enum {
    PPF_OK = 0,
    PPF_ERR_INVALID = -1,      /* bad argument or descriptor */
    PPF_ERR_CUDA = -2,         /* a CUDA runtime call failed */
    PPF_ERR_NOMEM = -3,        /* device allocation failed */
    PPF_ERR_UNSUPPORTED = -4,  /* size/configuration outside what the kernels support */
    PPF_ERR_STATE = -5,        /* call out of order (e.g. solve before initial) */
    PPF_ERR_NUMERIC = -6       /* a kernel reported a non-finite pivot or hit a wait bound */
};

enum { PPF_FP64 = 0, PPF_MIXED = 1, PPF_FP32 = 2 };

typedef struct ppf_plan ppf_plan;

/* Plan descriptor.  Mirrors the arguments of
 * fft_poisson_plan_cuda_create (01_Fortran/src/fft_3d_poisson.f90:70-108)
 * at one rank, plus the precision options of this library. */
typedef struct {
    int n1m, n2m, n3m;         /* cells along x, y, z (n1m, n2m even) */
    double L1, L2;             /* domain lengths along x and y (uniform spacing L/n) */
    int pbc1, pbc2, pbc3;      /* 1 = periodic, 0 = Neumann (per axis) */
    int precision;             /* PPF_FP64 | PPF_MIXED | PPF_FP32 */
    int max_sweeps;            /* PPF_MIXED: FP64-residual refinement sweeps after the
                                  first FP32 solve (0..8); <0 selects the default (2) */
    double sweep_tol;          /* PPF_MIXED: stop refining once ||du||/||u|| < tol (0 = never) */
    double lowk_threshold;     /* FP32 storage: z systems with lambda*dz_min^2 below this (the
                                  near-singular low wavenumbers, k^2 dz^2 << 1 at the finest
                                  z spacing) are solved in FP64 (<=0 selects the default 1e-3) */
} ppf_desc;

/* Create / destroy a plan on the current CUDA device.  Allocates the
 * spectral work buffers and the twiddle / wavenumber tables. */
PPF_API int ppf_plan_create(const ppf_desc *desc, ppf_plan **plan);
PPF_API int ppf_plan_destroy(ppf_plan *plan);

/* Solve lap(u) = f.  f_d: PRHS layout (not modified).  p_d: ghosted P layout
 * (written: interior = solution with zero arithmetic mean, ghosts per the
 * reference's Neumann extrapolation / periodic copy).  Metric arrays as in
 * the header comment.  Asynchronous on `stream`; no host synchronisation.
 * Replaces cuda_Poisson_FFT_1D (01_Fortran/src/fft_3d_poisson.f90:353-626). */
PPF_API int ppf_solve(ppf_plan *plan, const double *f_d, double *p_d,
              const double *dmx1_d, const double *dmx2_d,
              const double *dmx3_d, const double *dx3_d, void *stream);

/* Transpose of the solve map f -> u (interior cells) and, optionally, the
 * gradient with respect to the z metric arrays.  No reference counterpart:
 * the reference solve is not differentiable.
 *   g_d:   dJ/du, PRHS layout (n1m, n2m, n3m), FP64 device.
 *   df_d:  output dJ/df = M^T g, PRHS layout (may alias g_d).
 *   u_d:   the forward solution (ghosted P layout, as written by ppf_solve
 *          with the same metrics); needed only for the metric gradient.
 *   ddx3_d, ddmx3_d: output dJ/d dx3 and dJ/d dmx3 (n3m+2 doubles, Fortran
 *          indices 0..n3m+1, entries the solve does not read are 0), or NULL.
 * J is taken on the interior cells (ghost cells carry no cotangent).  The
 * adjoint runs one solve with the plan's precision (mixed refinement
 * included) on diag(1/dx3) g, spectral intermediates are recomputed, not
 * stored.  The first call on a plan allocates one ghosted FP64 field of
 * work memory (not capturable); later calls are asynchronous on `stream`. */
PPF_API int ppf_solve_adjoint(ppf_plan *plan, const double *g_d, double *df_d, const double *u_d,
              double *ddx3_d, double *ddmx3_d,
              const double *dmx1_d, const double *dmx2_d,
              const double *dmx3_d, const double *dx3_d, void *stream);

/* Batched solves of independent problems of uneven shape and boundary
 * conditions.  No reference counterpart (the reference solves one grid per
 * rank).  ppf_batch_create builds a plan per descriptor, spreads the
 * problems over `branches` concurrent branches (<= 0: 8) with one work
 * area per branch, and with PPF_BATCH_AUTOTUNE times the candidate tile
 * widths and radix orders of every distinct x and y transform on the
 * device and keeps the fastest.  ppf_batch_solve takes host arrays of
 * `count` device pointers (layouts as ppf_solve); the first call, and any
 * call with different pointers, captures all problems into one CUDA graph
 * (not itself capturable); every call then replays it with one graph launch
 * on `stream`.  ppf_batch_info(batch, i, info[8]): branch of problem i,
 * x tile width / run-time engine / radix order, the same for y, and the
 * number of branches (0 width = default).
 * With PPF_BATCH_PERSISTENT the whole batch runs as one persistent kernel
 * instead: a grid of CTAs resident on every SM takes tiles of every stage of
 * every problem from a device work queue (stage-major across the problems),
 * a stage starting once the problem's previous stage is complete (bounded
 * waits); each problem gets its own work memory, the transforms use the
 * run-time engine, and PPF_BATCH_AUTOTUNE has no effect.  The graph then
 * holds that one launch; info reports 0 branches. */
typedef struct ppf_batch ppf_batch;
#define PPF_BATCH_AUTOTUNE 1
#define PPF_BATCH_PERSISTENT 2
PPF_API int ppf_batch_create(const ppf_desc *descs, int count, int flags, int branches, ppf_batch **batch);
PPF_API int ppf_batch_destroy(ppf_batch *batch);
PPF_API int ppf_batch_solve(ppf_batch *batch, const double *const *f_d, double *const *p_d,
              const double *const *dmx1_d, const double *const *dmx2_d,
              const double *const *dmx3_d, const double *const *dx3_d, void *stream);
PPF_API int ppf_batch_info(const ppf_batch *batch, int index, int *info);

/* Same as ppf_solve with host arrays: copies in, solves, copies out and
 * synchronises `stream` before returning (the C++ driver's calling model,
 * 00_C/examples/modules.hpp:223-232). */
PPF_API int ppf_solve_host(ppf_plan *plan, const double *f_h, double *p_h,
                   const double *dmx1_h, const double *dmx2_h,
                   const double *dmx3_h, const double *dx3_h, void *stream);

/* ppf_solve_host without the final synchronisation: the copies in, the
 * solve and the copy out are enqueued on `stream` and the call returns.
 * The host arrays must stay valid (and p_h unread) until the stream has
 * finished; with page-locked host arrays the copies run asynchronously, so
 * a caller that alternates two plans on two streams overlaps one solve's
 * copy-out with the next solve's copy-in (they use separate copy engines).
 * No reference counterpart (the reference solve is synchronous). */
PPF_API int ppf_solve_host_async(ppf_plan *plan, const double *f_h, double *p_h,
                   const double *dmx1_h, const double *dmx2_h,
                   const double *dmx3_h, const double *dx3_h, void *stream);

/* Number of refinement sweeps the last PPF_MIXED solve executed (device
 * early exit on sweep_tol), and ||du||/||u|| of its last sweep.  Reads two
 * device scalars (synchronises `stream`). */
PPF_API int ppf_last_sweeps(ppf_plan *plan, int *sweeps, double *last_rel_update, void *stream);

/* Per-stage device timing.  While enabled, every solve records a CUDA
 * event after each kernel on the solve's stream; ppf_stage_times()
 * synchronises on the recorded events, returns the accumulated
 * milliseconds and launch counts per stage since the last call, and resets
 * them.  Stages (the reference's NVTX ranges, fft_3d_poisson.f90:377-624):
 * 0 z-coefficients, 1 x forward ("Poisson-F_x"), 2 y forward ("-F_y"),
 * 3 z tridiagonal ("-TDMA-z"), 4 y inverse ("-B_y"), 5 x inverse ("-B_x"),
 * 6 refinement gate, 7 ghost cells. */
#define PPF_NSTAGES 8
PPF_API int ppf_stage_timing(ppf_plan *plan, int enable);
PPF_API int ppf_stage_times(ppf_plan *plan, double *ms, int *launches);

/* Bytes of device work memory held by the plan for its solves: spectral
 * buffers, z-solve checkpoints, and for a mixed-precision plan its partial
 * sums and, when it refines (max_sweeps > 0), one FP32 ghosted field that
 * holds the first iterate. */
PPF_API int ppf_plan_workspace_bytes(const ppf_plan *plan, long long *bytes);

/* Batched tridiagonal solves on device arrays, system index fastest:
 * element (sys, row) at [row * n_sys + sys].  In place: d <- x.  a, b, c
 * are not modified (the reference overwrites c; callers that relied on
 * that scratch content get the unmodified coefficients back instead).
 * Replaces PaScaL_TDMA_many_solve_cuda (01_Fortran/PaScaL_TDMA/src/
 * pascal_tdma_cuda.f90:230-269) at nprocs=1 -> tdma_many_cuda
 * (tdmas_cuda.f90:35-102); C ABI of 00_C/PaScaL_TDMA/src/pascal_tdma.hpp:67-71. */
PPF_API int ppf_tdma_many(const double *a, const double *b, const double *c, double *d,
                  int n_sys, int n_row, void *stream);

/* Cyclic variant (periodic systems).  Replaces
 * PaScaL_TDMA_many_solve_cycle_cuda (pascal_tdma_cuda.f90:279-318) ->
 * tdma_cycl_many_cuda (tdmas_cuda.f90:114-217).  n_row >= 3. */
PPF_API int ppf_tdma_cycl_many(const double *a, const double *b, const double *c, double *d,
                       int n_sys, int n_row, void *stream);

/* Systems whose rows are split over ranks (z slabs), PaScaL_TDMA_many_solve_cuda
 * at nprocs > 1 (pascal_tdma_cuda.f90:243-266).  Step 1,
 * ppf_tdma_many_modified: the modified Thomas algorithm on this rank's
 * n_row (>= 3) rows (pascal_tdma_cuda.f90:332-473); a, c, d are overwritten
 * with the modified coefficients, b is read only, and the rank's two reduced
 * rows (b = 1) go to a_rd, c_rd, d_rd, element (sys, r) at [r * n_sys + sys],
 * r = 0 for the first local row, 1 for the last.  The caller gathers the
 * reduced rows of all ranks per system (2 * nranks rows, rank-major) and
 * solves them (ppf_tdma_many with b = 1), then step 2,
 * ppf_tdma_many_update (pascal_tdma_cuda.f90:483-520), finishes the local
 * rows from the reduced solution x_rd (same layout as d_rd).
 * pascal_poisson_fft_b200.dist drives the exchange with torch.distributed. */
PPF_API int ppf_tdma_many_modified(double *a, const double *b, double *c, double *d,
                           double *a_rd, double *c_rd, double *d_rd,
                           int n_sys, int n_row, void *stream);
PPF_API int ppf_tdma_many_update(const double *a, const double *c, double *d, const double *x_rd,
                         int n_sys, int n_row, void *stream);

/* z-slab (multi-rank) FP64 solve, the reference's np3 > 1 decomposition of
 * cuda_Poisson_FFT_1D (fft_3d_poisson.f90:353-626): the plan describes this
 * rank's slab (n3m = its z rows); pascal_poisson_fft_b200.dist.SlabPoisson
 * drives the steps and the exchanges between ranks.
 *   ppf_slab_systems:   doubles per z row of the spectrum (= systems: real and
 *                       imaginary parts are separate systems).
 *   ppf_slab_forward:   x and y forward transforms of f into spec (n3m rows).
 *   ppf_slab_coefficients: a, b, c of this rank's rows z0 .. z0+n3m-1 of the
 *                       global z operator (global dx3_g, dmx3_g of n3m_g+2
 *                       values), the pin at the global first row, and the
 *                       normalisation applied to spec; then the multi-rank
 *                       TDMA (ppf_tdma_many_modified / _update) solves spec.
 *   ppf_slab_inverse:   inverse transforms of spec into the interior of P.
 *   ppf_slab_sum:       deterministic interior sum of P into *sum_d (device).
 *   ppf_slab_shift:     P -= *shift_d on the interior (the global mean).
 *   ppf_slab_ghosts:    ghost update in the reference's order with z walls
 *                       only where flagged (the global ends); the ghost planes
 *                       between slabs must hold the neighbours' planes first. */
PPF_API int ppf_slab_systems(const ppf_plan *plan, int *n_sys);
PPF_API int ppf_slab_forward(ppf_plan *plan, const double *f_d, double *spec_d, void *stream);
PPF_API int ppf_slab_coefficients(ppf_plan *plan, double *a_d, double *b_d, double *c_d, double *spec_d,
                          const double *dx3_g, const double *dmx3_g, int z0, int n3m_g, void *stream);
PPF_API int ppf_slab_inverse(ppf_plan *plan, const double *spec_d, double *p_d, void *stream);
PPF_API int ppf_slab_sum(ppf_plan *plan, const double *p_d, double *sum_d, void *stream);
PPF_API int ppf_slab_shift(ppf_plan *plan, double *p_d, const double *shift_d, void *stream);
PPF_API int ppf_slab_ghosts(ppf_plan *plan, double *p_d, const double *dmx1_d, const double *dmx2_d,
                    const double *dmx3_d, int z_lo_wall, int z_hi_wall, void *stream);

/* Allocation-free FP64 solve, for callers that cannot allocate device
 * memory at solve time: a flow solver that reserved its whole device memory
 * budget at start-up, or an application whose memory is owned by another
 * framework.  No counterpart in the reference (whose solve allocates its
 * coefficient arrays on every call).  Same arguments and result as
 * ppf_plan_create + ppf_solve with precision PPF_FP64, but every work buffer
 * lives in one static device array of PPF_NOALLOC_SCRATCH_BYTES that each
 * GPU loading the library holds until the process exits; grids whose work
 * memory does not fit (about 128^3 cells) are rejected with
 * PPF_ERR_UNSUPPORTED and a message naming the bytes needed.  The first call
 * on a device looks up the array's device address and uploads the grid's
 * wavenumber and twiddle tables (a few KB, cached per CUDA context and grid;
 * again after a device reset or a change of grid); make that first call
 * before any stream capture.  All calls on a device share the array and it
 * keeps the last call's contents: calls whose kernels overlap on the GPU
 * (different streams, or different host threads without ordering) race on
 * it.  The caller passes inputs and outputs; nothing is allocated, freed or
 * cached beyond the array itself and a small static host staging table. */
#define PPF_NOALLOC_SCRATCH_BYTES (64u << 20)
PPF_API int ppf_solve_noalloc(const ppf_desc *desc, const double *f_d, double *p_d,
                              const double *dmx1_d, const double *dmx2_d,
                              const double *dmx3_d, const double *dx3_d, void *stream);

/* Ghost cells of a ghosted field P(0:n1m+1, 0:n2m+1, 0:n3m+1) on the device,
 * outside a solve.  walls != 0: the solve's update (quadratic Neumann
 * extrapolation along every non-periodic axis with its dmx array, then the
 * periodic copies; cuda_neumann_BC and cuda_ghostcell_update,
 * 01_Fortran/src/fft_3d_poisson.f90:666-852).  walls == 0: only the periodic
 * copies, the one-rank form of the example driver's subdomain halo update
 * (cuda_subdomain_ghostcell_update, 01_Fortran/examples/cuda_subdomain.f90:
 * 199-220) that follows a restart load (main.f90:136-139); the dmx arrays may
 * then be NULL.  Asynchronous on `stream`. */
PPF_API int ppf_ghost_update(double *P_d, int n1m, int n2m, int n3m, int pbc1, int pbc2, int pbc3,
                     const double *dmx1_d, const double *dmx2_d, const double *dmx3_d, int walls, void *stream);

/* Node values of a ghosted cell field for the 3-D instant-field dump:
 * G(i,j,k), i = 1..n1m, j = 1..n2m, k = 1..n3m, stored (n1m, n2m, n3m) x
 * fastest, the eight-cell weighted average of calc_C2g
 * (01_Fortran/examples/cuda_post.f90:338-353, used by
 * cuda_Post_Fileout_InstantField_3D, :294-331).  dx1, dx2, dx3: cell widths
 * (0:n*m+1).  Asynchronous on `stream`. */
PPF_API int ppf_cell_to_node(const double *P_d, int n1m, int n2m, int n3m, const double *dx1_d,
                     const double *dx2_d, const double *dx3_d, double *G_d, void *stream);

/* Thread-local message describing the last error ("" if none). */
PPF_API const char *ppf_last_error(void);

/* Library version string. */
PPF_API const char *ppf_version(void);

/* ---------------------------------------------------------------------
 * Reference-shaped entry points (one active plan per process, like the
 * module-global p_poi of 01_Fortran/src/fft_3d_poisson.f90:43-59).  These
 * are what the Fortran iso_c_binding shim binds.
 * ------------------------------------------------------------------- */

/* fft_poisson_plan_cuda_create (fft_3d_poisson.f90:70-108) at one rank:
 * n1,n2,n3 are face counts (cells + 1), n*sub = n* at one rank.  The MPI
 * ranks/communicators and CUDA thread shapes of the reference have no
 * meaning here and are not taken; np1=np2=np3=1 is implied. */
PPF_API int ppf_fft_poisson_plan_cuda_create(int n1, int n2, int n3,
                                     double L1, double L2, double L3,
                                     int pbc1, int pbc2, int pbc3);
/* cuda_Poisson_FFT_initial (fft_3d_poisson.f90:110-121). */
PPF_API int ppf_cuda_poisson_fft_initial(void);
/* cuda_Poisson_FFT_1D (fft_3d_poisson.f90:353-626): PRHS_d is read only. */
PPF_API int ppf_cuda_poisson_fft_1d(double *PRHS_d, double *P_d,
                            const double *dmx1_d, const double *dmx2_d,
                            const double *dmx3_d, const double *dx3_d);
/* cuda_Poisson_FFT_clean (fft_3d_poisson.f90:123-130). */
PPF_API int ppf_cuda_poisson_fft_clean(void);
/* Selects the precision of the module-global plan before
 * ppf_cuda_poisson_fft_initial (default PPF_FP64, the reference's). */
PPF_API int ppf_cuda_poisson_fft_set_precision(int precision, int max_sweeps);

#ifdef __cplusplus
}
#endif
#endif /* PPF_H */
