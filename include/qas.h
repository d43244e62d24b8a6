/*
 * qas.h -- C-ABI of libqas, the B200 (sm_100a) FP64 implementation of
 * qasMHD's per-step update.
 *
 * The reference exposes this path as non-virtual members of its dimension
 * classes (MHD1D / MHD2D / MHD3D, plus DMHD2D for the visco-resistive form)
 * operating in place on caller-owned host arrays in the layout
 *   val[m][ss], m = ro,mx,my,mz,bx,by,bz,en, ss = nx*(ny*k+j)+i,
 *   nx = XMESH+8 (4 ghost cells per side), bx/by/bz on the lower faces
 * (common/mhd_class.hpp:32-42, 2D/SERIAL/OTvortex/mhd2d_class.cpp:116-164).
 * Each entry point below names the reference member it replaces.
 *
 * Conventions
 *  - Every call returns qas_status; QAS_OK == 0.  No C++ exception crosses the ABI.
 *  - A context owns its device buffers and one CUDA stream on one device; calls on
 *    one context must come from one host thread at a time.  Distinct contexts are
 *    independent.
 *  - Host arrays stay owned by the caller.  Upload/download are synchronous.
 *  - Results are bit-identical to the reference CPU build for the same inputs.
 *  - Device-detected failures (non-positive density, non-finite values, a bounded
 *    device wait that ran out) latch in the context and are returned by the next call
 *    that synchronises (qas_sync, downloads, qas_run).
 */
#ifndef QAS_H
#define QAS_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QAS_ABI_VERSION 2

typedef enum {
  QAS_OK = 0,
  QAS_ERR_INVALID = 1,      /* bad argument (sizes, flags, null pointers)            */
  QAS_ERR_CUDA = 2,         /* CUDA runtime error (see qas_last_cuda_error)          */
  QAS_ERR_NOMEM = 3,        /* device (or host) allocation failed                    */
  QAS_ERR_NONFINITE = 4,    /* device check found rho<=0, p<=0 or a non-finite value */
  QAS_ERR_TIMEOUT = 5,      /* a bounded device-side wait gave up                    */
  QAS_ERR_UNSUPPORTED = 6,  /* combination not implemented                           */
  QAS_ERR_NO_DEVICE = 7,    /* no usable CUDA device                                 */
  QAS_ERR_IO = 8,           /* a file could not be written or read (message: qas_last_cuda_error) */
  QAS_ERR_HOST = 9          /* an exception in the library's host code, stopped at the C-ABI
                               (message: qas_last_cuda_error); no exception crosses the ABI */
} qas_status;

/* Grid: compile-time XMESH/YMESH/ZMESH of mymacros.hpp plus paras()'s spacing and gamma
 * (2D/SERIAL/OTvortex/mymacros.hpp:4-8, mhd2d_paras.cpp:3-39, common/mhd_class.hpp:20-24). */
typedef struct {
  int dim;               /* 1, 2 or 3                                           */
  int nxm, nym, nzm;     /* interior cells per axis (1 for unused axes)          */
  double dx, dy, dz;     /* cell sizes (unused axes ignored)                     */
  double gam;            /* specific-heat ratio (MHD::setgam)                    */
} qas_grid;

/* Scheme: RMN / ODR / R_K / CTW of mymacros.hpp (2D/SERIAL/OTvortex/mymacros.hpp:10-14).
 *   rmn: 0 Roe, 1 HLLD, 2 LHLLD, 3 MLAU  (riemann[] order, common/mhd_class.hpp:102-105)
 *   odr: 1..4 (interpol[ODR-1], l_interp, fcen, df1: common/mhd_class.hpp:107-113)
 *   rk : 1..3 SSP Runge-Kutta stages (rk_fac, mhd2d_solve.cpp:7)
 *   ctw: CUCT upwind weighting of the corner EMFs (mhd2d_solve.cpp:91-103)
 *   char_mode: face-value reconstruction of mhd_lrstate (common/mhd_func.c:108-161): 0 in
 *     characteristic variables with the mhd_eigen_mi/ae eigenvectors (the reference's active
 *     code, default); 1 in primitive variables, each field on its own (mhd_reconst,
 *     common/mhd_eigen.c:667-706, the reference's debug alternative); 2 in characteristic
 *     variables with the Athena-type eigenvectors of mhd_eigen_st for every state (mhd_c_reconst,
 *     common/mhd_eigen.c:5-173,436-511, the reference's third option).  Appended field: a
 *     zero-initialised struct keeps the default.  The adjoint takes 0 only. */
typedef struct {
  int rmn, odr, rk, ctw;
  int char_mode;
} qas_scheme;

/* Boundary flags per field and axis, the dnxs/dnys/dnzs arrays of common/mhd_class.hpp:40:
 * 0 periodic, +1 Neumann, -1 Dirichlet, +2 open, -2 zero-fixed (common/common_func.h:256-271). */
typedef struct {
  int dnx[8], dny[8], dnz[8];
} qas_bc;

typedef struct qas_ctx qas_ctx;

/* exec_() loop settings (mhd2d_class.cpp:35-61, mhd1d_class.cpp:32-53, mhd3d_class.cpp:48-76). */
typedef struct {
  int max_steps;     /* upper bound on steps taken by this call (<=0: no bound)                 */
  int flg;           /* exec_ flag: 1 = refresh dt by setdt every 2nd step, 0 = constant dt      */
  int stop_rule;     /* 0: run exactly max_steps; 1: exec_ rule n<nmax && tim<tmax (2D/3D);
                        2: 1D rule n<nmax with nmax = nrec*nout (mhd1d_class.cpp:24-29)          */
  double cfl;        /* CFL number (CFL macro)                                                   */
  double dtrec;      /* DTREC macro                                                              */
  int nout;          /* N_OUT macro; tmax = dtrec*nout                                           */
  int use_graph;     /* capture the step loop in a CUDA graph                                    */
  double nu0, eta0;  /* uniform viscosity / resistivity: when max(2nu0,eta0) > 1e-15 each step is
                        followed by the sub-cycled dissipative update of DMHD2D::exec_ /
                        DMHD3D::exec_ (2D and 3D) */
} qas_run_opts;

typedef struct {
  int steps;         /* steps taken by this call            */
  int n;             /* exec_'s step counter after the call  */
  int nmax;          /* nmax fixed by the first setdt        */
  double tim;        /* simulated time                       */
  double dt;         /* current dt                           */
} qas_run_info;

/* Library / device */
const char *qas_status_str(qas_status s);
int qas_abi_version(void);
const char *qas_last_cuda_error(void);

/* Context lifecycle.  Replaces the MHD{1,2,3}D constructor's array allocation and the
 * paras() settings (mhd2d_class.cpp:116-164, mhd2d_paras.cpp:3-39).  `device` < 0 uses
 * the current device. */
qas_status qas_create(qas_ctx **ctx, const qas_grid *grid, const qas_scheme *scheme, const qas_bc *bc, int device);
qas_status qas_destroy(qas_ctx *ctx);

/* Number of cells nd = nx*ny*nz including ghosts. */
qas_status qas_cells(const qas_ctx *ctx, long long *nd);

/* Copy the 8 host arrays val[0..7] (nd doubles each, reference layout incl. ghosts)
 * to / from the device.  Replaces the host-resident state of common/mhd_class.hpp:32-42. */
qas_status qas_upload(qas_ctx *ctx, double *const val[8]);
qas_status qas_download(qas_ctx *ctx, double *val[8]);
/* The derived arrays of common/mhd_class.hpp:34-37 (vx, vy, vz, pr into prim[0..3]; cell-centre
 * cx, cy, cz into cc[0..2]; NULL arrays or entries are skipped), evaluated from the current state
 * as prmtv() does at the start of ideal(): cell-centre B by fcen[ODR-1] with its ghost fill, then
 * v = m/ro, p from the energy (the gravity form subtracts ro*phi_g; the state is not modified). */
qas_status qas_primitives(qas_ctx *ctx, double *prim[4], double *cc[3]);
/* Same with one contiguous host block of 8*nd doubles (field m at block + m*nd). */
qas_status qas_upload_block(qas_ctx *ctx, const double *block);
qas_status qas_download_block(qas_ctx *ctx, double *block);
/* Asynchronous forms: the eight copies are queued on the context's stream behind the work
 * already there and the call returns without waiting; later calls on the context are ordered
 * after them.  The host block must stay valid -- and, for an upload, unchanged -- until
 * qas_sync returns; a download's values are there only then.  With pinned host memory
 * (cudaHostAlloc) the copies overlap the caller's host work; with pageable memory the driver
 * may finish them before the call returns.  The synchronous forms above are these plus
 * qas_sync. */
qas_status qas_upload_block_async(qas_ctx *ctx, const double *block);
qas_status qas_download_block_async(qas_ctx *ctx, double *block);
/* Device address of the context's state block (8*nd doubles, field-major); valid until
 * qas_destroy.  Lets device-resident callers (CUDA, PyTorch) share the state without copies. */
qas_status qas_device_state(qas_ctx *ctx, double **d_block);
/* The context's CUDA stream (cudaStream_t as void*). */
qas_status qas_stream(qas_ctx *ctx, void **stream);

/* Ghost fill of the 8 state fields: MHD2D::bound (mhd2d_class.cpp:3-9 -> bc2d,
 * common/common_func.c:60-138); 1D bc1d (:34-58); 3D single-rank mpi_sdrv3d +
 * mpi_x/y/zbc3d (mpi/common_mpi.c:198-525). */
qas_status qas_bound(qas_ctx *ctx);

/* One SSP-RK step of the ideal equations with the given dt, including the per-stage
 * ghost fill: MHD1D/2D/3D::ideal(dt) (1D/SERIAL/shock/mhd1d_solve.cpp:3-124,
 * 2D/SERIAL/OTvortex/mhd2d_solve.cpp:3-400, 3D/MPI/KHI/mhd3d_solve.cpp:3-729).
 * Like the reference, it does not fill the ghosts first: call qas_bound before. */
qas_status qas_step(qas_ctx *ctx, double dt);

/* setdt's reduction vmax = max(1, max over the interior of |v| + c_f) and the CFL
 * time step dt = cfl*dr/vmax (mhd2d_class.cpp:11-33, mhd1d_class.cpp:11-30,
 * mhd3d_class.cpp:15-46). */
qas_status qas_cfl_vmax(qas_ctx *ctx, double *vmax);
qas_status qas_cfl_dt(qas_ctx *ctx, double cfl, double *dt);

/* The exec_() stepping loop on the device: setdt(1) once (on the first call), then
 * { tim += dt; bound; ideal(dt); [dissipative sub-cycles]; setdt(flg*(n%2==0)) } per step,
 * with dt, tim, n and the stop test kept on the device (graph-captured when use_graph).
 * Output files of dout_() are not written. */
qas_status qas_run(qas_ctx *ctx, const qas_run_opts *opts, qas_run_info *info);
/* Reset exec_'s counters (n = 0, tim = 0, setdt(1) pending) without touching the state. */
qas_status qas_run_reset(qas_ctx *ctx);

/* One exec_ step on host arrays: the same result, bits and loop state as qas_upload_block(in)
 * + qas_run(opts, one step) + qas_download_block(out) -- the drop-in for a call of ideal()
 * (mhd2d_solve.cpp:3-400 via exec_, mhd2d_class.cpp:35-61) on the caller's val[] arrays, which
 * the reference updates in place (in == out is allowed).  In and out are blocks of 8*nd
 * doubles in the qas_upload_block layout, in host memory or in device memory.  From the second step of a run on, 2D and 3D contexts
 * without Hall, gravity or dissipation overlap the copies with the kernels: the last axis is
 * processed in windows of planes (QAS_OPT_PIPE_ITEMS), the upload of later ones runs beside the first
 * stage of earlier ones and the download of finished items beside the last stage of later
 * ones; pinned host memory is needed for the overlap.  The first such call allocates two
 * stage buffers (16 doubles per cell; when they do not fit, every call takes the serial
 * phases) and, when they fit, the work arrays of two more stage lanes (61 doubles per cell
 * each; without them the stages share one stream).
 * opts->max_steps is ignored (one step). */
qas_status qas_step_host(qas_ctx *ctx, const double *in, double *out, const qas_run_opts *opts, qas_run_info *info);
/* The plan of qas_step_host's wave along a last axis of `planes` padded planes (host only, no
 * GPU): `windows` as QAS_OPT_PIPE_ITEMS (0: the default), own_lanes = 1 for the ranges used when
 * every stage has a stream of its own (each plane computed once), 0 for the shared-stream ranges
 * (every item over its full halo).  *nitems items and the issue *lag; with out != NULL (room for
 * max_items items), QAS_PIPE_ITEM_INTS ints per item: nseg, ends (holds the ghost planes), then
 * for each of two segments nine [lo, hi) plane ranges: copied, updated, ghost-filled, primitives,
 * shock detector, in-plane face states and fluxes, last-axis face states (cells), last-axis
 * fluxes (faces), EMFs (empty ranges for a missing segment). */
#define QAS_PIPE_ITEM_INTS 38
qas_status qas_pipe_plan(int planes, int windows, int own_lanes, int *out, int max_items, int *nitems, int *lag);

/* Visco-resistive update with uniform coefficients: DMHD2D::setdc + the sub-cycled
 * dsptv of DMHD2D::exec_ (2D/SERIAL/MRX/dmhd2d_class.cpp:19-26, dmhd2d_solve.cpp:3-151),
 * and of DMHD3D::exec_ (3D/MPI/MRX/dmhd3d_class.cpp:20-28, dmhd3d_solve.cpp:3-179) in 3D.
 * qas_dsptv is one dsptv(dt) call (no ghost fill before).  2D and 3D (QAS_ERR_UNSUPPORTED
 * in 1D, which has no dissipative driver in the reference). */
qas_status qas_dissipate(qas_ctx *ctx, double dt, double nu0, double eta0);
/* Per-cell viscosity and resistivity profiles (the API's nu/eta arrays, common/mhd_class.hpp:
 * nd doubles each, host, reference layout; NULL for one of them = zero), as the reconnection
 * drivers' setdc fills them (2D/SERIAL/MRX/dmhd2d_init_.cpp:85-106, 3D/MPI/MRX/dmhd3d_init_.cpp:
 * 98-127): once installed, the dissipative step uses them -- rnu = 0.5*(ro*nu at the two cells),
 * eta averaged over the four cells around each edge, the sub-cycle count from their maximum of
 * max(2 nu, eta) -- and runs after every ideal step of qas_run; the scalar nu0/eta0 of the run
 * options and of qas_dissipate/qas_dsptv must then be 0 (QAS_ERR_INVALID otherwise).  Both
 * NULL removes them.  2D/3D only; a gravity context refuses them (no such driver). */
qas_status qas_set_dissipation(qas_ctx *ctx, const double *nu, const double *eta);
qas_status qas_dsptv(qas_ctx *ctx, double dt, double nu0, double eta0);

/* max over the interior of |D_x bx + D_y by + D_z bz| with the ODR-consistent
 * difference df1[ODR-1] (common/common_interp.h:17-24) scaled by 1/dx etc.; the CT
 * update keeps it at round-off (the check of 2D/SERIAL/python/batch.py:126-131). */
qas_status qas_max_divb(qas_ctx *ctx, double *maxdivb);

/* Wait for the context's stream and report any latched device error. */
qas_status qas_sync(qas_ctx *ctx);

/* Host-only diagnostics (no device needed): the ghost-fill map that qas_create builds for
 * group (0 state, 1 cell-centre B, 2 shock detector dv), field and axis.  src[i], fac[i]
 * for i < n (n = the axis extent incl. ghosts): after all fill passes of that axis, cell i
 * holds fac[i] * (value at src[i]).  Returns QAS_ERR_INVALID for flags the reference
 * leaves unset. */
qas_status qas_bc_map(const qas_grid *grid, const qas_bc *bc, int group, int field, int axis, int *src,
                      double *fac, int n);

/* Diagnostics: per-kernel device time measured live with CUDA events on the context's
 * stream.  Runs `nsteps` exec_ steps (the same work as qas_run, launched eagerly) with an
 * event pair around every kernel launch and returns, per kernel, the number of launches and
 * the summed durations.  *count receives the number of entries written (<= max_entries). */
typedef struct {
  char name[32];
  long long launches;
  double total_ms;
} qas_kernel_time;
qas_status qas_profile_run(qas_ctx *ctx, const qas_run_opts *opts, int nsteps, qas_kernel_time *out,
                           int max_entries, int *count);

/* Hall form of the 1D driver (1D/SERIAL/h-shock, HMHD1D): di = ion inertia length, de = the
 * "artificial" electron inertia length (absolute).  Each exec_ step then runs
 * hmax = 1 + (int)(dt/haldt) Hall sub-cycles hall_(dt/hmax), each followed by bound(),
 * between the ghost fill and ideal(dt) (hmhd1d_class.cpp:15-44; haldt: :3-13), with
 * vphix = di*pi/dx (hmhd1d_paras.cpp:29-34).  The sub-cycle count is read back each step, so
 * qas_run runs such a context without graph capture.  With de != 0 the by/bz fluxes of ideal()
 * and hall_() get the electron-inertia correction crcte: a conjugate-gradient solve of
 * (1 - de^2 d2/dx2) E = E_flux per flux (hmhd1d_solve.cpp:266-426), run in one CTA with the
 * reference's summation order.  QAS_ERR_UNSUPPORTED for dim != 1.
 * qas_hall: one hall_(dt) call (no ghost fill before), QAS_ERR_UNSUPPORTED without the Hall form. */
qas_status qas_set_hall(qas_ctx *ctx, double di, double de);
qas_status qas_hall(qas_ctx *ctx, double dt);

/* Gravity form of the 2D/3D drivers (2D/SERIAL/RTI, 3D/MPI/RTI: the API's phi_g,
 * common/mhd_class.hpp:39): phi_g = the gravitational potential of every padded cell (nd
 * doubles, host, reference layout), copied to the device; NULL switches gravity off.  With it
 * prmtv and setdt see en - ro*phi_g (and store (en - ro*phi_g) + ro*phi_g back, as the
 * drivers do), the energy flux carries flux_ro*0.5*(phi_L+phi_R), the momentum update the
 * source -rk_fac[rk][1]*ro*0.5*(phi(+1)-phi(-1))*dt/dx per axis, and every ghost fill of the
 * state sets the energy of the last axis' ghost layers from the first/last interior layer
 * (mhd2d_class.cpp:10-32 / mhd3d_class.cpp:14-40 of those drivers).  The state's en must
 * already include ro*phi_g, as the drivers' init_ leaves it.  QAS_ERR_UNSUPPORTED in 1D;
 * the dissipative and adjoint forms refuse a context with gravity (no such driver). */
qas_status qas_set_gravity(qas_ctx *ctx, const double *phi_g);

/* Tuning options (defaults are the measured best on B200).
 *   QAS_OPT_FUSED_SWEEP: 0 = reconstruction and Riemann flux of each direction in two
 *   kernels with the face states in HBM (default in 1D and 2D); 1 = one fused sweep kernel
 *   per direction, the face states kept on chip (default in 3D; 4th-order interpolation only,
 *   other orders keep the two kernels).
 *   QAS_OPT_LR_STAGING: 1 = the reconstruction stages its stencils in shared memory with
 *   TMA tensor copies (available for 2D/3D, 4th-order interpolation, even padded x extent;
 *   QAS_ERR_UNSUPPORTED otherwise); 0 = it reads them from global memory (default: measured
 *   faster on B200, where this kernel is bound by FP64 dependency latency, not by loads).
 * All forms give bit-identical results. */
#define QAS_OPT_FUSED_SWEEP 1
#define QAS_OPT_LR_STAGING 2
#define QAS_OPT_PIPE_ITEMS 3 /* windows of planes of qas_step_host's wave, 1..64 (default 32) */
#define QAS_OPT_PIPE_LANES 4 /* streams of qas_step_host's stages, 1..3 (default 3 when their work arrays
                                fit); set before the first qas_step_host of the context */
/* Failure-path hook for tests of the bounded waits: value >= 0 makes every CTA of the TMA-staged
 * reconstruction (QAS_OPT_LR_STAGING = 1) skip the load of its plane number `value`, with each
 * mbarrier wait bounded at 100 us instead of 2 s, so the wait for that plane runs out: the kernel
 * latches the error, waits for its own loads in flight, returns, and the next synchronising call
 * reports QAS_ERR_TIMEOUT (the state is then not a valid step).  value < 0 restores the defaults.
 * QAS_ERR_UNSUPPORTED where the staged form is not available. */
#define QAS_OPT_TEST_TMA_STALL 5
qas_status qas_set_option(qas_ctx *ctx, int option, int value);

/* Thread-block tile (tx*ty*tz <= 128 threads, tx a multiple of 32) of one cell kernel
 * ("k_prim", "k_dv", "k_lr", "k_flux", "k_emf", "k_update") or of all of them ("all"). */
qas_status qas_set_tile(qas_ctx *ctx, const char *kernel, int tx, int ty, int tz);
qas_status qas_get_tile(const qas_ctx *ctx, const char *kernel, int *tx, int *ty, int *tz);

/* Autotuner: for each cell kernel, time the candidate tiles over `trial_steps` exec_ steps
 * with CUDA events and keep the fastest.  The state, dt, time and step counter are restored
 * afterwards (results do not depend on the tile: every tile gives bit-identical states).
 * Choices are cached per (dim, ODR, RMN, grid-size bucket) for the life of the process. */
qas_status qas_autotune(qas_ctx *ctx, int trial_steps);

/* Diagnostics: measured FP64 throughput of the current device (TFLOP/s, FMA = 2 flops),
 * from independent DFMA chains on every SM timed with CUDA events; the FP64 roof of the
 * step's kernels. */
qas_status qas_fp64_peak(double *tflops);

/* Number of kernels this context has launched (eager launches plus kernels inside
 * replayed graphs), for launch accounting. */
qas_status qas_kernel_launches(const qas_ctx *ctx, long long *count);

/* ------------------------------------------------------------------------------------
 * Batched ensemble: many independent instances stepped by one set of kernel launches per
 * stage (one graph-captured launch sequence for the whole ensemble).  The reference runs
 * one simulation per process with a compile-time grid; this entry point has no counterpart
 * there beyond running many of its exec_() loops.  All instances share ODR and R_K; 2D and
 * 3D instances may be mixed (1D instances only with 1D ones: QAS_ERR_INVALID otherwise); grid
 * sizes, gamma, boundary flags, Riemann solver, CUCT flag and reconstruction are per instance.
 * Each instance keeps its own dt (setdt every 2nd step), time and step counter.
 * ------------------------------------------------------------------------------------ */
typedef struct qas_batch qas_batch;
qas_status qas_batch_create(qas_batch **batch, int n, const qas_grid *grids, const qas_scheme *schemes,
                            const qas_bc *bcs, int device);
qas_status qas_batch_destroy(qas_batch *batch);
qas_status qas_batch_cells(const qas_batch *batch, int instance, long long *nd);
/* state of one instance as one contiguous host block of 8*nd doubles (field-major) */
qas_status qas_batch_upload(qas_batch *batch, int instance, const double *block);
qas_status qas_batch_download(qas_batch *batch, int instance, double *block);
/* exec_ loops of every instance; info (n entries, may be NULL) receives each instance's counters */
qas_status qas_batch_run(qas_batch *batch, const qas_run_opts *opts, qas_run_info *info);
qas_status qas_batch_set_tile(qas_batch *batch, const char *kernel, int tx, int ty, int tz);
/* time candidate tiles per kernel over trial_steps steps (state restored) and keep the fastest */
qas_status qas_batch_autotune(qas_batch *batch, int trial_steps);
qas_status qas_batch_stream(qas_batch *batch, void **stream);
qas_status qas_batch_kernel_launches(const qas_batch *batch, long long *count);

/* ------------------------------------------------------------------------------------
 * The reference's on-disk formats for the context's state.
 * qas_dout: dout_() of MHD1D (1D/SERIAL/shock/mhd1d_class.cpp:57-95), MHD2D
 * (2D/SERIAL/OTvortex/mhd2d_class.cpp:63-114) and single-rank MHD3D
 * (3D/MPI/KHI/mhd3d_class.cpp:78-145) into directory `dir`: with n == 0 the header files
 * (params, offsets/xoff, mpinum in 3D, t, coordinates x_i = (i - 4 + 0.5) dx + origin[0] ...),
 * otherwise t.dat is appended; then outdat_<cnt>.dat (3D: outdat_<cnt>_00000.dat as float).
 * Asynchronous: the state is snapshot in the context's stream order and written by a host
 * thread while the caller keeps stepping; qas_dout_wait joins it and returns its status (a
 * new qas_dout first waits for the previous one).
 * qas_bkup_save / qas_bkup_load: bkup_save / bkup_load (common/common_func.c:280-344):
 * bkup_stamp.dat ("n cnt"), bkup_time.dat (tim, dt, trec), bkup_data_<rank>.dat.  As in the
 * reference, a missing stamp file is not an error: *loaded = 0 and nothing changes.
 * ------------------------------------------------------------------------------------ */
qas_status qas_dout(qas_ctx *ctx, const char *dir, int n, int cnt, double tim, const double *const coord[3]);
qas_status qas_dout_wait(qas_ctx *ctx);
qas_status qas_bkup_save(qas_ctx *ctx, const char *dir, int n, int cnt, double tim, double dt, double trec,
                         int rank);
qas_status qas_bkup_load(qas_ctx *ctx, const char *dir, int rank, int *loaded, int *n, int *cnt, double *tim,
                         double *dt, double *trec);

/* ------------------------------------------------------------------------------------
 * One domain split into slabs along its last axis (z in 3D, y in 2D), each slab a context on
 * its own GPU (or several on one): the reference's rank decomposition and halo driver
 * (mpi/common_mpi.c:198-525, mpi_sdrv3d + mpi_x/y/zbc3d; the MPI_Allreduce(MAX) of the CFL
 * speed in MHD3D::setdt, 3D/MPI/KHI/mhd3d_class.cpp:15-46) inside one process.  Ghost planes
 * whose source is another slab (internal boundaries, the wrap of a periodic axis) are copied
 * from it (peer copies between GPUs) after each ghost fill, after the primitives and after
 * the shock detector; the control block is replicated; results are bit-identical to the
 * single-domain context.  The split axis must be periodic for all 8 fields or physical for
 * all 8 (QAS_ERR_UNSUPPORTED otherwise), and each slab needs >= 8 planes.  Ideal MHD only
 * (QAS_ERR_UNSUPPORTED for nu0/eta0 > 0).
 * qas_dd_plan: the split (lo[0..nparts], global interior plane offsets) and the ghost-plane
 * copies of a decomposition, host only (no device needed).
 * devices: nparts CUDA device ordinals, or NULL for the current device.
 * Blocks: 8 fields over the GLOBAL padded grid, the layout of qas_upload_block.
 * ------------------------------------------------------------------------------------ */
typedef struct qas_dd qas_dd;
typedef struct {
  int part;       /* slab whose ghost planes are written               */
  int src_part;   /* slab that holds the source planes                 */
  int src_plane;  /* first source plane (padded index along the axis)  */
  int dst_plane;  /* first ghost plane                                 */
  int nplanes;    /* always 4                                          */
} qas_dd_copy;
qas_status qas_dd_plan(const qas_grid *grid, const qas_bc *bc, int nparts, int *lo, qas_dd_copy *copies,
                       int max_copies, int *ncopies);
qas_status qas_dd_create(qas_dd **dd, const qas_grid *grid, const qas_scheme *scheme, const qas_bc *bc, int nparts,
                         const int *devices);
qas_status qas_dd_destroy(qas_dd *dd);
qas_status qas_dd_upload_block(qas_dd *dd, const double *block);
qas_status qas_dd_download_block(qas_dd *dd, double *block);
qas_status qas_dd_run(qas_dd *dd, const qas_run_opts *opts, qas_run_info *info);
qas_status qas_dd_parts(const qas_dd *dd, int *nparts);
qas_status qas_dd_kernel_launches(const qas_dd *dd, long long *kernels, long long *copies);

/* ------------------------------------------------------------------------------------
 * Discrete adjoint of the 2D step (no counterpart in the reference, which has no
 * derivatives): the exec_ step body -- bound(), ideal(dt) (MHD2D::ideal,
 * 2D/SERIAL/OTvortex/mhd2d_solve.cpp:3-400) and, with eta0 > 0, setdc + the sub-cycled
 * DMHD2D::dsptv (2D/SERIAL/MRX/dmhd2d_class.cpp:19-26) with uniform eta and nu = 0 --
 * for RMN = Roe, ODR = 4 (characteristic WCNS4), any R_K, CTW and valid boundary flags.
 *
 * qas_adjoint_forward runs `nsteps` steps from the current device state with the given
 * dt per step (dts[nsteps], host), keeping a snapshot every `ckpt_every` steps; the state
 * afterwards is the final state (bit-identical to qas_run with the same dt sequence).
 * qas_adjoint_backward takes dL/d(final state) (host, 8*nd doubles, field-major like
 * qas_download_block) and returns dL/d(initial state) in the same layout and dL/deta0
 * (may be NULL).  It recomputes each checkpoint segment with its intermediates recorded
 * on a device tape and reverses it; dt and the sub-cycle counts are held fixed.  The
 * context's state is the forward run's final state again when it returns.
 * Status: QAS_ERR_UNSUPPORTED for other dims/solvers/orders or more than 8 sub-cycles,
 * QAS_ERR_INVALID for a backward call without a forward run.
 * ------------------------------------------------------------------------------------ */
qas_status qas_adjoint_forward(qas_ctx *ctx, int nsteps, int ckpt_every, const double *dts, double eta0);
qas_status qas_adjoint_backward(qas_ctx *ctx, const double *dldu_final, double *dldu0, double *dldeta0);
/* Both in one call, for a loss whose gradient with respect to the final state is known before
 * the run (a loss linear in the final state, such as a weighted sum of its fields):
 * qas_adjoint_forward, then qas_adjoint_backward with dldu_final; same results, same status. */
qas_status qas_adjoint_run(qas_ctx *ctx, int nsteps, int ckpt_every, const double *dts, double eta0,
                           const double *dldu_final, double *dldu0, double *dldeta0);

/* ------------------------------------------------------------------------------------
 * Allocation-free max |div B| (no counterpart in the reference, whose caller owns host
 * arrays and never allocates device memory): the same value as qas_max_divb, for a state
 * the caller already holds in device memory, without a context and without allocating.
 * It serves callers whose device memory is all handed to an arena or caching allocator
 * under a fixed budget (a framework's memory pool), where a library cudaMalloc would fail
 * or eat into that budget.  It is a synchronous host query: it ends with a device-to-host
 * copy of the result and synchronises `stream`.
 * d_state: 8 fields of the reference's ghost-padded layout, field m at d_state +
 * m*field_stride (field_stride >= nd); stream: a cudaStream_t (NULL = default stream).
 * Scratch is a static 512 KiB device array (every device that loads the library holds it
 * until exit) sized for QAS_NOALLOC_MAX_ROWS interior rows (nym*nzm); larger grids return
 * QAS_ERR_UNSUPPORTED with the reason in qas_last_cuda_error().  The first call on a device
 * loads the module (which may allocate): make it before the allocation-free section.  An
 * error already pending on the calling thread is returned (QAS_ERR_CUDA) and left pending.
 * Calls that overlap in time on one device share the scratch and race: serialise them.
 * ------------------------------------------------------------------------------------ */
#define QAS_NOALLOC_MAX_ROWS 65536
qas_status qas_max_divb_noalloc(const qas_grid *grid, int odr, const double *d_state, long long field_stride,
                                void *stream, double *maxdivb);

#ifdef __cplusplus
}
#endif
#endif
