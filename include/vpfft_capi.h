/*
 * vpfft_capi.h -- C ABI of vpfft_b200, a B200 (sm_100a) implementation of
 * VPFFT's fixed-point solve on a periodic 3D voxel polycrystal.
 *
 * Plain C types only (pointers, sizes, doubles); no exceptions cross this
 * boundary and nothing calls exit(): every entry point returns a vpfft_status.
 * Host arrays are caller-owned and only read or written during the call.
 *
 * Layout conventions (the reference's, so arrays written for it can be passed
 * unchanged):
 *   voxel index        v = x*Ny*Nz + y*Nz + z            (MaterialGrid.h:121-124)
 *   orientation R      9 doubles per voxel, row-major 3x3 (SMatrix3x3, LinearAlgebra.h:114)
 *   5-vectors          deviatoric basis coefficients      (EigenRep, LinearAlgebra.h:298-521;
 *                      basis EigenBasis, LinearAlgebra.h:207-247)
 *   5x5 matrices       column-major m[j*5+i]              (SMatrix5x5, LinearAlgebra.h:574)
 *   per-voxel arrays   voxel-major: R[v*9+k], sigma[v*5+c], crss[v*12+s]
 *
 * Threading: a vpfft_grid is bound to the CUDA device current at creation and
 * owns one CUDA stream; it is not thread-safe.  Different grids may be used
 * from different threads.
 */
#ifndef VPFFT_CAPI_H
#define VPFFT_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VPFFT_NUM_SLIP_SYSTEMS 12

typedef enum {
  VPFFT_OK = 0,
  VPFFT_ERR_INVALID_ARGUMENT = 1,
  VPFFT_ERR_UNSUPPORTED_SIZE = 2, /* a grid dimension is not a product of 2, 3 and 5, or > 512 */
  VPFFT_ERR_CUDA = 3,             /* a CUDA runtime call failed; see vpfft_last_error() */
  VPFFT_ERR_OUT_OF_MEMORY = 4,
  VPFFT_ERR_NO_DEVICE = 5,        /* no usable CUDA device: there is no CPU fallback */
  VPFFT_ERR_MAX_RSS_TINY = 6,     /* a voxel's max resolved shear stress < 1e-10
                                     (the reference exits: MaterialGrid.h:560-564,
                                     MaterialGrid.cpp:186-190) */
  VPFFT_ERR_NONFINITE = 7,        /* NaN/Inf produced (e.g. singular reference medium) */
  VPFFT_ERR_NOT_INITIALIZED = 8,  /* fields not set before a solve */
  VPFFT_ERR_IO = 9,               /* file could not be read or parsed */
  VPFFT_ERR_CANCELLED = 10,
  /* 11 is not used */
  VPFFT_ERR_BUSY = 12             /* the grid has a request in flight in a batch */
} vpfft_status;

/* Bits of vpfft_stats.status_bits and vpfft_batch_result.status_bits: what a
 * solve that returned VPFFT_OK still reports.  The reference's paths for the
 * last two are silent (the fixed-point loop ends at NumMaxIterations with no
 * flag, MaterialGrid.cpp:1046-1068; a voxel's NR returns its last iterate at
 * its cap, Solvers.cpp:167-170, 213-221). */
#define VPFFT_STATUS_MAX_RSS_TINY 0x1       /* a voxel's max resolved shear < 1e-10 (the call fails) */
#define VPFFT_STATUS_NONFINITE 0x2          /* NaN/Inf appeared (the call fails) */
#define VPFFT_STATUS_DEVICE_TIMEOUT 0x4     /* a bounded device-side wait gave up (the call
                                               fails with VPFFT_ERR_CUDA) */
#define VPFFT_STATUS_LOOP_NOT_CONVERGED 0x100 /* the loop stopped at max_iter with delta_sigma
                                               or delta_eps above eps */
#define VPFFT_STATUS_NR_CAPPED 0x200        /* some voxel's Newton-Raphson solve stopped at its
                                               iteration cap (count: nr_not_converged) */

typedef enum {
  VPFFT_PREC_FP64 = 0,  /* everything in FP64: the GPU oracle path */
  VPFFT_PREC_MIXED = 1  /* FP32 fields, FFT and Green operator; an FP32 Newton predictor
                           whose stress an FP64 residual certifies, else an FP64 Newton
                           step (FP64 residual and Jacobian); FP64 reductions with a
                           compensated final sum (vpfft_solver_options.mixed_certify_step) */
} vpfft_precision;

/* Per-slip-system material constants.  The reference hard-codes them in
 * MaterialGrid::InitializeMemory (MaterialGrid.cpp:322-336, 390); the
 * defaults below (vpfft_material_default) are those values. */
typedef struct {
  double gamma_dot_base[VPFFT_NUM_SLIP_SYSTEMS];  /* reference rate, default 15.5 */
  int32_t rate_sensitivity[VPFFT_NUM_SLIP_SYSTEMS]; /* power-law exponent n, default 10 */
  double crss[VPFFT_NUM_SLIP_SYSTEMS];            /* initial CRSS tau_s, default 11 */
  double tau0[VPFFT_NUM_SLIP_SYSTEMS];            /* Voce tau0, default 11 */
  double tau1[VPFFT_NUM_SLIP_SYSTEMS];            /* Voce tau1, default 11 */
  double theta0[VPFFT_NUM_SLIP_SYSTEMS];          /* Voce theta0, default 430 */
  double theta1[VPFFT_NUM_SLIP_SYSTEMS];          /* Voce theta1, default 110 */
  double hardening[VPFFT_NUM_SLIP_SYSTEMS * VPFFT_NUM_SLIP_SYSTEMS]; /* h[s*12+t], default 1 */
} vpfft_material;

/* Newton-Raphson and fixed-point constants.  The reference hard-codes them
 * (MaterialGrid.cpp:159-160, 909-911); defaults are those values. */
typedef struct {
  double init_nr_epsilon;     /* 5e-4  (InitializeComputation) */
  int32_t init_nr_max_iter;   /* 1000 */
  double nr_epsilon;          /* 5e-4  (fixed-point loop) */
  double nr_max_resolved;     /* 1e9 */
  int32_t nr_max_iter;        /* 100 */
  int32_t green_operator;     /* the x pass's Green operator (no counterpart in the reference,
                                 which recomputes it per wave vector, MaterialGrid.cpp:682-743):
                                 0 (default) = chosen per grid size: where a stored table of the
                                 operator's costly part (10 values per wave vector of the half
                                 spectrum) would take at most 512 MiB, the first solve of that
                                 size times the x pass computing the operator against one
                                 reading the table and keeps the faster
                                 (vpfft_grid_green_operator); 1 = always compute; 2 = always
                                 store (rebuilt at each fixed-point loop, since L0 and the voxel
                                 lengths change per increment).  All three give the same bits. */
  double mixed_certify_step;  /* VPFFT_PREC_MIXED only (no counterpart in the reference): after
                                 the FP32 Newton predictor, the FP64 residual at the predicted
                                 stress gives an estimate of the Newton step still to take; where
                                 it is at most this fraction of |sigma| the predicted stress is
                                 kept with its FP64 strain rate, elsewhere the FP64 Newton step
                                 (FP64 residual and Jacobian) is taken.  Default 1e-5; 0 always
                                 takes the step. */
} vpfft_solver_options;

typedef struct {
  int32_t iterations;         /* fixed-point iterations executed */
  int32_t converged;          /* 1 when both error norms fell below epsilon */
  double stress_error;        /* final delta_sigma (MaterialGrid.cpp:1052) */
  double strain_rate_error;   /* final delta_eps   (MaterialGrid.cpp:1053) */
  double avg_strain_rate[5];  /* <edot> of the last iteration */
  int64_t nr_not_converged;   /* voxel-iterations whose NR hit its cap */
  int32_t status_bits;        /* OR of VPFFT_STATUS_* bits */
  int32_t pad_;
  double seconds_init;        /* InitializeComputation + reference medium */
  double seconds_loop;        /* the fixed-point loop */
  double seconds_post;        /* texture, voxel length, hardening */
  double L0[25];              /* reference medium of the increment, column-major */
  int64_t nr_fp64_steps;      /* mixed precision: voxel-iterations that took the FP64 Newton
                                 step (the others kept the FP32 predictor's stress, certified by
                                 the FP64 residual; vpfft_solver_options.mixed_certify_step) */
} vpfft_stats;

typedef enum {
  VPFFT_FIELD_STRESS = 0,          /* N x 5   Stress(x,y,z)            MaterialGrid.h:166-173 */
  VPFFT_FIELD_LAGRANGE = 1,        /* N x 5   LagrangeMultiplier       MaterialGrid.h:178-185 */
  VPFFT_FIELD_ORIENTATION = 2,     /* N x 9   Orientation              MaterialGrid.h:129-136 */
  VPFFT_FIELD_CRSS = 3,            /* N x 12  CRSS                     MaterialGrid.h:431-434 */
  VPFFT_FIELD_ACCUMULATED_SHEAR = 4, /* N     AccumulatedShear         MaterialGrid.h:293 */
  VPFFT_FIELD_POLARIZATION = 5,    /* N x 5   Re PolarizationField of the last iteration */
  VPFFT_FIELD_STRAIN_RATE_VARIATION = 6, /* N x 5 Re DisplacementVariation (d~) of the last iteration */
  VPFFT_FIELD_STRAIN_RATE = 7,     /* N x 5   ApplyConstitutiveEquations(sigma) */
  VPFFT_FIELD_SCHMID = 8           /* N x 60  SchmidtTensorList (12 x 5 per voxel) */
} vpfft_field;

typedef struct vpfft_grid vpfft_grid;

/* ------------------------------------------------------------------ library */
const char *vpfft_version(void);
const char *vpfft_status_string(vpfft_status s);
/* number of usable CUDA devices (0 on a machine without a GPU) */
int vpfft_device_count(void);
void vpfft_material_default(vpfft_material *m);
void vpfft_solver_options_default(vpfft_solver_options *o);

/* ------------------------------------------------------------------ MaterialGrid
 * Replaces VPFFT::DataStructures::MaterialGrid (MaterialGrid.h:59-577).     */

/* MaterialGrid(int DimX, int DimY, int DimZ) (MaterialGrid.h:72-78) + InitializeMemory
 * (MaterialGrid.cpp:312-394).  material/options may be NULL for the defaults. */
vpfft_status vpfft_grid_create(int nx, int ny, int nz, const vpfft_material *material,
                               const vpfft_solver_options *options, vpfft_precision precision,
                               vpfft_grid **out);
/* The reference never frees (no destructor; Cleanup is private and unused,
 * MaterialGrid.cpp:287-305). */
vpfft_status vpfft_grid_destroy(vpfft_grid *g);
/* NumX/NumY/NumZ (MaterialGrid.h:235-237) */
vpfft_status vpfft_grid_dims(const vpfft_grid *g, int *nx, int *ny, int *nz);
/* SendDataAndInitialize(SMatrix3x3*, EigenRep*) (MaterialGrid.cpp:425-534):
 * copies orientations (N x 9) and stresses (N x 5, may be NULL = zeros) to the
 * device and resets CRSS to the material's initial values. */
vpfft_status vpfft_grid_set_fields(vpfft_grid *g, const double *orientations,
                                   const double *stress);
/* Same, from device pointers already holding the arrays (FP64, same layout). */
vpfft_status vpfft_grid_set_fields_device(vpfft_grid *g, const double *d_orientations,
                                          const double *d_stress);
/* SetVoxelLength (MaterialGrid.h:97-102) */
vpfft_status vpfft_grid_set_voxel_length(vpfft_grid *g, double hx, double hy, double hz);
vpfft_status vpfft_grid_get_voxel_length(const vpfft_grid *g, double h[3]);
/* Per-voxel CRSS (N x 12) or NULL to reset to the material's uniform values
 * (LocalCRSS, MaterialGrid.cpp:384-391). */
vpfft_status vpfft_grid_set_crss(vpfft_grid *g, const double *crss);
/* Read any field to a host buffer (see vpfft_field for sizes); FP32 fields
 * are widened to double. */
vpfft_status vpfft_grid_get_field(vpfft_grid *g, vpfft_field which, double *dst);
/* Write a field from a host buffer (snapshot/restore). */
vpfft_status vpfft_grid_set_field(vpfft_grid *g, vpfft_field which, const double *src);
/* Checkpoint of a whole grid.  The reference's MaterialGrid has none: its only
 * saved state is the text pair WriteRandomMaterial / ReadRandomMaterial
 * (UnitTester.cpp:116-167: orientation and stress).  A snapshot holds every
 * state a later call reads -- stress, Lagrange multiplier, orientation,
 * polarization, accumulated shear, per-voxel CRSS once hardening has run,
 * voxel lengths, L0 and the last macroscopic strain rate -- as FP64 (FP32
 * fields widen exactly), so a grid restored from it continues bit for bit as
 * the original would.  vpfft_grid_snapshot_size gives the bytes (a header plus
 * 25 or 37 doubles per voxel); vpfft_grid_restore accepts a snapshot of a
 * grid of the same dimensions and precision only.  A restore that fails after
 * its header checks (a CUDA error while the fields are copied) leaves the grid
 * without fields or reference medium: restore it again, or set its fields,
 * before the next solve (which otherwise returns VPFFT_ERR_NOT_INITIALIZED). */
vpfft_status vpfft_grid_snapshot_size(const vpfft_grid *g, size_t *bytes);
vpfft_status vpfft_grid_snapshot(vpfft_grid *g, void *buf, size_t cap);
vpfft_status vpfft_grid_restore(vpfft_grid *g, const void *buf, size_t size);

/* RunSingleStrainStep(Edot, NumMaxIterations, TimeStep, ConvergenceEpsilon) -> <sigma>
 * (MaterialGrid.cpp:897-1084).  stats may be NULL. */
vpfft_status vpfft_run_single_strain_step(vpfft_grid *g, const double edot[5], int max_iter,
                                          double dt, double eps, double avg_stress_out[5],
                                          vpfft_stats *stats);

/* Callback after every increment of vpfft_run: step index, accumulated macroscopic
 * strain and <sigma> (the row RunVPFFT writes to Stress_Strain.txt,
 * MaterialGrid.cpp:1217-1226).  Return nonzero to stop. */
typedef int (*vpfft_step_callback)(int step, const double strain5[5], const double stress5[5],
                                   void *user);
/* RunVPFFT (MaterialGrid.cpp:1202-1228).  If stress_strain_path is not NULL the
 * same text file as the reference is written there. */
vpfft_status vpfft_run(vpfft_grid *g, const double edot[5], int max_iter, int n_steps, double dt,
                       double eps, const char *stress_strain_path, vpfft_step_callback cb,
                       void *user);

/* --- phases of RunSingleStrainStep, for drivers that time or script them --- */
/* InitializeComputation (MaterialGrid.cpp:153-210) */
vpfft_status vpfft_initialize_computation(vpfft_grid *g, const double edot[5]);
/* BuildLinearRefMediumStiffness (MaterialGrid.cpp:219-282); L0 out column-major */
vpfft_status vpfft_build_reference_medium(vpfft_grid *g, double L0_out[25]);
/* The fixed-point loop body (MaterialGrid.cpp:930-1068) run until convergence or
 * max_iter; needs the two phases above first.  history (may be NULL) receives
 * 12 doubles per iteration: <sigma>(5), <edot>(5), delta_sigma, delta_eps. */
vpfft_status vpfft_fixed_point(vpfft_grid *g, const double edot[5], int max_iter, double eps,
                               double *history, vpfft_stats *stats);
/* OrientationEvolutionWithFFT + UpdateVoxelLength + UpdateHardeningCRSS
 * (MaterialGrid.cpp:1074-1080, 769-876, 1190-1196, 1127-1157) */
vpfft_status vpfft_post_increment(vpfft_grid *g, const double edot[5], double dt);
/* Blocks until the grid's stream is idle. */
vpfft_status vpfft_grid_synchronize(vpfft_grid *g);
/* The grid's CUDA stream (a cudaStream_t), for callers that time with events. */
void *vpfft_grid_stream(vpfft_grid *g);
/* Count of this library's kernel launches on the grid so far. */
int64_t vpfft_grid_launch_count(const vpfft_grid *g);
/* Device time per kernel of the fixed-point loop, measured with CUDA events on
 * the grid's stream while profiling is enabled (enabling resets the sums).
 * Phases: 0 fft_z_r2c, 1 fft_y_forward, 2 fft_x_green, 3 fft_y_inverse,
 * 4 fft_z_c2r, 5 nr_update, 6 iter_finish.  The reference has no
 * profiling (README.make:40-44 lists it as a TODO). */
#define VPFFT_NUM_PHASES 7
vpfft_status vpfft_grid_set_profiling(vpfft_grid *g, int enabled);
vpfft_status vpfft_grid_phase_times(const vpfft_grid *g, double *ms_total, int64_t *launches);
const char *vpfft_phase_name(int phase);
/* The Green operator in use (vpfft_solver_options.green_operator): *mode = 1
 * computed per wave vector, 2 read from the stored table, 0 not chosen yet;
 * ms_compute / ms_table (may be NULL) get the x pass's times measured when the
 * choice was made (0 where not timed). */
vpfft_status vpfft_grid_green_operator(const vpfft_grid *g, int *mode, double *ms_compute,
                                       double *ms_table);
/* Last error message of the grid (or of the library when g is NULL). */
const char *vpfft_last_error(const vpfft_grid *g);

/* ------------------------------------------------------------------ Solvers
 * Batched device versions of the per-voxel routines of VPFFT::Solvers
 * (Solvers.h:51-153).  All arrays are host arrays of n voxels; schmid is
 * n x 12 x 5, crss n x 12.  They run on the current CUDA device.        */

/* SolveConstitutiveEquations (Solvers.cpp:19-101) */
vpfft_status vpfft_solve_constitutive(int n, const double *stress0, const double *schmid,
                                      const double *crss, const vpfft_material *m,
                                      const double edot[5], double eps, double max_rss,
                                      int max_iter, double *stress_out);
/* SolveConstrainedConstitutiveEquations (Solvers.cpp:111-222); L0 column-major;
 * nr_error (may be NULL) gets NR_Error_Out per voxel. */
vpfft_status vpfft_solve_constrained_constitutive(int n, const double *stress0,
                                                  const double *schmid, const double *crss,
                                                  const vpfft_material *m, const double edot[5],
                                                  const double *lambda, const double *dtilde,
                                                  const double L0[25], double eps,
                                                  double max_rss, int max_iter,
                                                  double *stress_out, double *nr_error);
/* The same constrained solve, with NO device memory allocation.  No
 * counterpart in the reference.  For callers that cannot allocate: a
 * macro-scale driver calling the point solve from inside its own Newton loop
 * typically gives the device to its own memory pool, where a cudaMalloc can
 * fail and every cudaFree synchronises the device.  The arrays are staged in
 * a fixed device array of VPFFT_NOALLOC_MAX_POINTS points (2.9 MiB per
 * device); larger n returns VPFFT_ERR_UNSUPPORTED_SIZE.
 * The first call on each device (n = 0 is enough) sets up: it looks up the
 * array's address and has the CUDA runtime load the array and this call's
 * kernels, which under the runtime's default lazy module loading allocates
 * about 3 MiB of device memory.  Make that first call before the caller's
 * memory pool reserves the device; later calls allocate nothing.
 * Every call runs its copies and kernels on the legacy default stream: no call
 * may overlap a stream capture anywhere in the process (on any device), and a
 * call is ordered after the work of the caller's blocking streams (streams
 * made with plain cudaStreamCreate); only streams created with
 * cudaStreamNonBlocking are not stalled.  Calls share the array, so they are
 * serialised by a process-wide lock (overlapping calls would otherwise race on
 * it).  A call returns when its results are on the host.
 * not_converged (may be NULL) gets the number of points whose NR error is not
 * below eps. */
#define VPFFT_NOALLOC_MAX_POINTS 4096
vpfft_status vpfft_solve_constrained_constitutive_noalloc(
    int n, const double *stress0, const double *schmid, const double *crss,
    const vpfft_material *m, const double edot[5], const double *lambda, const double *dtilde,
    const double L0[25], double eps, double max_rss, int max_iter, double *stress_out,
    double *nr_error, int64_t *not_converged);
/* ApplyConstitutiveEquations (Solvers.cpp:255-274) */
vpfft_status vpfft_apply_constitutive(int n, const double *stress, const double *schmid,
                                      const double *crss, const vpfft_material *m,
                                      double *strain_rate_out);
/* SolveSachEquation (Solvers.cpp:230-243) */
vpfft_status vpfft_solve_sachs(int n, const double *schmid, const double *crss,
                               const double edot[5], double *stress_out);
/* UpdateSchmidtTensors for n orientations (MaterialGrid.cpp:107-124): n x 9 -> n x 60 */
vpfft_status vpfft_schmid_tensors(int n, const double *orientations, double *schmid_out);
/* The symmetrised, projected Green operator applied to n complex 5-vectors at
 * wave-vector indices (ix,iy,iz) of an nx x ny x nz grid with voxel lengths h,
 * including the Nyquist-plane override and the Hermitian average of k and -k
 * that the reference's "real part of a c2c transform" amounts to
 * (MaterialGrid.cpp:682-743, 583-615).  phat/dhat: n x 5 x 2 (re, im). */
vpfft_status vpfft_green_apply(int n, const int32_t *k_index, int nx, int ny, int nz,
                               const double h[3], const double L0[25], const double *phat,
                               double *dhat, vpfft_precision precision);

/* ------------------------------------------------------------------ FFT
 * The device 3D real<->half-complex transform used by the solve, exposed for
 * testing: forward is unnormalised (FFTW_FORWARD sign), inverse divides by N.
 * real: n_comp x N (component-major); spec: n_comp x nx x ny x (nz/2+1) x 2. */
vpfft_status vpfft_fft3d_r2c(int nx, int ny, int nz, int n_comp, const double *real,
                             double *spec, vpfft_precision precision);
/* Tile movement of the FP32 forward y pass: 1 moves the tiles
 * of y lines of 64, 128 or 256 points with the Tensor Memory Accelerator
 * (bulk tensor copies on mbarriers), 0 uses the warp-copy pass for every
 * size (the default); -1 only queries.  Both give the same bits.  Returns the previous
 * setting.  Process-wide; a tuning and diagnostic switch with no counterpart
 * in the reference. */
int vpfft_set_tma_passes(int enable);
vpfft_status vpfft_fft3d_c2r(int nx, int ny, int nz, int n_comp, const double *spec,
                             double *real, vpfft_precision precision);

/* ------------------------------------------------------------------ fixtures
 * Host-only generators of synthetic microstructures (no GPU needed). */
/* Periodic Voronoi polycrystal: n_grains seeds uniform in [0,nx)x[0,ny)x[0,nz),
 * each voxel takes the orientation of the nearest seed under the minimum-image
 * distance (ties -> lower seed index); orientations are uniform on SO(3) by
 * Shoemake's method.  Pseudo-random numbers: SplitMix64 seeded with `seed`.
 * orientations_out: N x 9; grain_out (may be NULL): N int32 seed index. */
vpfft_status vpfft_fixture_polycrystal(int nx, int ny, int nz, int n_grains, uint64_t seed,
                                       double *orientations_out, int32_t *grain_out);
/* EigenRep(SMatrix3x3) of a velocity gradient (LinearAlgebra.h:307-312): only
 * the symmetric part survives the projection. */
void vpfft_edot_from_matrix(const double L[9], double edot_out[5]);
/* EigenRep::ToMatrixRep (LinearAlgebra.h:352-360) */
void vpfft_matrix_from_edot(const double edot[5], double L_out[9]);

/* ------------------------------------------------------------------ batches
 * Many RVEs (grids of possibly different sizes) advanced together: every
 * phase of an increment (initialisation, reference medium, the five FFT
 * passes with the Green operator, the Newton-Raphson sweep, the reductions,
 * the texture/hardening update) is ONE kernel launch over all RVEs in that
 * phase, and the fixed-point iterations of a tick are replayed from a captured
 * CUDA graph while the set of iterating RVEs is unchanged.  The reference has
 * no counterpart (it solves one RVE per MPI job); each request is one
 * RunSingleStrainStep (MaterialGrid.cpp:897-1084) on a caller-owned grid,
 * whose fields and texture persist across requests.
 *
 * Continuous batching: vpfft_batch_step runs one tick -- requests that arrived
 * since the last tick are admitted while a slot is free and their spectra fit
 * the HBM budget (FIFO; a request waits while its grid has one in flight),
 * newly admitted RVEs are initialised while the others iterate, converged RVEs
 * get their post-increment update and are reported by vpfft_batch_poll.  A
 * batch is bound to the device current at creation and is not thread-safe. */
typedef struct vpfft_batch vpfft_batch;
typedef struct {
  int32_t max_slots;            /* RVEs in flight at once (default 256) */
  int32_t iterations_per_tick;  /* fixed-point iterations enqueued per tick (default 8) */
  int64_t hbm_budget_bytes;     /* device memory for in-flight spectra (default 8 GiB) */
  int32_t use_graphs;           /* replay the tick's iterations from a CUDA graph (default 1) */
  int32_t fft_tiles;            /* tile family of the batched FFT passes: -1 (the default) =
                                   autotuned per RVE size: the first admission of a size times
                                   the five-pass chain in every family and keeps the fastest
                                   (vpfft_batch_get_tunings); 0, 1, 2 = tiles of about 512,
                                   1024, 2048 complex values per buffer (clamped per axis to
                                   the longest its line engine has).  A family only regroups
                                   lines into blocks and every family performs the same
                                   operations, so results are the same bit for bit in every
                                   family, in both precisions, and as the single-grid path. */
} vpfft_batch_options;
typedef struct {
  int64_t request_id;
  int32_t status;               /* vpfft_status of the request */
  int32_t iterations;           /* fixed-point iterations executed */
  int32_t converged;
  int32_t status_bits;          /* OR of VPFFT_STATUS_* bits */
  double avg_stress[5];         /* <sigma> of the last iteration (the step's return value) */
  double stress_error;          /* final delta_sigma */
  double strain_rate_error;     /* final delta_eps */
  int64_t nr_not_converged;     /* voxel-iterations whose NR hit its cap */
  double seconds_queued;        /* submit -> admission */
  double seconds_total;         /* submit -> completion (after the tick that finished it) */
} vpfft_batch_result;
typedef struct {
  int64_t queued, active, completed;
  int64_t ticks, graph_replays, kernel_launches;
  int64_t arena_bytes_in_use, arena_bytes;
  int64_t admissions_deferred_for_memory;  /* ticks at which the head request did not fit */
} vpfft_batch_info;
void vpfft_batch_options_default(vpfft_batch_options *o);
vpfft_status vpfft_batch_create(vpfft_precision precision, const vpfft_material *material,
                                const vpfft_solver_options *options,
                                const vpfft_batch_options *batch_options, vpfft_batch **out);
vpfft_status vpfft_batch_destroy(vpfft_batch *b);
/* Queue one increment (RunSingleStrainStep) on grid g, which must have the
 * batch's precision, material and solver options and its fields set.  The
 * grid belongs to the batch until the request completes (other calls on it
 * return VPFFT_ERR_BUSY). */
vpfft_status vpfft_batch_submit(vpfft_batch *b, vpfft_grid *g, const double edot[5], int max_iter,
                                double dt, double eps, int64_t *request_id);
/* One tick; *pending (may be NULL) = queued + active requests afterwards. */
vpfft_status vpfft_batch_step(vpfft_batch *b, int *pending);
/* Ticks until every submitted request has completed. */
vpfft_status vpfft_batch_run(vpfft_batch *b);
/* Completed requests since the last poll, oldest first (at most cap). */
vpfft_status vpfft_batch_poll(vpfft_batch *b, vpfft_batch_result *out, int cap, int *n_out);
/* A queued request is dropped; an active one stops at the next tick with its
 * grid as the last executed iteration left it (no texture/hardening update).
 * Both complete with status VPFFT_ERR_CANCELLED. */
vpfft_status vpfft_batch_cancel(vpfft_batch *b, int64_t request_id);
vpfft_status vpfft_batch_get_info(const vpfft_batch *b, vpfft_batch_info *info);
/* Autotuner of the batched FFT passes.  The first tick that admits an RVE of a
 * size new to the process times the five-pass chain of every tile family over
 * the RVEs of that size admitted in that tick (one warm-up, three timed, CUDA
 * events on the batch's stream, before their initialisation rewrites the field
 * the chain writes) and keeps the fastest; later batches of the process reuse
 * the choice.  One entry per size this batch has admitted, in order of first
 * admission.  No reference counterpart (the reference plans its FFTs with
 * FFTW_ESTIMATE, MaterialGrid.cpp:344-376). */
typedef struct {
  int32_t nx, ny, nz;
  int32_t fft_tiles;            /* family in use (0, 1, 2 as in vpfft_batch_options) */
  int32_t families;             /* families the size's line engines offer (1: no choice) */
  int32_t source;               /* 0 set by the options, 1 one family only, 2 timed earlier in
                                   this process, 3 timed by this batch */
  double ms_per_chain[3];       /* mean time of the five passes per family (0: not timed) */
} vpfft_tile_tuning;
/* Copies min(cap, count) entries; *n_out = count. */
vpfft_status vpfft_batch_get_tunings(const vpfft_batch *b, vpfft_tile_tuning *out, int cap,
                                     int *n_out);
const char *vpfft_batch_last_error(const vpfft_batch *b);

/* ------------------------------------------------------------------ text I/O
 * The reference's text formats, byte-compatible (numbers through C++ streams
 * with the reference's defaults).  Host code: no device needed except for
 * vpfft_grid_print. */
typedef enum {
  VPFFT_PRINT_STRAIN = 0,       /* MaterialGrid::PrintStrain (MaterialGrid.cpp:15-35): d~, re/im */
  VPFFT_PRINT_STRESS = 1,       /* PrintStress (40-55) */
  VPFFT_PRINT_LAGRANGE = 2,     /* PrintLagrangeMultiplier (60-75), x outermost */
  VPFFT_PRINT_POLARIZATION = 3  /* PrintPolarization (80-100), re/im */
} vpfft_print_kind;
/* One line per voxel "x y z v0 v1 ..." from host arrays: re N x 5
 * (voxel-major), im N x 5 or NULL (zeros) for the complex kinds. */
vpfft_status vpfft_print_field(const char *path, vpfft_print_kind kind, int nx, int ny, int nz,
                               const double *re, const double *im);
/* The same from a grid's fields.  The imaginary parts are written as 0: the
 * reference's P has none, and the imaginary part of its d~ (a by-product of
 * its c2c transform that the algorithm never uses) is not formed here. */
vpfft_status vpfft_grid_print(vpfft_grid *g, vpfft_print_kind kind, const char *path);
/* UnitTester::WriteRandomMaterial / ReadRandomMaterial (UnitTester.cpp:116-167):
 * per voxel (x outermost) the 9 orientation entries and the 5 stress values. */
vpfft_status vpfft_write_random_material(const char *path, int nx, int ny, int nz,
                                         const double *orientations, const double *stress);
vpfft_status vpfft_read_random_material(const char *path, int nx, int ny, int nz,
                                        double *orientations, double *stress);
/* UnitTester::ReadRicardoData (UnitTester.cpp:237-265): N lines of
 * "phi1 Phi phi2 x y z i j" (Euler angles in degrees, 1-based voxel indices,
 * two ignored integers) -> active Euler matrices (LinearAlgebra.cpp:160-181)
 * written into orientations (N x 9); indices out of range are an error. */
vpfft_status vpfft_read_euler_texture(const char *path, int nx, int ny, int nz,
                                      double *orientations);

/* SMatrix3x3::BuildActiveEulerMatrix (LinearAlgebra.cpp:160-181), radians,
 * with the reference's single-precision cosf/sinf. */
vpfft_status vpfft_euler_matrix(double phi, double theta, double psi, double orientation[9]);
/* The two-grain microstructure of the config's TwoGrainInit
 * (UnitTester::SetMaterialGrid, UnitTester.cpp:46-74). */
vpfft_status vpfft_fixture_two_grain(int nx, int ny, int nz, double *orientations);

/* ------------------------------------------------------------------ config
 * Utilities::ConfigFile (Config.h:21-85, Config.cpp:11-300) with its defects
 * fixed: slip-system lists are read into indices 0..11 (the reference writes
 * 1..12 into size-12 vectors), Parse returns its status, continuation lines
 * are detected correctly, and NRTolerence/TimeStep are double.  Errors are
 * returned, never exit(). */
typedef struct {
  int32_t num_x, num_y, num_z;       /* GridDimension */
  double input_strain_rate[9];       /* InputStrainRate, row-major 3x3 */
  int32_t max_nr_iter;               /* MaxNRIter */
  double nr_tolerance;               /* NRTolerence */
  double time_step;                  /* TimeStep */
  int32_t num_time_iter;             /* NumTimeIter */
  int32_t init_method;               /* 0 = TwoGrainInit, 1 = FileInit */
  char input_microstructure[1024];   /* FileInit filename */
  vpfft_material material;           /* CRSS, GammaDotBase, RateSensitivity, Tau0, Tau1,
                                        Theta0, Theta1, HardeningMatrix */
  double voxel_length[3];            /* VoxelLength (default 1 1 1) */
  double convergence_epsilon;        /* ConvergenceEpsilon (default 1e-5) */
  int32_t max_iter;                  /* MaxIter: fixed-point iterations (default 100) */
  int32_t precision;                 /* Precision: FP64 | MIXED (default FP64) */
} vpfft_config;
vpfft_status vpfft_config_read(const char *path, vpfft_config *out, char *err, size_t err_len);

#ifdef __cplusplus
}
#endif

#endif /* VPFFT_CAPI_H */
