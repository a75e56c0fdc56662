/*
 * mfcfd_b200 -- B200 (sm_100a) meshfree LSKUM 2-D Euler pseudo-time loop.
 *
 * C ABI.  Plain pointers and sizes; every function returns an int status
 * (0 = MFCFD_OK, negative = error) and never exits, aborts or prints.
 *
 * This boundary replaces the reference's Fortran module procedures over
 * module-global state (Nischay-Pro/mfcfd, src_mpi_primal):
 *   meshfree_solver.F90:83     call q_lskum()          -> create/set_state/run
 *   q_lskum.F90:16-79          the pseudo-time loop    -> mfcfd_run
 *   fpi_solver.F90:13-83       one iteration           -> one step of mfcfd_run
 *   compute_force_coeffs.F90:11-102  Cl, Cd, Cm, cp    -> mfcfd_forces
 *   initial_conditions.F90:9-70      freestream/restart -> create / set_state
 * The reference has no C ABI, plugin or operator registry; its Fortran host
 * binds these entry points through ISO_C_BINDING (see the Fortran module
 * include/mfcfd_b200_mod.F90).
 *
 * Array conventions follow the Fortran arrays the reference keeps in
 * `type(points) :: point` (src_mpi_primal/data_structure.F90:13-49):
 *   prim(4,N)  -> double[N][4] (rho, u1, u2, pr per point, caller's order)
 *   conn(N,20) -> int, column-major: slot r of point i at conn[(r-1)*ld_conn + i-1],
 *                 values are 1-based point numbers.
 * The library copies every input on create/set and writes only into
 * caller-provided outputs; it keeps no host pointer past a call.  Points are
 * renumbered internally; all inputs and outputs use the caller's order.
 *
 * Threading: one host thread per handle at a time; handles are independent.
 * Some calls use host threads of their own inside the call (state
 * reordering, mfcfd_adjoint_many) and join them before returning.
 */
#ifndef MFCFD_B200_H
#define MFCFD_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define MFCFD_OK             0
#define MFCFD_ERR_ARG       -1  /* bad argument (null pointer, size, range)      */
#define MFCFD_ERR_CUDA      -2  /* CUDA runtime error (see mfcfd_last_error)     */
#define MFCFD_ERR_NONFINITE -3  /* residue became NaN; the loop stopped there     */
#define MFCFD_ERR_TIMEOUT   -4  /* a bounded device wait gave up                  */
#define MFCFD_ERR_OOM       -5  /* device allocation failed                       */
#define MFCFD_ERR_GRID      -6  /* grid would give a singular least-squares system
                                   (an empty split list) or bad connectivity     */
#define MFCFD_ERR_NODEV     -7  /* no CUDA device / unsupported device            */
#define MFCFD_ERR_STATE     -8  /* call not valid in the handle's current state   */

/* precision of the pseudo-time loop */
#define MFCFD_FP64        0
#define MFCFD_FP32_MIXED  1

/* point renumbering */
#define MFCFD_ORDER_KIND  0   /* stable partition wall | outer | interior */
#define MFCFD_ORDER_RCM   1   /* reverse Cuthill-McKee, then the partition */

/* Grid as the reference reads it from point/point.h5 group /1 (or the legacy
 * partGrid text file): src_mpi_primal/point_preprocessor.F90:353-371. */
typedef struct mfcfd_grid {
    int n;                      /* local points (single rank: max_points)  */
    const double *x, *y;        /* coordinates                             */
    const double *nx, *ny;      /* file normals (used for interior points
                                   only when format == 2, quadtree)        */
    const double *min_dist;     /* Venkatakrishnan length scale            */
    const int *flag_1;          /* 0 wall, 1 interior, 2 outer             */
    const int *flag_2;          /* shape number, 0 = not on a shape        */
    const int *left, *right;    /* 1-based ring neighbours (boundary pts)  */
    const int *nbhs;            /* stencil size, 0..20                     */
    const int *conn;            /* Fortran conn(N,20), column-major, 1-based */
    int ld_conn;                /* leading dimension of conn (>= n)        */
    int shapes;                 /* number of shapes (-shapes)              */
} mfcfd_grid;

/* Case parameters: the reference's case.in keys (readcase.F90:12-125) plus
 * Mach/aoa (parameter.F90:5-6; the CUDA tree reads them from input.nml). */
typedef struct mfcfd_params {
    double cfl;                 /* -cfl                                    */
    double power;               /* -power: LSQ weights dist**power         */
    double vl_const;            /* -vl_const: Venkatakrishnan constant     */
    double mach;                /* freestream Mach number                  */
    double aoa;                 /* angle of attack, degrees                */
    int    rks;                 /* 4 (-tscheme ssprk43) or 1 (first)       */
    double euler;               /* 1.0 (ssprk43) or 2.0 (first)            */
    int    inner_iterations;    /* -inner_iterations                       */
    int    interior_points_normal_flag; /* 0: (0,1), 1: (1,0)             */
    int    format;              /* 1 legacy, 2 quadtree (-format_file)     */
    int    restart;             /* 1: -restart_solution same (res_old given) */
    double res_old;             /* residual norm of iteration 2 when restart */
    int    precision;           /* MFCFD_FP64 or MFCFD_FP32_MIXED          */
    int    ordering;            /* MFCFD_ORDER_KIND or MFCFD_ORDER_RCM     */
} mfcfd_params;

typedef struct mfcfd mfcfd_t;

/* objectives J (mfcfd_objective, mfcfd_adjoint, mfcfd_tangent) */
#define MFCFD_OBJ_CL          0  /* sum over shapes of Cl (compute_force_coeffs.F90)   */
#define MFCFD_OBJ_CD          1  /* sum over shapes of Cd: the reference's J            */
#define MFCFD_OBJ_ENTROPY     2  /* sum |log(p/rho^gamma) - log(pr_inf)|
                                    (compute_entropy.F90:10-40)                         */
#define MFCFD_OBJ_ENSTROPHY   3  /* sum (du2/dx - du1/dy)^2, least-squares gradients
                                    (compute_enstrophy.F90:9-89)                        */
#define MFCFD_OBJ_STAGNATION  4  /* sum (p0_inf - p0)^2 / (p0_inf^2 N), stagnation-
                                    pressure loss (stagnation_values.F90:43-76)         */

/* J of the current state (the reference's objective routines of
 * src_mpi_primal; Cl/Cd summed over shapes). */
int mfcfd_objective(mfcfd_t *h, int objective, double *J);

/* Reverse-mode derivative of the loop (the reference's checkpointed adjoint
 * q_lskum_chkpts_b + FPI_SOLVER_B, src_mpi_adjoint/sensitivity_files/
 * q_lskum_chkpts_b.F90:23-300).  From the handle's current state (held
 * fixed) it runs n_iters iterations, J = an MFCFD_OBJ_* objective of the final
 * state (the reference's J is Cd), and writes dJ/dx, dJ/dy per point
 * (caller order) -- the content of sensitivity/sensitivity.dat.  min_dist is
 * data (not a function of x, y), as in the reference.  prim snapshots are
 * kept in HBM within ckpt_bytes (32 bytes a point each, binomial placement);
 * *J (may be NULL) gets the objective, *n_forward (may be NULL) the number of
 * forward iterations run, recomputation included.  The handle is left at the
 * final state.  FP64 handles with power == 0 only (else MFCFD_ERR_ARG). */
int mfcfd_adjoint(mfcfd_t *h, int objective, int n_iters, size_t ckpt_bytes, double *J,
                  double *dJdx, double *dJdy, int *n_forward);

/* mfcfd_adjoint of n_handles independent solvers (grids of any sizes) in one
 * call: the adjoint a batch of cases needs, the reference running one case
 * per process.  Each handle's buffers and snapshot pool (ckpt_bytes each) are
 * allocated first, one handle after the other; then the reverse sweeps run,
 * each on its handle's own stream: handles of 65,536 points or more one
 * after another on one host thread (each fills the GPU alone), every
 * smaller handle on a host thread of its own, side by side with them.  Results
 * per handle are those of mfcfd_adjoint on it (bit for bit): J[i] (J may be
 * NULL), dJdx[i], dJdy[i] (caller order), n_forward[i] (may be NULL),
 * status[i] (may be NULL; MFCFD_OK or that handle's error).  Handles must be
 * distinct and on distinct streams; handles may live on different devices
 * (each handle's work runs with its device current; the caller's current
 * device is restored).  Returns MFCFD_OK or the first handle's error. */
#define MFCFD_ADJOINT_MANY_MAX 256
int mfcfd_adjoint_many(int n_handles, mfcfd_t *const *handles, int objective, int n_iters,
                       size_t ckpt_bytes, double *J, double *const *dJdx, double *const *dJdy,
                       int *n_forward, int *status);

/* Forward-mode (tangent) derivative of the loop (the reference's Q_LSKUM_D,
 * src_mpi_forward/sensitivity_files/q_lskum_d.F90:28-89, which seeds
 * pointd%x(1) = 1).  From the handle's current state (held fixed) it runs
 * n_iters iterations with the grid moved along the direction (dx, dy) per
 * point (caller order; NULL = 0) and writes J = an MFCFD_OBJ_* objective of
 * the final state and dJ/de along the direction.  For the gradient of
 * mfcfd_adjoint over the same iterations, dJ/de = sum_i dJdx_i dx_i +
 * dJdy_i dy_i.  The handle's state is left unchanged.  FP64 handles with
 * power == 0 only (else MFCFD_ERR_ARG). */
int mfcfd_tangent(mfcfd_t *h, int objective, int n_iters, const double *dx, const double *dy,
                  double *J, double *dJ);

/* Sets the default parameters of the reference's readcase (cfl 0,
 * power 0, vl_const 150, ssprk43, no inner iterations, legacy format) with
 * Mach 0.63 and aoa 2 (parameter.F90:5-6). */
int mfcfd_default_params(mfcfd_params *p);

/* Builds a solver on the current CUDA device: normals (point_normals.F90),
 * split connectivity (generate_connectivity.F90), renumbering, device
 * arrays, and the freestream initial state (initial_conditions.F90:9-20). */
int mfcfd_create(const mfcfd_grid *grid, const mfcfd_params *params, mfcfd_t **out);

/* Frees every device and host resource of the handle.  NULL is a no-op. */
int mfcfd_destroy(mfcfd_t *h);

/* Loads prim(4,N) (restart_sol, initial_conditions.F90:44-70).  The
 * reordering into the handle's point order runs on up to 8 host threads of
 * the library's own, joined before the call returns. */
int mfcfd_set_state(mfcfd_t *h, const double *prim);

/* Copies prim(4,N) out (reordered as mfcfd_set_state does). */
int mfcfd_get_state(mfcfd_t *h, double *prim);

/* Runs iterations it_first .. it_first+n_iters-1 of the q_lskum loop
 * (q_lskum.F90:59-73, fpi_solver.F90:13-83).  residue (n_iters entries, may
 * be NULL) receives the reference's residue per iteration: 0 for it <= 2
 * (no restart), else log10(res_new/res_old).  Like the reference, the loop
 * stops after the first iteration whose residue is NaN; *n_done (may be
 * NULL) is the number of iterations done and the return value is then
 * MFCFD_ERR_NONFINITE. */
int mfcfd_run(mfcfd_t *h, int it_first, int n_iters, double *residue, int *n_done);

/* Cl, Cd, Cm per shape (`shapes` entries each, any may be NULL) and cp per
 * shape point in grid order (flag_2 > 0, may be NULL) for the current state
 * (compute_force_coeffs.F90:11-102). */
int mfcfd_forces(mfcfd_t *h, double *cl, double *cd, double *cm, double *cp);

/* Uses the given cudaStream_t (NULL = the handle's own stream). */
int mfcfd_set_stream(mfcfd_t *h, void *stream);

/* The CUDA tree's post-processing fields of the current state, per point in
 * caller order (any may be NULL): the Mach number as print_primal_output
 * forms it, sqrt(|u|^2 / c) (src_cuda/post_processing.F90:24-27); the entropy
 * |log(p/rho^gamma) - log(pr_inf)| and their sum over the points
 * (src_cuda/compute_entropy.F90:10-30); the D2-distance adaptation sensor
 * normalised by its maximum (src_cuda/adaptation_sensors.F90:7-101) -- the
 * last three columns of output.dat. */
int mfcfd_output_fields(mfcfd_t *h, double *mach, double *entropy, double *sensor,
                        double *total_entropy);

/* Copies an internal per-point array out in caller order, for stage-level
 * checks: "q" (4/pt, the last stage's input), "dq" (8/pt: d/dx of q1..q4 then
 * d/dy), "qm" (8/pt: max of q1..q4 then min), "delta" (1), "nx", "ny" (1),
 * "flux_res" (4/pt, last stage; kept only when the handle was told to keep
 * diagnostics by mfcfd_keep_diagnostics). */
int mfcfd_get_array(mfcfd_t *h, const char *name, double *out);

/* Whether the flux pass also stores flux_res for mfcfd_get_array (0/1). */
int mfcfd_keep_diagnostics(mfcfd_t *h, int on);

/* Number of points and of wall, outer and interior points. */
int mfcfd_info(mfcfd_t *h, int *n, int *n_wall, int *n_outer, int *n_interior);

/* Human-readable text of a status code (static storage). */
const char *mfcfd_strerror(int status);

/* The last error message recorded on the handle (static per handle; empty
 * when none).  h may be NULL for errors of mfcfd_create. */
const char *mfcfd_last_error(mfcfd_t *h);

/* Device kernels launched by the handle since creation (all kinds). */
long long mfcfd_launch_count(mfcfd_t *h);

/* Diagnostic, no counterpart in the reference: the FP64 FMA throughput of
 * the current device in TFLOP/s (one FMA = 2 flops), measured with a
 * kernel of independent FMA chains (best of five launches after a warm-up).
 * The flux pass, which is bound by FP64 issue, is reported against it.
 * Allocates a small scratch buffer. */
int mfcfd_measure_fp64_peak(double *tflops);

/* A partitioned grid: one rank's part of a point set split over ranks, as
 * the reference runs it on several MPI ranks (point.h5 groups /1 .. /P,
 * point_preprocessor.F90:177-546; PETSc ghost vectors,
 * petsc_data_structure.F90:21-54).  grid holds the rank's points: the first
 * n_local are owned (full rows), the rest are ghosts, of which only x, y and
 * min_dist are read (the reference's ghost rows, :489-501); stencils of owned
 * points may name ghosts.  plen is the point count of all ranks (the residual
 * norm's divisor, fpi_solver.F90:57-63).  FP64 loop only.  The handle runs
 * iterations one phase at a time with mfcfd_part_phase (mfcfd_run refuses
 * it); between phases the caller refreshes the ghost rows from their owners
 * (mfcfd_part_rows gives the device rows, mfcfd_part_index their order). */
int mfcfd_create_part(const mfcfd_grid *grid, const mfcfd_params *params, int n_local,
                      int plen, mfcfd_t **out);

/* Phases of one iteration of a partitioned grid (fpi_solver.F90:13-83):
 * BEGIN; per stage rk = 1..rks: GRAD (eval_q_derivatives, and func_delta at
 * rk 1) -> refresh dq and qm ghost rows; INNER t = 1..m -> refresh dq;
 * FLUX (cal_flux_residual + state_update) -> refresh prim, then GHOSTS (q of
 * the ghost rows from their prim); END writes the rank's sum of res_sqr to
 * *value, which the caller adds over the ranks (MPI_Reduce + Bcast,
 * fpi_solver.F90:57-61) before the residue. */
#define MFCFD_PHASE_BEGIN  0
#define MFCFD_PHASE_GRAD   1
#define MFCFD_PHASE_INNER  2
#define MFCFD_PHASE_FLUX   3
#define MFCFD_PHASE_GHOSTS 4
#define MFCFD_PHASE_END    5
int mfcfd_part_phase(mfcfd_t *h, int phase, int rk, int t, double *value);

/* Device rows the last phase wrote, for the ghost refresh: name "prim" (4
 * doubles a row), "dq" or "qm" (8 doubles a row), in the handle's internal
 * row order (mfcfd_part_index). */
int mfcfd_part_rows(mfcfd_t *h, const char *name, void **rows, int *row_doubles);

/* internal[i] = internal row of point i (caller order), for all grid.n points. */
int mfcfd_part_index(mfcfd_t *h, int *internal);

/* Largest n_iters one mfcfd_run_noalloc call accepts. */
#define MFCFD_NOALLOC_MAX_ITERS 65536

/* mfcfd_run without any device allocation.  No counterpart in the
 * reference.  For callers that cannot allocate device memory while they run
 * (a host whose device memory belongs to its own pool, a service that
 * allocates only at start-up):
 * mfcfd_run may grow its residue-history buffer with cudaMalloc and
 * instantiates CUDA graphs; this call keeps the history in a fixed
 * per-device array of MFCFD_NOALLOC_MAX_ITERS doubles (512 KiB, held by every
 * GPU that loads the library until exit), launches the kernels directly and
 * allocates nothing.  Same arguments, results and status codes as mfcfd_run;
 * n_iters above MFCFD_NOALLOC_MAX_ITERS gives MFCFD_ERR_ARG.  The array's
 * device address is looked up by mfcfd_create, with the handle's device
 * current (the first create on a device loads the library's module there,
 * which places the array); the call itself runs on the handle's device
 * whatever device the caller has current.  All calls on a device share the
 * array, so calls that overlap on the GPU (handles on concurrent streams)
 * race on it. */
int mfcfd_run_noalloc(mfcfd_t *h, int it_first, int n_iters, double *residue, int *n_done);

/* Runs iteration `it` with a CUDA event after every kernel on the handle's
 * stream and returns the mean duration per launch in ms of the gradient,
 * inner-iteration, flux and residual kernels (ms[0..3]) and of the whole
 * iteration (ms[4]).  The state advances by that iteration, as mfcfd_run
 * would advance it (no CUDA graph). */
int mfcfd_profile_iteration(mfcfd_t *h, int it, double *ms);

/* ------------------------------------------------------------------------
 * Batched runs: many independent grids (instances) advanced together on one
 * GPU.  No counterpart in the reference, which runs one grid per process
 * (meshfree_solver.F90:83 -> q_lskum); every instance follows exactly the
 * loop of mfcfd_run, and its states and residues are bit-identical to those
 * of a handle created from the same grid and parameters.  The points of all
 * instances share one set of device arrays; every pass is one grid-stride
 * launch over the tiles (16 points) of the instances still running, so
 * small grids do not pay a launch each.  Instances retire independently.
 * ------------------------------------------------------------------------ */
typedef struct mfcfd_batch mfcfd_batch_t;

#define MFCFD_BATCH_MAX 256  /* instances per batch */

/* Why an instance stopped in the last mfcfd_batch_run. */
#define MFCFD_BATCH_RUNNING    0  /* not run                                  */
#define MFCFD_BATCH_CONVERGED  1  /* residue <= tol                           */
#define MFCFD_BATCH_MAX_ITERS  2  /* ran max_iters iterations                 */
#define MFCFD_BATCH_NONFINITE  3  /* residue NaN (the loop's exit, as mfcfd_run) */

/* Builds a batch of n_inst (1..MFCFD_BATCH_MAX) instances: grids[i] with
 * params[i], each checked and set up as mfcfd_create does, starting from the
 * freestream state at iteration 1.  cfl, power, rks, euler,
 * inner_iterations and precision must be equal in all params (else
 * MFCFD_ERR_ARG); mach, aoa, vl_const and the rest may differ.  Errors are
 * reported by mfcfd_last_error(NULL). */
int mfcfd_batch_create(int n_inst, const mfcfd_grid *const *grids, const mfcfd_params *params,
                       mfcfd_batch_t **out);

/* Frees the batch.  NULL is a no-op. */
int mfcfd_batch_destroy(mfcfd_batch_t *b);

/* Uses the given cudaStream_t (NULL = the batch's own stream). */
int mfcfd_batch_set_stream(mfcfd_batch_t *b, void *stream);

/* prim(4,N_inst) of one instance in and out, as mfcfd_set_state/get_state. */
int mfcfd_batch_set_state(mfcfd_batch_t *b, int inst, const double *prim);
int mfcfd_batch_get_state(mfcfd_batch_t *b, int inst, double *prim);

/* Advances every instance from its own iteration counter until its residue
 * is <= tol, or it has run max_iters iterations in this call, or its residue
 * is NaN (residue as mfcfd_run defines it; 0 for the first two iterations
 * of a fresh run).  Per instance (arrays of n_inst, any may be NULL):
 * iters_done, the MFCFD_BATCH_* reason it stopped, and residue history rows
 * residue[inst * max_iters + k], k < iters_done[inst].  The host is not
 * involved between iterations (retirement happens on the device); it polls
 * a counter every 16 iterations to stop once no instance runs.  Returns
 * MFCFD_ERR_NONFINITE if an instance stopped on a NaN residue (the others
 * still ran), else MFCFD_OK. */
int mfcfd_batch_run(mfcfd_batch_t *b, double tol, int max_iters, int *iters_done, int *state,
                    double *residue);

/* Cl, Cd, Cm and cp of one instance, as mfcfd_forces. */
int mfcfd_batch_forces(mfcfd_batch_t *b, int inst, double *cl, double *cd, double *cm,
                       double *cp);

/* Autotuner: times iters iterations (>= 2) of each candidate launch shape
 * (block size 256 or 128 of the point passes; blocks of every grid-stride
 * pass as 1, 2 or 4 waves of resident blocks, or sized for 1, 2 or 4 points
 * per thread of the point passes and 1, 2 or 4 two-tile chunks per warp of
 * the flux pass) on a copy of the current state, keeps the fastest and
 * restores the state.  Results do not
 * depend on the launch shape.  *ms_per_iter (may be NULL) gets the best time
 * per iteration. */
int mfcfd_batch_tune(mfcfd_batch_t *b, int iters, double *ms_per_iter);

/* Sets the launch shape by hand: block size of the D and I passes (128 or
 * 256) and the blocks of the D/I and F passes (0 = one wave of resident
 * blocks). */
int mfcfd_batch_set_launch(mfcfd_batch_t *b, int point_block, int point_grid, int flux_grid);

/* Instances, total points (sum of N_inst), the current launch shape. */
int mfcfd_batch_info(mfcfd_batch_t *b, int *n_inst, long long *n_points, int *point_block,
                     int *point_grid, int *flux_grid);

/* Last error of the batch (NULL: of mfcfd_batch_create) and kernel count. */
const char *mfcfd_batch_last_error(mfcfd_batch_t *b);
long long mfcfd_batch_launch_count(mfcfd_batch_t *b);

#ifdef __cplusplus
}
#endif
#endif /* MFCFD_B200_H */
