/*
 * CPU oracle for the meshfree LSKUM 2-D Euler pseudo-time loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C, FP64 restatement of the
 * reference primal solver (the .F90 files of src_mpi_primal in
 * Nischay-Pro/mfcfd), one function per reference routine, same loop order
 * and same expression association.  Only tests/, __graft_entry__.smoke() and the CPU-baseline leg
 * of bench.py may call it, and only as the checker or the timed CPU baseline.
 * The product library never links or calls it.
 *
 * Parity status: UNPINNED.  The reference ships no golden vectors, fixtures,
 * grids or tests for this path, and its Fortran/MPI/PETSc/HDF5 toolchain is
 * absent here, so the restatement cannot be checked against reference output.
 * The fixtures under tests/golden/ are produced by this oracle (regression pins).
 *
 * Layouts follow the Fortran arrays: prim(4,N) is prim[(c-1) + 4*(i-1)],
 * dq(2,4,N) / qm(2,4,N) are [(a-1) + 2*(c-1) + 8*(i-1)], conn(N,20) is
 * column-major with 1-based point numbers: conn[(r-1)*ldconn + (i-1)].
 */
#ifndef LSKUM_ORACLE_H
#define LSKUM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_params {
    double cfl;          /* -cfl                                  */
    double power;        /* -power  (LSQ weights dist**power)     */
    double vl_const;     /* -vl_const (Venkatakrishnan K)         */
    double mach;         /* parameter.F90 Mach                    */
    double aoa;          /* parameter.F90 aoa (degrees)           */
    int    rks;          /* 4 for ssprk43, 1 for first            */
    double euler;        /* 1 for ssprk43, 2 for first            */
    int    inner_iterations;
    int    interior_points_normal_flag;
    int    format;       /* 1 legacy, 2 quadtree                  */
    int    shapes;
    int    restart;      /* 0: residue reset at it<=2             */
    double res_old;      /* res_old when restart==1               */
} orc_params;

typedef struct orc orc_t;

orc_t *orc_create(int n, const double *x, const double *y, const double *nx,
                  const double *ny, const double *min_dist, const int *flag_1,
                  const int *flag_2, const int *left, const int *right,
                  const int *nbhs, const int *conn, int ldconn,
                  const orc_params *p);
/* One rank's part of a partitioned point set: points 1..n_local are owned
 * (local_points), n_local+1..n ghosts; loops the reference runs over
 * local_points, and the point classification, skip the ghosts; plen is the
 * global point count of the residual norm (fpi_solver.F90:57-63). */
orc_t *orc_create_part(int n, int n_local, int plen, const double *x, const double *y,
                       const double *nx, const double *ny, const double *min_dist,
                       const int *flag_1, const int *flag_2, const int *left,
                       const int *right, const int *nbhs, const int *conn, int ldconn,
                       const orc_params *p);
void orc_destroy(orc_t *h);

/* freestream initial condition (initial_conditions.F90:9-42) */
void orc_init_freestream(orc_t *h);
void orc_set_prim(orc_t *h, const double *prim);
void orc_get_prim(const orc_t *h, double *prim);

/* the q_lskum loop (q_lskum.F90:59-73): it = it_first .. it_first+n-1 */
int orc_run(orc_t *h, int it_first, int n_iters, double *residue, int *n_done);

/* compute_cl_cd_cm (compute_force_coeffs.F90:11-102) on the current state.
 * cl/cd/cm have `shapes` entries; cp (optional) gets one value per shape point
 * in file order. */
void orc_forces(orc_t *h, double *cl, double *cd, double *cm, double *cp);

/* individual reference routines, for stage-level tests */
void orc_func_delta(orc_t *h);
void orc_eval_q_variables(orc_t *h);
void orc_eval_q_derivatives(orc_t *h);
void orc_eval_q_inner_loop(orc_t *h);
void orc_eval_update_innerloop(orc_t *h);
void orc_cal_flux_residual(orc_t *h);
void orc_state_update(orc_t *h, int rk);
void orc_save_prim_old(orc_t *h);
double orc_sum_res_sqr(const orc_t *h);

/* The CUDA tree's post-processing fields of the current state, per point:
 * the Mach number as print_primal_output forms it, sqrt(|u|^2 / c)
 * (src_cuda/post_processing.F90:24-27), the entropy |log(p/rho^gamma) -
 * log(pr_inf)| (src_cuda/compute_entropy.F90:10-30) and the D2-distance
 * adaptation sensor normalised by its maximum (src_cuda/adaptation_sensors.F90:
 * 7-101).  Any output may be NULL; returns the total entropy. */
double orc_output_fields(const orc_t *h, double *mach, double *entropy, double *sensor);

/* Secondary objectives of the current state (src_mpi_primal): kind 2 total
 * entropy (compute_entropy.F90:10-40), 3 total enstrophy
 * (compute_enstrophy.F90:9-89), 4 stagnation-pressure loss
 * (stagnation_values.F90:43-76, objective_function_J). */
double orc_objective(const orc_t *h, int kind);

/* copies an internal array out: name is one of
 * "prim","prim_old","q","dq","qm","flux_res","delta","nx","ny","temp" */
int orc_get(const orc_t *h, const char *name, double *out);
/* copies an array in: "prim", "dq" or "qm" (ghost refresh of a partition) */
int orc_set(orc_t *h, const char *name, const double *in);
/* split-connectivity counts: out[4*(i-1)+d] for d = xpos,xneg,ypos,yneg */
void orc_get_split_counts(const orc_t *h, int *out);
int orc_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
