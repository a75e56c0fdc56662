/*
 * CPU oracle for the meshfree LSKUM 2-D Euler pseudo-time loop.
 *
 * TEST INFRASTRUCTURE ONLY (checker and timed CPU baseline; never the product).
 * Parity status: UNPINNED -- the reference ships no golden vectors or tests for
 * this path and cannot be built here (Fortran + MPI + PETSc + HDF5 absent).
 *
 * Restates, in C and FP64, the reference's src_mpi_primal routines with the
 * same loop order and the same left-to-right expression association as the
 * Fortran source (Fortran evaluates a*b*c as (a*b)*c and a-b-c as (a-b)-c).
 * Build with -ffp-contract=off for the parity variant.
 *
 * Single-rank semantics (proc == 1): max_points == local_points == N, no
 * ghosts, plen = N, PETSc ghost updates are no-ops.
 *
 * Per-point loops carry `omp parallel for`: every iteration writes only its
 * own point, so the result does not depend on the thread count.  The two
 * reductions (residual and forces) stay serial, in the reference's order.
 */
#include "lskum_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXNB 20

/* parameter.F90:7-10: rho_inf, pr_inf, gamma, pi */
static const double RHO_INF = 1.0;
#define PR_INF (1.0 / 1.4)
static const double GAMMA = 1.4;

struct orc {
    int n, ldconn;
    int n_local;  /* owned points (local_points); points n_local+1..n are ghosts */
    int plen;     /* points in the residual norm (all ranks' owned points) */
    orc_params p;
    double pi, theta, q_inf[4];
    double *x, *y, *nx, *ny, *min_dist;
    int *flag_1, *flag_2, *left, *right, *nbhs, *conn;
    int wall_points, outer_points, interior_points, shape_points;
    int *wall_idx, *outer_idx, *interior_idx, *shape_idx; /* 1-based */
    int *nb_cnt[4];   /* xpos, xneg, ypos, yneg counts */
    int *nb_conn[4];  /* (N,20) column-major, 1-based   */
    double *prim, *prim_old, *flux_res, *q, *dq, *qm, *temp, *delta;
    double sum_res_sqr, res_old, res_new, residue;
};

/* 1-based Fortran-style accessors */
#define X(i) (h->x[(i) - 1])
#define Y(i) (h->y[(i) - 1])
#define NX(i) (h->nx[(i) - 1])
#define NY(i) (h->ny[(i) - 1])
#define MIND(i) (h->min_dist[(i) - 1])
#define NBHS(i) (h->nbhs[(i) - 1])
#define CONN(i, r) (h->conn[((r) - 1) * h->ldconn + (i) - 1])
#define PRIM(c, i) (h->prim[((c) - 1) + 4 * ((i) - 1)])
#define PRIMO(c, i) (h->prim_old[((c) - 1) + 4 * ((i) - 1)])
#define FRES(c, i) (h->flux_res[((c) - 1) + 4 * ((i) - 1)])
#define Q(c, i) (h->q[((c) - 1) + 4 * ((i) - 1)])
#define DQ(a, c, i) (h->dq[((a) - 1) + 2 * ((c) - 1) + 8 * ((i) - 1)])
#define QM(a, c, i) (h->qm[((a) - 1) + 2 * ((c) - 1) + 8 * ((i) - 1)])
#define TMP(a, c, i) (h->temp[((a) - 1) + 3 * ((c) - 1) + 12 * ((i) - 1)])
#define SPLITN(d, i) (h->nb_cnt[d][(i) - 1])
#define SPLITC(d, i, j) (h->nb_conn[d][((j) - 1) * h->n + (i) - 1])

enum { XPOS = 0, XNEG = 1, YPOS = 2, YNEG = 3 };

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* parameter.F90:16-34 setup_case_parameters                                */
static void setup_case_parameters(orc_t *h) {
    h->pi = 4.0 * atan(1.0);
    h->theta = h->p.aoa * h->pi / 180.0;
    h->q_inf[0] = RHO_INF;
    h->q_inf[1] = h->p.mach * cos(h->theta);
    h->q_inf[2] = h->p.mach * sin(h->theta);
    h->q_inf[3] = PR_INF;
}

/* point_normals.F90:8-105 compute_normals */
static void compute_normals(orc_t *h) {
    for (int pass = 0; pass < 2; ++pass) {
        int cnt = pass == 0 ? h->wall_points : h->outer_points;
        const int *idx = pass == 0 ? h->wall_idx : h->outer_idx;
        for (int i = 0; i < cnt; ++i) {
            int m = idx[i], l = h->left[m - 1], r = h->right[m - 1];
            double lx = X(l), ly = Y(l), mx = X(m), my = Y(m), rx = X(r), ry = Y(r);
            double nx1 = my - ly, nx2 = ry - my;
            double ny1 = mx - lx, ny2 = rx - mx;
            double nx = 0.5 * (nx1 + nx2);
            double ny = 0.5 * (ny1 + ny2);
            double det = sqrt(nx * nx + ny * ny);
            nx = -nx / det;
            ny = ny / det;
            NX(m) = nx;
            NY(m) = ny;
        }
    }
    if (h->p.interior_points_normal_flag == 0 && h->p.format != 2) {
        for (int i = 0; i < h->interior_points; ++i) {
            int k = h->interior_idx[i];
            NX(k) = 0.0;
            NY(k) = 1.0;
        }
    } else if (h->p.interior_points_normal_flag == 1 && h->p.format != 2) {
        for (int i = 0; i < h->interior_points; ++i) {
            int k = h->interior_idx[i];
            NX(k) = 1.0;
            NY(k) = 0.0;
        }
    }
}

/* generate_connectivity.F90:8-256: sign split of conn into the four lists.
 * kind 1 = interior (all four by sign), 0 = wall (x by sign, every nbh in
 * yneg), 2 = outer (x by sign, every nbh in ypos). */
static void split_point(orc_t *h, int i, int kind) {
    double xi = X(i), yi = Y(i), nx = NX(i), ny = NY(i);
    double tx = ny, ty = -nx;
    for (int d = 0; d < 4; ++d) SPLITN(d, i) = 0;
    for (int r = 1; r <= NBHS(i); ++r) {
        int nbh = CONN(i, r);
        double delx = X(nbh) - xi, dely = Y(nbh) - yi;
        double dels = delx * tx + dely * ty;
        double deln = delx * nx + dely * ny;
        if (dels <= 0.0) { SPLITN(XPOS, i) += 1; SPLITC(XPOS, i, SPLITN(XPOS, i)) = nbh; }
        if (dels >= 0.0) { SPLITN(XNEG, i) += 1; SPLITC(XNEG, i, SPLITN(XNEG, i)) = nbh; }
        if (kind == 1) {
            if (deln <= 0.0) { SPLITN(YPOS, i) += 1; SPLITC(YPOS, i, SPLITN(YPOS, i)) = nbh; }
            if (deln >= 0.0) { SPLITN(YNEG, i) += 1; SPLITC(YNEG, i, SPLITN(YNEG, i)) = nbh; }
        } else if (kind == 0) {
            SPLITN(YNEG, i) += 1; SPLITC(YNEG, i, SPLITN(YNEG, i)) = nbh;
        } else {
            SPLITN(YPOS, i) += 1; SPLITC(YPOS, i, SPLITN(YPOS, i)) = nbh;
        }
    }
}

static void generate_connectivity(orc_t *h) {
    for (int k = 0; k < h->interior_points; ++k) split_point(h, h->interior_idx[k], 1);
    for (int k = 0; k < h->wall_points; ++k) split_point(h, h->wall_idx[k], 0);
    for (int k = 0; k < h->outer_points; ++k) split_point(h, h->outer_idx[k], 2);
}

/* ------------------------------------------------------------------------ */
orc_t *orc_create(int n, const double *x, const double *y, const double *nx,
                  const double *ny, const double *min_dist, const int *flag_1,
                  const int *flag_2, const int *left, const int *right,
                  const int *nbhs, const int *conn, int ldconn,
                  const orc_params *p) {
    return orc_create_part(n, n, n, x, y, nx, ny, min_dist, flag_1, flag_2, left, right, nbhs,
                           conn, ldconn, p);
}

/* One rank's part of a partitioned point set (point_preprocessor.F90:177-546,
 * petsc_data_structure.F90:21-54): points 1..n_local are owned, the rest are
 * ghosts whose prim, dq and qm the caller refreshes between phases; plen is
 * the global point count of the residual norm. */
orc_t *orc_create_part(int n, int n_local, int plen, const double *x, const double *y,
                       const double *nx, const double *ny, const double *min_dist,
                       const int *flag_1, const int *flag_2, const int *left,
                       const int *right, const int *nbhs, const int *conn, int ldconn,
                       const orc_params *p) {
    orc_t *h = (orc_t *)calloc(1, sizeof(orc_t));
    h->n = n;
    h->n_local = n_local;
    h->plen = plen;
    h->ldconn = ldconn;
    h->p = *p;
    size_t nd = (size_t)n * sizeof(double), ni = (size_t)n * sizeof(int);
    h->x = malloc(nd); memcpy(h->x, x, nd);
    h->y = malloc(nd); memcpy(h->y, y, nd);
    h->nx = malloc(nd); memcpy(h->nx, nx, nd);
    h->ny = malloc(nd); memcpy(h->ny, ny, nd);
    h->min_dist = malloc(nd); memcpy(h->min_dist, min_dist, nd);
    h->flag_1 = malloc(ni); memcpy(h->flag_1, flag_1, ni);
    h->flag_2 = malloc(ni); memcpy(h->flag_2, flag_2, ni);
    h->left = malloc(ni); memcpy(h->left, left, ni);
    h->right = malloc(ni); memcpy(h->right, right, ni);
    h->nbhs = malloc(ni); memcpy(h->nbhs, nbhs, ni);
    h->conn = malloc((size_t)ldconn * MAXNB * sizeof(int));
    memcpy(h->conn, conn, (size_t)ldconn * MAXNB * sizeof(int));
    /* point_preprocessor.F90:374-435: type counts and index lists */
    h->wall_idx = malloc(ni); h->outer_idx = malloc(ni);
    h->interior_idx = malloc(ni); h->shape_idx = malloc(ni);
    for (int k = 1; k <= n_local; ++k) {
        int f = flag_1[k - 1];
        if (f == 0) h->wall_idx[h->wall_points++] = k;
        else if (f == 1) h->interior_idx[h->interior_points++] = k;
        else if (f == 2) h->outer_idx[h->outer_points++] = k;
        if (flag_2[k - 1] > 0) h->shape_idx[h->shape_points++] = k;
    }
    for (int d = 0; d < 4; ++d) {
        h->nb_cnt[d] = calloc((size_t)n, sizeof(int));
        h->nb_conn[d] = calloc((size_t)n * MAXNB, sizeof(int));
    }
    h->prim = calloc((size_t)4 * n, sizeof(double));
    h->prim_old = calloc((size_t)4 * n, sizeof(double));
    h->flux_res = calloc((size_t)4 * n, sizeof(double));
    h->q = calloc((size_t)4 * n, sizeof(double));
    h->dq = calloc((size_t)8 * n, sizeof(double));
    h->qm = calloc((size_t)8 * n, sizeof(double));
    h->temp = calloc((size_t)12 * n, sizeof(double));
    h->delta = calloc((size_t)n, sizeof(double));
    h->res_old = p->res_old;
    setup_case_parameters(h);
    /* q_lskum.F90:33-34 */
    compute_normals(h);
    generate_connectivity(h);
    orc_init_freestream(h);
    return h;
}

void orc_destroy(orc_t *h) {
    if (!h) return;
    free(h->x); free(h->y); free(h->nx); free(h->ny); free(h->min_dist);
    free(h->flag_1); free(h->flag_2); free(h->left); free(h->right);
    free(h->nbhs); free(h->conn);
    free(h->wall_idx); free(h->outer_idx); free(h->interior_idx); free(h->shape_idx);
    for (int d = 0; d < 4; ++d) { free(h->nb_cnt[d]); free(h->nb_conn[d]); }
    free(h->prim); free(h->prim_old); free(h->flux_res); free(h->q);
    free(h->dq); free(h->qm); free(h->temp); free(h->delta);
    free(h);
}

/* initial_conditions.F90:9-20 */
void orc_init_freestream(orc_t *h) {
    for (int k = 1; k <= h->n; ++k)
        for (int c = 1; c <= 4; ++c) PRIM(c, k) = h->q_inf[c - 1];
}

void orc_set_prim(orc_t *h, const double *prim) {
    memcpy(h->prim, prim, (size_t)4 * h->n * sizeof(double));
}
void orc_get_prim(const orc_t *h, double *prim) {
    memcpy(prim, h->prim, (size_t)4 * h->n * sizeof(double));
}

void orc_save_prim_old(orc_t *h) {
    memcpy(h->prim_old, h->prim, (size_t)4 * h->n_local * sizeof(double));
}

/* ------------------------------------------------------------------------ */
/* q_variables.F90:8-37 eval_q_variables */
void orc_eval_q_variables(orc_t *h) {
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= h->n; ++k) {
        double rho = PRIM(1, k), u1 = PRIM(2, k), u2 = PRIM(3, k), pr = PRIM(4, k);
        double beta = 0.5 * rho / pr;
        Q(1, k) = (log(rho) + (log(beta) * 2.5)) - beta * (u1 * u1 + u2 * u2);
        double two_times_beta = 2.0 * beta;
        Q(2, k) = two_times_beta * u1;
        Q(3, k) = two_times_beta * u2;
        Q(4, k) = -two_times_beta;
    }
}

/* q_variables.F90:41-112 eval_q_derivatives */
void orc_eval_q_derivatives(orc_t *h) {
    const double power = h->p.power;
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= h->n_local; ++i) {
        double x_i = X(i), y_i = Y(i);
        double sum_delx_sqr = 0.0, sum_dely_sqr = 0.0, sum_delx_dely = 0.0;
        double sum_delx_delq[4] = {0, 0, 0, 0}, sum_dely_delq[4] = {0, 0, 0, 0};
        for (int c = 1; c <= 4; ++c) { QM(1, c, i) = Q(c, i); QM(2, c, i) = Q(c, i); }
        for (int k = 1; k <= NBHS(i); ++k) {
            int nbh = CONN(i, k);
            for (int r = 1; r <= 4; ++r) {
                if (Q(r, nbh) > QM(1, r, i)) QM(1, r, i) = Q(r, nbh);
                if (Q(r, nbh) < QM(2, r, i)) QM(2, r, i) = Q(r, nbh);
            }
            double delx = X(nbh) - x_i, dely = Y(nbh) - y_i;
            double dist = sqrt(delx * delx + dely * dely);
            double weights = pow(dist, power);
            sum_delx_sqr = sum_delx_sqr + delx * delx * weights;
            sum_dely_sqr = sum_dely_sqr + dely * dely * weights;
            sum_delx_dely = sum_delx_dely + delx * dely * weights;
            for (int r = 1; r <= 4; ++r) {
                sum_delx_delq[r - 1] = sum_delx_delq[r - 1] + weights * delx * (Q(r, nbh) - Q(r, i));
                sum_dely_delq[r - 1] = sum_dely_delq[r - 1] + weights * dely * (Q(r, nbh) - Q(r, i));
            }
        }
        double det = sum_delx_sqr * sum_dely_sqr - sum_delx_dely * sum_delx_dely;
        double one_by_det = 1.0 / det;
        for (int r = 1; r <= 4; ++r) {
            DQ(1, r, i) = (sum_delx_delq[r - 1] * sum_dely_sqr - sum_dely_delq[r - 1] * sum_delx_dely) * one_by_det;
            DQ(2, r, i) = (sum_dely_delq[r - 1] * sum_delx_sqr - sum_delx_delq[r - 1] * sum_delx_dely) * one_by_det;
        }
    }
}

/* q_variables.F90:115-212 eval_q_inner_loop */
void orc_eval_q_inner_loop(orc_t *h) {
    const double power = h->p.power;
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= h->n_local; ++i) {
        double x_i = X(i), y_i = Y(i);
        double sum_delx_sqr = 0.0, sum_dely_sqr = 0.0, sum_delx_dely = 0.0;
        double sdx[4] = {0, 0, 0, 0}, sdy[4] = {0, 0, 0, 0};
        double qi[4] = {Q(1, i), Q(2, i), Q(3, i), Q(4, i)};
        for (int k = 1; k <= NBHS(i); ++k) {
            int nbh = CONN(i, k);
            double delx = X(nbh) - x_i, dely = Y(nbh) - y_i;
            double dist = sqrt(delx * delx + dely * dely);
            double weights = pow(dist, power);
            sum_delx_sqr = sum_delx_sqr + delx * delx * weights;
            sum_dely_sqr = sum_dely_sqr + dely * dely * weights;
            sum_delx_dely = sum_delx_dely + delx * dely * weights;
            for (int r = 1; r <= 4; ++r) {
                double temp1 = qi[r - 1] - 0.5 * (delx * DQ(1, r, i) + dely * DQ(2, r, i));
                double temp2 = Q(r, nbh) - 0.5 * (delx * DQ(1, r, nbh) + dely * DQ(2, r, nbh));
                sdx[r - 1] = sdx[r - 1] + (weights * delx * (temp2 - temp1));
                sdy[r - 1] = sdy[r - 1] + (weights * dely * (temp2 - temp1));
            }
        }
        double det = sum_delx_sqr * sum_dely_sqr - sum_delx_dely * sum_delx_dely;
        double one_by_det = 1.0 / det;
        for (int r = 1; r <= 4; ++r) {
            TMP(1, r, i) = one_by_det * (sdx[r - 1] * sum_dely_sqr - sdy[r - 1] * sum_delx_dely);
            TMP(2, r, i) = one_by_det * (sdy[r - 1] * sum_delx_sqr - sdx[r - 1] * sum_delx_dely);
        }
    }
}

/* q_variables.F90:215-227 eval_update_innerloop */
void orc_eval_update_innerloop(orc_t *h) {
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= h->n_local; ++i)
        for (int r = 1; r <= 4; ++r) {
            DQ(1, r, i) = TMP(1, r, i);
            DQ(2, r, i) = TMP(2, r, i);
        }
}

/* q_variables.F90:230-256 qtilde_to_primitive */
static inline void qtilde_to_primitive(const double qt[4], double *u1, double *u2,
                                       double *rho, double *pr) {
    double q1 = qt[0], q2 = qt[1], q3 = qt[2], q4 = qt[3];
    double beta = -q4 * 0.5;
    double temp = 0.5 / beta;
    *u1 = q2 * temp;
    *u2 = q3 * temp;
    double temp1 = q1 + beta * ((*u1) * (*u1) + (*u2) * (*u2));
    double temp2 = temp1 - (log(beta) / (GAMMA - 1));
    *rho = exp(temp2);
    *pr = (*rho) * temp;
}

/* limiters.F90:64-110 venkat_limiter.  The threshold literal 10e-6 is a
 * default-real (single precision) constant promoted to double. */
static inline void venkat_limiter(const orc_t *h, const double qtilde[4], double phi[4], int k) {
    const double thr = (double)10e-6f;
    for (int r = 1; r <= 4; ++r) {
        double q = Q(r, k);
        double del_neg = qtilde[r - 1] - q;
        double del_pos = 0.0;
        if (fabs(del_neg) <= thr) {
            phi[r - 1] = 1.0;
        } else if (fabs(del_neg) > thr) {
            if (del_neg > 0.0) del_pos = QM(1, r, k) - q;
            else if (del_neg < 0.0) del_pos = QM(2, r, k) - q;
            double epsi = h->p.vl_const * MIND(k);
            epsi = pow(epsi, 3.0);
            double num = (del_pos * del_pos) + (epsi * epsi);
            num = num * del_neg + 2.0 * del_neg * del_neg * del_pos;
            double den = del_pos * del_pos + 2.0 * del_neg * del_neg;
            den = den + del_neg * del_pos + epsi * epsi;
            den = den * del_neg;
            double temp = num / den;
            phi[r - 1] = temp < 1.0 ? temp : 1.0;
        }
    }
}

/* split_fluxes.F90:8-190 (Gxp, Gxn, Gyp, Gyn) */
static inline void flux_Gx(double G[4], int pos, double nx, double ny, double u1,
                           double u2, double rho, double pr, double pi) {
    double tx = ny, ty = -nx;
    double ut = u1 * tx + u2 * ty;
    double un = u1 * nx + u2 * ny;
    double beta = 0.5 * rho / pr;
    double S1 = ut * sqrt(beta);
    double B1 = 0.5 * exp(-S1 * S1) / sqrt(pi * beta);
    double pr_by_rho = pr / rho;
    double u_sqr = ut * ut + un * un;
    double temp1, temp2;
    if (pos) {
        double A1pos = 0.5 * (1.0 + erf(S1));
        G[0] = rho * (ut * A1pos + B1);
        temp1 = pr_by_rho + ut * ut;
        temp2 = temp1 * A1pos + ut * B1;
        G[1] = rho * temp2;
        temp1 = ut * un * A1pos + un * B1;
        G[2] = rho * temp1;
        temp1 = (7.0 * pr_by_rho) + u_sqr;
        temp2 = 0.5 * ut * temp1 * A1pos;
        temp1 = (6.0 * pr_by_rho) + u_sqr;
        G[3] = rho * (temp2 + 0.5 * temp1 * B1);
    } else {
        double A1neg = 0.5 * (1.0 - erf(S1));
        G[0] = rho * (ut * A1neg - B1);
        temp1 = pr_by_rho + ut * ut;
        temp2 = temp1 * A1neg - ut * B1;
        G[1] = rho * temp2;
        temp1 = ut * un * A1neg - un * B1;
        G[2] = rho * temp1;
        temp1 = (7.0 * pr_by_rho) + u_sqr;
        temp2 = 0.5 * ut * temp1 * A1neg;
        temp1 = (6.0 * pr_by_rho) + u_sqr;
        G[3] = rho * (temp2 - 0.5 * temp1 * B1);
    }
}

static inline void flux_Gy(double G[4], int pos, double nx, double ny, double u1,
                           double u2, double rho, double pr, double pi) {
    double tx = ny, ty = -nx;
    double ut = u1 * tx + u2 * ty;
    double un = u1 * nx + u2 * ny;
    double beta = 0.5 * rho / pr;
    double S2 = un * sqrt(beta);
    double B2 = 0.5 * exp(-S2 * S2) / sqrt(pi * beta);
    double pr_by_rho = pr / rho;
    double u_sqr = ut * ut + un * un;
    double temp1, temp2;
    if (pos) {
        double A2pos = 0.5 * (1.0 + erf(S2));
        G[0] = rho * (un * A2pos + B2);
        temp1 = pr_by_rho + un * un;
        temp2 = temp1 * A2pos + un * B2;
        G[2] = rho * temp2;
        temp1 = ut * un * A2pos + ut * B2;
        G[1] = rho * temp1;
        temp1 = (7.0 * pr_by_rho) + u_sqr;
        temp2 = 0.5 * un * temp1 * A2pos;
        temp1 = (6.0 * pr_by_rho) + u_sqr;
        G[3] = rho * (temp2 + 0.5 * temp1 * B2);
    } else {
        double A2neg = 0.5 * (1.0 - erf(S2));
        G[0] = rho * (un * A2neg - B2);
        temp1 = pr_by_rho + un * un;
        temp2 = temp1 * A2neg - un * B2;
        G[2] = rho * temp2;
        temp1 = ut * un * A2neg - ut * B2;
        G[1] = rho * temp1;
        temp1 = (7.0 * pr_by_rho) + u_sqr;
        temp2 = 0.5 * un * temp1 * A2neg;
        temp1 = (6.0 * pr_by_rho) + u_sqr;
        G[3] = rho * (temp2 - 0.5 * temp1 * B2);
    }
}

/* quadrant_fluxes.F90:12-248.  quad: 1 = GxI (A1neg,A2neg), 2 = GxII
 * (A1pos,A2neg), 3 = GxIII (A1pos,A2pos), 4 = GxIV (A1neg,A2pos). */
static inline void flux_quad(double G[4], int quad, double nx, double ny, double u1,
                             double u2, double rho, double pr, double pi) {
    double tx = ny, ty = -nx;
    double ut = u1 * tx + u2 * ty;
    double un = u1 * nx + u2 * ny;
    double beta = 0.5 * rho / pr;
    double S1 = ut * sqrt(beta);
    double S2 = un * sqrt(beta);
    double B1 = 0.5 * exp(-S1 * S1) / sqrt(pi * beta);
    double B2 = 0.5 * exp(-S2 * S2) / sqrt(pi * beta);
    double pr_by_rho = pr / rho;
    double u_sqr = ut * ut + un * un;
    double temp1, temp2, temp3, temp4;
    if (quad == 1) {
        double A1neg = 0.5 * (1.0 - erf(S1));
        double A2neg = 0.5 * (1.0 - erf(S2));
        G[0] = rho * A2neg * (ut * A1neg - B1);
        temp1 = pr_by_rho + ut * ut;
        temp2 = temp1 * A1neg - ut * B1;
        G[1] = rho * A2neg * temp2;
        temp1 = ut * A1neg - B1;
        temp2 = un * A2neg - B2;
        G[2] = rho * temp1 * temp2;
        temp1 = (7.0 * pr_by_rho) + u_sqr;
        temp2 = 0.5 * ut * temp1 * A1neg;
        temp1 = (6.0 * pr_by_rho) + u_sqr;
        temp3 = 0.5 * B1 * temp1;
        temp1 = ut * A1neg - B1;
        temp4 = 0.5 * rho * un * B2 * temp1;
        G[3] = rho * A2neg * (temp2 - temp3) - temp4;
    } else if (quad == 2) {
        double A1pos = 0.5 * (1.0 + erf(S1));
        double A2neg = 0.5 * (1.0 - erf(S2));
        G[0] = rho * A2neg * (ut * A1pos + B1);
        temp1 = pr_by_rho + ut * ut;
        temp2 = temp1 * A1pos + ut * B1;
        G[1] = rho * A2neg * temp2;
        temp1 = ut * A1pos + B1;
        temp2 = un * A2neg - B2;
        G[2] = rho * temp1 * temp2;
        temp1 = (7.0 * pr_by_rho) + u_sqr;
        temp2 = 0.5 * ut * temp1 * A1pos;
        temp1 = (6.0 * pr_by_rho) + u_sqr;
        temp3 = 0.5 * B1 * temp1;
        temp1 = ut * A1pos + B1;
        temp4 = 0.5 * rho * un * B2 * temp1;
        G[3] = rho * A2neg * (temp2 + temp3) - temp4;
    } else if (quad == 3) {
        double A1pos = 0.5 * (1.0 + erf(S1));
        double A2pos = 0.5 * (1.0 + erf(S2));
        G[0] = rho * A2pos * (ut * A1pos + B1);
        temp1 = pr_by_rho + ut * ut;
        temp2 = temp1 * A1pos + ut * B1;
        G[1] = rho * A2pos * temp2;
        temp1 = ut * A1pos + B1;
        temp2 = un * A2pos + B2;
        G[2] = rho * temp1 * temp2;
        temp1 = (7.0 * pr_by_rho) + u_sqr;
        temp2 = 0.5 * ut * temp1 * A1pos;
        temp1 = (6.0 * pr_by_rho) + u_sqr;
        temp3 = 0.5 * B1 * temp1;
        temp1 = ut * A1pos + B1;
        temp4 = 0.5 * rho * un * B2 * temp1;
        G[3] = rho * A2pos * (temp2 + temp3) + temp4;
    } else {
        double A1neg = 0.5 * (1.0 - erf(S1));
        double A2pos = 0.5 * (1.0 + erf(S2));
        G[0] = rho * A2pos * (ut * A1neg - B1);
        temp1 = pr_by_rho + ut * ut;
        temp2 = temp1 * A1neg - ut * B1;
        G[1] = rho * A2pos * temp2;
        temp1 = ut * A1neg - B1;
        temp2 = un * A2pos + B2;
        G[2] = rho * temp1 * temp2;
        temp1 = (7.0 * pr_by_rho) + u_sqr;
        temp2 = 0.5 * ut * temp1 * A1neg;
        temp1 = (6.0 * pr_by_rho) + u_sqr;
        temp3 = 0.5 * B1 * temp1;
        temp1 = ut * A1neg - B1;
        temp4 = 0.5 * rho * un * B2 * temp1;
        G[3] = rho * A2pos * (temp2 - temp3) + temp4;
    }
}

/* Flux kinds used by the direction routines. */
enum { F_GXP, F_GXN, F_GYP, F_GYN, F_QI, F_QII, F_QIII, F_QIV };

static inline void eval_flux(const orc_t *h, int kind, double G[4], double nx, double ny,
                             double u1, double u2, double rho, double pr) {
    switch (kind) {
    case F_GXP: flux_Gx(G, 1, nx, ny, u1, u2, rho, pr, h->pi); break;
    case F_GXN: flux_Gx(G, 0, nx, ny, u1, u2, rho, pr, h->pi); break;
    case F_GYP: flux_Gy(G, 1, nx, ny, u1, u2, rho, pr, h->pi); break;
    case F_GYN: flux_Gy(G, 0, nx, ny, u1, u2, rho, pr, h->pi); break;
    case F_QI: flux_quad(G, 1, nx, ny, u1, u2, rho, pr, h->pi); break;
    case F_QII: flux_quad(G, 2, nx, ny, u1, u2, rho, pr, h->pi); break;
    case F_QIII: flux_quad(G, 3, nx, ny, u1, u2, rho, pr, h->pi); break;
    default: flux_quad(G, 4, nx, ny, u1, u2, rho, pr, h->pi); break;
    }
}

/* The common body of {wall,outer,interior}_fluxes.F90 dG* routines: LSQ of
 * split-flux differences over one direction list.  yderiv selects the
 * y-derivative formula (the dGy* routines). */
static void dG_direction(const orc_t *h, double G[4], int i, int list, int kind, int yderiv) {
    const double power = h->p.power;
    double sum_delx_sqr = 0.0, sum_dely_sqr = 0.0, sum_delx_dely = 0.0;
    double sum_delx_delf[4] = {0, 0, 0, 0}, sum_dely_delf[4] = {0, 0, 0, 0};
    double x_i = X(i), y_i = Y(i), nx = NX(i), ny = NY(i);
    double tx = ny, ty = -nx;
    for (int j = 1; j <= SPLITN(list, i); ++j) {
        int k = SPLITC(list, i, j);
        double delx = X(k) - x_i, dely = Y(k) - y_i;
        double dels = delx * tx + dely * ty;
        double deln = delx * nx + dely * ny;
        double dist = sqrt(dels * dels + deln * deln);
        double weights = pow(dist, power);
        double dels_weights = dels * weights, deln_weights = deln * weights;
        sum_delx_sqr = sum_delx_sqr + dels * dels_weights;
        sum_dely_sqr = sum_dely_sqr + deln * deln_weights;
        sum_delx_dely = sum_delx_dely + dels * deln_weights;
        double qtilde_i[4], qtilde_k[4], phi_i[4], phi_k[4];
        for (int r = 1; r <= 4; ++r) {
            qtilde_i[r - 1] = Q(r, i) - 0.5 * (delx * DQ(1, r, i) + dely * DQ(2, r, i));
            qtilde_k[r - 1] = Q(r, k) - 0.5 * (delx * DQ(1, r, k) + dely * DQ(2, r, k));
        }
        venkat_limiter(h, qtilde_i, phi_i, i);
        venkat_limiter(h, qtilde_k, phi_k, k);
        for (int r = 1; r <= 4; ++r) {
            qtilde_i[r - 1] = Q(r, i) - 0.5 * phi_i[r - 1] * (delx * DQ(1, r, i) + dely * DQ(2, r, i));
            qtilde_k[r - 1] = Q(r, k) - 0.5 * phi_k[r - 1] * (delx * DQ(1, r, k) + dely * DQ(2, r, k));
        }
        double u1, u2, rho, pr, G_i[4], G_k[4];
        qtilde_to_primitive(qtilde_i, &u1, &u2, &rho, &pr);
        eval_flux(h, kind, G_i, nx, ny, u1, u2, rho, pr);
        qtilde_to_primitive(qtilde_k, &u1, &u2, &rho, &pr);
        eval_flux(h, kind, G_k, nx, ny, u1, u2, rho, pr);
        for (int r = 0; r < 4; ++r) {
            sum_delx_delf[r] = sum_delx_delf[r] + (G_k[r] - G_i[r]) * dels_weights;
            sum_dely_delf[r] = sum_dely_delf[r] + (G_k[r] - G_i[r]) * deln_weights;
        }
    }
    double det = sum_delx_sqr * sum_dely_sqr - sum_delx_dely * sum_delx_dely;
    double one_by_det = 1.0 / det;
    for (int r = 0; r < 4; ++r) {
        if (!yderiv)
            G[r] = (sum_delx_delf[r] * sum_dely_sqr - sum_dely_delf[r] * sum_delx_dely) * one_by_det;
        else
            G[r] = (sum_dely_delf[r] * sum_delx_sqr - sum_delx_delf[r] * sum_delx_dely) * one_by_det;
    }
}

/* flux_residual.F90:14-73 cal_flux_residual.
 * wall:     wall_dGx_pos -> GxII, wall_dGx_neg -> GxI, wall_dGy_neg -> Gyn
 * outer:    outer_dGx_pos -> GxIII, outer_dGx_neg -> GxIV, outer_dGy_pos -> Gyp
 * interior: Gxp, Gxn, Gyp, Gyn */
void orc_cal_flux_residual(orc_t *h) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < h->wall_points; ++i) {
        int k = h->wall_idx[i];
        double Gxp[4], Gxn[4], Gyn[4];
        dG_direction(h, Gxp, k, XPOS, F_QII, 0);
        dG_direction(h, Gxn, k, XNEG, F_QI, 0);
        dG_direction(h, Gyn, k, YNEG, F_GYN, 1);
        for (int r = 1; r <= 4; ++r) FRES(r, k) = Gxp[r - 1] + Gxn[r - 1] + Gyn[r - 1];
        for (int r = 1; r <= 4; ++r) FRES(r, k) = 2.0 * h->delta[k - 1] * FRES(r, k);
    }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < h->outer_points; ++i) {
        int k = h->outer_idx[i];
        double Gxp[4], Gxn[4], Gyp[4];
        dG_direction(h, Gxp, k, XPOS, F_QIII, 0);
        dG_direction(h, Gxn, k, XNEG, F_QIV, 0);
        dG_direction(h, Gyp, k, YPOS, F_GYP, 1);
        for (int r = 1; r <= 4; ++r)
            FRES(r, k) = h->delta[k - 1] * (Gxp[r - 1] + Gxn[r - 1] + Gyp[r - 1]);
    }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < h->interior_points; ++i) {
        int k = h->interior_idx[i];
        double Gxp[4], Gxn[4], Gyp[4], Gyn[4];
        dG_direction(h, Gxp, k, XPOS, F_GXP, 0);
        dG_direction(h, Gxn, k, XNEG, F_GXN, 0);
        dG_direction(h, Gyp, k, YPOS, F_GYP, 1);
        dG_direction(h, Gyn, k, YNEG, F_GYN, 1);
        for (int r = 1; r <= 4; ++r)
            FRES(r, k) = h->delta[k - 1] * (Gxp[r - 1] + Gxn[r - 1] + Gyp[r - 1] + Gyn[r - 1]);
    }
}

/* ------------------------------------------------------------------------ */
/* state_update.F90:144-163 primitive_to_conserved */
static inline void primitive_to_conserved(const double *prim, double nx, double ny, double U[4]) {
    double rho = prim[0];
    U[0] = rho;
    double temp1 = rho * prim[1];
    double temp2 = rho * prim[2];
    U[3] = 2.5 * prim[3] + 0.5 * (temp1 * temp1 + temp2 * temp2) / rho;
    U[1] = temp1 * ny - temp2 * nx;
    U[2] = temp1 * nx + temp2 * ny;
}

/* state_update.F90:239-294 conserved_vector_Ubar (outer kinetic boundary) */
static inline void conserved_vector_Ubar(const orc_t *h, const double *prim, double Ubar[4],
                                         double nx, double ny) {
    const double pi = h->pi;
    double u1_inf = h->q_inf[1], u2_inf = h->q_inf[2];
    double tx = ny, ty = -nx;
    double u1_inf_rot = u1_inf * tx + u2_inf * ty;
    double u2_inf_rot = u1_inf * nx + u2_inf * ny;
    double temp1 = (u1_inf_rot * u1_inf_rot + u2_inf_rot * u2_inf_rot);
    double e_inf = PR_INF / (RHO_INF * (GAMMA - 1.0)) + 0.5 * (temp1);
    double beta = (0.5 * RHO_INF) / PR_INF;
    double S2 = u2_inf_rot * sqrt(beta);
    double B2_inf = exp(-S2 * S2) / (2.0 * sqrt(pi * beta));
    double A2n_inf = 0.5 * (1.0 - erf(S2));
    double rho = prim[0], u1 = prim[1], u2 = prim[2], pr = prim[3];
    double u1_rot = u1 * tx + u2 * ty;
    double u2_rot = u1 * nx + u2 * ny;
    temp1 = (u1_rot * u1_rot + u2_rot * u2_rot);
    double e = pr / (rho * (GAMMA - 1.0)) + 0.5 * (temp1);
    beta = (rho) / (2.0 * pr);
    S2 = u2_rot * sqrt(beta);
    double B2 = exp(-S2 * S2) / (2.0 * sqrt(pi * beta));
    double A2p = 0.5 * (1.0 + erf(S2));
    Ubar[0] = (RHO_INF * A2n_inf) + (rho * A2p);
    Ubar[1] = (RHO_INF * u1_inf_rot * A2n_inf) + (rho * u1_rot * A2p);
    temp1 = RHO_INF * (u2_inf_rot * A2n_inf - B2_inf);
    double temp2 = rho * (u2_rot * A2p + B2);
    Ubar[2] = temp1 + temp2;
    temp1 = (RHO_INF * A2n_inf * e_inf - 0.5 * RHO_INF * u2_inf_rot * B2_inf);
    temp2 = (rho * A2p * e + 0.5 * rho * u2_rot * B2);
    Ubar[3] = temp1 + temp2;
}

/* state_update.F90:10-141 state_update.  Returns the per-point res_sqr in
 * res (wall/interior; 0 for outer) so the serial sum keeps reference order. */
static void update_point(orc_t *h, int k, int rk, int kind, double *res) {
    const double obt = 1.0 / 3.0, tbt = 2.0 / 3.0;
    const double euler = h->p.euler;
    double nx = NX(k), ny = NY(k), U[4], U_old[4];
    if (kind == 2) {
        conserved_vector_Ubar(h, &PRIM(1, k), U, nx, ny);
        conserved_vector_Ubar(h, &PRIMO(1, k), U_old, nx, ny);
    } else {
        primitive_to_conserved(&PRIM(1, k), nx, ny, U);
        primitive_to_conserved(&PRIMO(1, k), nx, ny, U_old);
    }
    double temp = U[0];
    for (int r = 0; r < 4; ++r) {
        if (rk != 3) U[r] = U[r] - (0.5 * euler * FRES(r + 1, k));
        else U[r] = tbt * U_old[r] + obt * (U[r] - 0.5 * FRES(r + 1, k));
    }
    if (kind == 0) U[2] = 0.0;
    double U2_rot = U[1], U3_rot = U[2];
    U[1] = U2_rot * ny + U3_rot * nx;
    U[2] = U3_rot * ny - U2_rot * nx;
    *res = (kind == 2) ? 0.0 : (U[0] - temp) * (U[0] - temp);
    PRIM(1, k) = U[0];
    temp = 1.0 / U[0];
    PRIM(2, k) = U[1] * temp;
    PRIM(3, k) = U[2] * temp;
    PRIM(4, k) = 0.4 * (U[3] - (0.5 * temp) * (U[1] * U[1] + U[2] * U[2]));
}

void orc_state_update(orc_t *h, int rk) {
    double *res = malloc(sizeof(double) * (size_t)(h->n > 0 ? h->n : 1));
    int nw = h->wall_points, no = h->outer_points, ni = h->interior_points;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nw; ++i) update_point(h, h->wall_idx[i], rk, 0, &res[i]);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < no; ++i) update_point(h, h->outer_idx[i], rk, 2, &res[nw + i]);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < ni; ++i) update_point(h, h->interior_idx[i], rk, 1, &res[nw + no + i]);
    /* sum_res_sqr accumulates wall points, then interior points */
    double s = 0.0;
    for (int i = 0; i < nw; ++i) s = s + res[i];
    for (int i = 0; i < ni; ++i) s = s + res[nw + no + i];
    h->sum_res_sqr = s;
    free(res);
}

double orc_sum_res_sqr(const orc_t *h) { return h->sum_res_sqr; }

/* state_update.F90:190-236 func_delta */
void orc_func_delta(orc_t *h) {
    const double cfl = h->p.cfl;
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= h->n_local; ++i) {
        double min_delt = 1.0;
        for (int r = 1; r <= NBHS(i); ++r) {
            int k = CONN(i, r);
            double rho = PRIM(1, k), u1 = PRIM(2, k), u2 = PRIM(3, k), pr = PRIM(4, k);
            double x_i = X(i), y_i = Y(i), x_k = X(k), y_k = Y(k);
            double dist = (x_k - x_i) * (x_k - x_i) + (y_k - y_i) * (y_k - y_i);
            dist = sqrt(dist);
            double mod_u = sqrt(u1 * u1 + u2 * u2);
            double delta_t = dist / (mod_u + 3.0 * sqrt(pr / rho));
            delta_t = cfl * delta_t;
            if (min_delt > delta_t) min_delt = delta_t;
        }
        h->delta[i - 1] = min_delt;
    }
}

/* fpi_solver.F90:13-83 (the objective/cp-file write is left to orc_forces) */
static void fpi_solver(orc_t *h, int t) {
    orc_save_prim_old(h);
    orc_func_delta(h);
    for (int rk = 1; rk <= h->p.rks; ++rk) {
        orc_eval_q_variables(h);
        orc_eval_q_derivatives(h);
        for (int i = 1; i <= h->p.inner_iterations; ++i) {
            orc_eval_q_inner_loop(h);
            orc_eval_update_innerloop(h);
        }
        orc_cal_flux_residual(h);
        orc_state_update(h, rk);
    }
    h->res_new = sqrt(h->sum_res_sqr) / h->plen;
    if (t <= 2 && h->p.restart == 0) {
        h->res_old = h->res_new;
        h->residue = 0.0;
    } else {
        h->residue = log10(h->res_new / h->res_old);
    }
}

/* q_lskum.F90:59-73 */
int orc_run(orc_t *h, int it_first, int n_iters, double *residue, int *n_done) {
    int done = 0;
    for (int it = it_first; it < it_first + n_iters; ++it) {
        fpi_solver(h, it);
        if (residue) residue[done] = h->residue;
        ++done;
        if (isnan(h->residue)) break;
    }
    if (n_done) *n_done = done;
    return isnan(h->residue) ? 1 : 0;
}

/* compute_force_coeffs.F90:11-102 */
/* src_cuda/adaptation_sensors.F90:35-101 sensor_D2_distance, one point */
static double d2_distance(const orc_t *h, int i) {
    double u1_i = PRIM(2, i), u2_i = PRIM(3, i), rho_i = PRIM(1, i), pr_i = PRIM(4, i);
    double maxi = 0.0;
    for (int r = 1; r <= NBHS(i); ++r) {
        int j = CONN(i, r);
        double u1_j = PRIM(2, j), u2_j = PRIM(3, j), rho_j = PRIM(1, j), pr_j = PRIM(4, j);
        double temp1 = (pr_i * pr_i * rho_j) / (pr_j * pr_j * rho_i);
        temp1 = log(temp1);
        temp1 = (rho_j - rho_i) * temp1;
        double u_sqr = (u1_j - u1_i) * (u1_j - u1_i) + (u2_j - u2_i) * (u2_j - u2_i);
        double temp2 = (rho_j / rho_i) + (pr_i * rho_j) / (pr_j * rho_i);
        temp2 = temp2 * u_sqr;
        temp2 = (0.5 * rho_i * rho_i / pr_i) * temp2;
        double temp3 = rho_i * (((pr_i * rho_j) / (pr_j * rho_i)) - 1);
        temp3 = temp3 + rho_j * (((pr_j * rho_i) / (pr_i * rho_j)) - 1);
        temp3 = 2 * temp3;
        double D2_dist = temp1 + temp2 + temp3;
        if (D2_dist > maxi) maxi = D2_dist;
    }
    return maxi;
}

double orc_output_fields(const orc_t *h, double *mach, double *entropy, double *sensor) {
    const double gamma = GAMMA;
    double total_entropy = 0.0, max_sensor = 0.0;
    double temp2 = log(PR_INF);
    double *d2 = malloc(sizeof(double) * (size_t)h->n);
    for (int k = 1; k <= h->n; ++k) {
        /* post_processing.F90:24-27 */
        double sos = sqrt(gamma * PRIM(4, k) / PRIM(1, k));
        double vel_mag = PRIM(2, k) * PRIM(2, k) + PRIM(3, k) * PRIM(3, k);
        if (mach) mach[k - 1] = sqrt(vel_mag / sos);
        /* compute_entropy.F90:21-27 */
        double temp1 = pow(PRIM(1, k), gamma);
        temp1 = PRIM(4, k) / temp1;
        temp1 = log(temp1);
        if (entropy) entropy[k - 1] = fabs(temp1 - temp2);
        total_entropy = total_entropy + fabs(temp1 - temp2);
        d2[k - 1] = d2_distance(h, k);
    }
    /* adaptation_sensors.F90:18-30 */
    for (int k = 0; k < h->n; ++k)
        if (d2[k] >= max_sensor) max_sensor = d2[k];
    if (sensor)
        for (int k = 0; k < h->n; ++k) sensor[k] = d2[k] / max_sensor;
    free(d2);
    return total_entropy;
}

double orc_objective(const orc_t *h, int kind) {
    const double gamma = GAMMA;
    if (kind == 2) {
        /* compute_entropy.F90:19-30 */
        double total_entropy = 0.0, temp2 = log(PR_INF);
        for (int k = 1; k <= h->n; ++k) {
            double temp1 = pow(PRIM(1, k), gamma);
            temp1 = PRIM(4, k) / temp1;
            temp1 = log(temp1);
            total_entropy = total_entropy + fabs(temp1 - temp2);
        }
        return total_entropy;
    }
    if (kind == 3) {
        /* compute_enstrophy.F90:25-79 */
        double total_enstrophy = 0.0;
        for (int i = 1; i <= h->n; ++i) {
            double x_i = X(i), y_i = Y(i);
            double sum_delx_sqr = 0.0, sum_dely_sqr = 0.0, sum_delx_dely = 0.0;
            double sum_delx_delu1 = 0.0, sum_dely_delu1 = 0.0, sum_delx_delu2 = 0.0,
                   sum_dely_delu2 = 0.0;
            for (int k = 1; k <= NBHS(i); ++k) {
                int nbh = CONN(i, k);
                double delx = X(nbh) - x_i, dely = Y(nbh) - y_i;
                double dist = sqrt(delx * delx + dely * dely);
                double weights = pow(dist, h->p.power);
                sum_delx_sqr = sum_delx_sqr + delx * delx * weights;
                sum_dely_sqr = sum_dely_sqr + dely * dely * weights;
                sum_delx_dely = sum_delx_dely + delx * dely * weights;
                sum_delx_delu1 = sum_delx_delu1 + weights * delx * (PRIM(2, nbh) - PRIM(2, i));
                sum_delx_delu2 = sum_delx_delu2 + weights * delx * (PRIM(3, nbh) - PRIM(3, i));
                sum_dely_delu1 = sum_dely_delu1 + weights * dely * (PRIM(2, nbh) - PRIM(2, i));
                sum_dely_delu2 = sum_dely_delu2 + weights * dely * (PRIM(3, nbh) - PRIM(3, i));
            }
            double det = sum_delx_sqr * sum_dely_sqr - sum_delx_dely * sum_delx_dely;
            double one_by_det = 1.0 / det;
            double du2_dx = (sum_delx_delu2 * sum_dely_sqr - sum_dely_delu2 * sum_delx_dely) * one_by_det;
            double du1_dy = (sum_dely_delu1 * sum_delx_sqr - sum_delx_delu1 * sum_delx_dely) * one_by_det;
            double temp = du2_dx - du1_dy;
            total_enstrophy = total_enstrophy + temp * temp;
        }
        return total_enstrophy;
    }
    /* stagnation_values.F90:52-73 objective_function_J */
    double gammaPower = gamma / (gamma - 1);
    double p0_inf = PR_INF * pow(1 + ((gamma - 1) / 2) * h->p.mach * h->p.mach, gammaPower);
    double constant = 1 / (p0_inf * p0_inf * h->n);
    double p0_sum = 0.0;
    for (int i = 1; i <= h->n; ++i) {
        double angle = sqrt(gamma * PRIM(4, i) / PRIM(1, i));
        double mach_t = sqrt(PRIM(2, i) * PRIM(2, i) + PRIM(3, i) * PRIM(3, i)) / angle;
        double p0 = PRIM(4, i) * pow(1 + ((gamma - 1) / 2) * mach_t * mach_t, gammaPower);
        p0_sum = p0_sum + (p0_inf - p0) * (p0_inf - p0);
    }
    return p0_sum * constant;
}

void orc_forces(orc_t *h, double *cl, double *cd, double *cm, double *cp_out) {
    int shapes = h->p.shapes;
    double *H = calloc((size_t)shapes, sizeof(double));
    double *V = calloc((size_t)shapes, sizeof(double));
    double *pm = calloc((size_t)shapes, sizeof(double));
    double temp = 0.5 * RHO_INF * h->p.mach * h->p.mach;
    for (int j = 0; j < h->shape_points; ++j) {
        int m = h->shape_idx[j], r = h->right[m - 1], l = h->left[m - 1];
        double lx = X(l), ly = Y(l), mx = X(m), my = Y(m), rx = X(r), ry = Y(r);
        double ds1 = (mx - lx) * (mx - lx) + (my - ly) * (my - ly);
        ds1 = sqrt(ds1);
        double ds2 = (rx - mx) * (rx - mx) + (ry - my) * (ry - my);
        ds2 = sqrt(ds2);
        double ds = 0.5 * (ds1 + ds2);
        double nx = NX(m), ny = NY(m);
        double cp = PRIM(4, m) - PR_INF;
        cp = -cp / temp;
        if (cp_out) cp_out[j] = cp;
        int s = h->flag_2[m - 1] - 1;
        H[s] = H[s] + cp * nx * ds;
        V[s] = V[s] + cp * ny * ds;
        pm[s] = pm[s] + (-cp * ny * ds * (mx - 0.25) + cp * nx * ds * (my));
    }
    for (int s = 0; s < shapes; ++s) {
        cl[s] = V[s] * cos(h->theta) - H[s] * sin(h->theta);
        cd[s] = H[s] * cos(h->theta) + V[s] * sin(h->theta);
        cm[s] = pm[s];
    }
    free(H); free(V); free(pm);
}

int orc_get(const orc_t *h, const char *name, double *out) {
    size_t n = (size_t)h->n;
    const double *src = NULL;
    size_t cnt = 0;
    if (!strcmp(name, "prim")) { src = h->prim; cnt = 4 * n; }
    else if (!strcmp(name, "prim_old")) { src = h->prim_old; cnt = 4 * n; }
    else if (!strcmp(name, "q")) { src = h->q; cnt = 4 * n; }
    else if (!strcmp(name, "dq")) { src = h->dq; cnt = 8 * n; }
    else if (!strcmp(name, "qm")) { src = h->qm; cnt = 8 * n; }
    else if (!strcmp(name, "flux_res")) { src = h->flux_res; cnt = 4 * n; }
    else if (!strcmp(name, "delta")) { src = h->delta; cnt = n; }
    else if (!strcmp(name, "nx")) { src = h->nx; cnt = n; }
    else if (!strcmp(name, "ny")) { src = h->ny; cnt = n; }
    else if (!strcmp(name, "temp")) { src = h->temp; cnt = 12 * n; }
    else return -1;
    memcpy(out, src, cnt * sizeof(double));
    return 0;
}

int orc_set(orc_t *h, const char *name, const double *in) {
    size_t n = (size_t)h->n;
    double *dst = NULL;
    size_t cnt = 0;
    if (!strcmp(name, "prim")) { dst = h->prim; cnt = 4 * n; }
    else if (!strcmp(name, "dq")) { dst = h->dq; cnt = 8 * n; }
    else if (!strcmp(name, "qm")) { dst = h->qm; cnt = 8 * n; }
    else return -1;
    memcpy(dst, in, cnt * sizeof(double));
    return 0;
}

void orc_get_split_counts(const orc_t *h, int *out) {
    for (int i = 0; i < h->n; ++i)
        for (int d = 0; d < 4; ++d) out[4 * i + d] = h->nb_cnt[d][i];
}
