// Internal interface of the reverse (adjoint) kernels.
#pragma once

#include <cuda_runtime.h>

#include "primal.h"

namespace lskum {

constexpr int ADJ_CW = 22;  // contribution record per (point, slot)
// flux pass: per (point, slot) the neighbour side's record (adjoint of its
// reconstructed u1, u2, rho, p; its rho; delx/dely adjoint; padding)
constexpr int NBREC = 8;
// q-derivative pass: per point the record its neighbours' side reads
constexpr int GREC = 24;
enum { ADJ_GATHER_INNER = 1, ADJ_GATHER_GRAD = 2 };

struct AdjConsts {
    double q_inf[4];
};

// Shape points in grid order with their renumbered ring neighbours.
struct AdjShape {
    int npts;
    const int *idx, *left, *right;
    const double *nx, *ny;
};

// Source lists of the gather forms of the force and normal reverses (one
// thread per boundary point; see k_forces_b_gather).  Null pointers select
// the single-thread kernels.
struct AdjGather {
    int nbnd;
    const int *fptr, *fsrc;  // forces: 3 j + role, per boundary point
    const int *nptr, *nsrc;  // normals: 2 j + role, per boundary point
};

cudaError_t init_adjoint_kernels();
void launch_update_b(const Geom &g, const Consts &c, const AdjConsts &a, const R4 *prim_in,
                     const R4 *prim_old, const R4 *fr, const double *pb_out, double *pb_in,
                     double *pb_old, double *frb, double *nxb, double *nyb, int rk,
                     cudaStream_t s);
// kst: the stage's kinetic-state tape of the forward re-run ([n][kp][KS_TAPE],
// written by the flux pass with StageBufs::kstape), or nullptr to recompute
// The flux pass reverses in two kernels: k_flux_b per point (its fluxes,
// kinetic states and own reconstruction; writes nbrec [n][kp][NBREC]) and
// k_flux_b_nbr per neighbour over the transposed stencil (the neighbour's
// reconstruction; writes back [n][kp] (delx, dely) adjoint parts that
// belong to the point as well), then k_back_sum adds those to the point.
// nbrec and back may share the contribution buffer (n*kp*(NBREC+2) <=
// n*kp*ADJ_CW doubles).
void launch_flux_b(const Geom &g, const Consts &c, const R4 *q_in, const double *dq,
                   const double *qm, const double *delta, const double *frb, double *qb,
                   double *dqb, double *qmb, double *xb, double *yb, double *nxb, double *nyb,
                   double *deltab, double *nbrec, double *back, const int *tptr,
                   const int *tlist, const double *kst, cudaStream_t s);
void launch_inner_b(const Geom &g, const R4 *q, const double *dq_in, const double *dqb_out,
                    double *dqb_in, double *qb, double *xb, double *yb, double *contrib,
                    cudaStream_t s);
// spdA: |u| + 3 sqrt(p/rho) of primA as the forward pass used it (taped).
// Two kernels: k_grad_b per point (its own side; writes grec [n][GREC], which
// may share the contribution buffer) and k_grad_b_nbr per neighbour over the
// transposed stencil (adds to qb, pb = primA's adjoint, xb, yb).
void launch_grad_b(const Geom &g, const Consts &c, const R4 *q, const R4 *primA,
                   const double *spdA, const double *dqb, const double *qmb,
                   const double *deltab, bool with_delta, double *qb, double *pb, double *xb,
                   double *yb, double *grec, const int *tptr, const int *tlist,
                   cudaStream_t s);
void launch_gather(int n, int kp, const int *tptr, const int *tlist, const double *contrib,
                   int mode, double *a4, double *a8, double *b8, double *xb, double *yb,
                   cudaStream_t s);
void launch_qvar_b(int n, const R4 *prim, const double *qb, double *pb, cudaStream_t s);
void launch_forces_b(const AdjShape &t, const AdjGather &gth, const R4 *prim, const double2 *xy,
                     double mach, double cos_t, double sin_t, int objective, double *pb,
                     double *xb, double *yb, double *nxb, double *nyb, cudaStream_t s);
void launch_normals_b(int nbnd, const AdjGather &gth, const int *left, const int *right,
                      const double2 *xy, const double *nxb, const double *nyb, double *xb,
                      double *yb, cudaStream_t s);

}  // namespace lskum
