// mfcfd_tangent: forward-mode (tangent) derivative of the pseudo-time loop.
//
// The reference's tangent driver Q_LSKUM_D (src_mpi_forward/sensitivity_files/
// q_lskum_d.F90:28-89) seeds pointd%x(1) = 1, differentiates
// COMPUTE_NORMALS_D and every FPI_SOLVER_D iteration and returns the
// derivative of the objective.  Here the seed is any direction (dx, dy) over
// all points: the loop runs n iterations from the handle's state (held
// fixed) with every quantity carried as a Dual (value, derivative), and the
// result is J = sum over shapes of Cl or Cd of the final state and dJ/de in
// that direction.  For the reverse-mode gradient g of mfcfd_adjoint,
// dJ/de = <g, (dx, dy)> (the dot-product test).
//
// The kernels are plain thread-per-point passes over the same device
// templates as the primal (reconstruct, kstate, split/quadrant fluxes,
// q_from_prim, prim_to_conserved, conserved_ubar) instantiated on Dual, with
// each list sum in slot order; min_dist is data, as in the reference.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

// handle.h (and through it the primal device templates) comes before
// dual.cuh: the templates' double instantiations must see only the libm
// overloads, and the Dual ones are found by argument-dependent lookup.
#include "handle.h"
#include "dual.cuh"
#include "objective.h"

using namespace lskum;
using lskum_host::cuda_fail;
using lskum_host::dmalloc;
using lskum_host::fail;

namespace {

constexpr int TB = 128;
constexpr double OBT = 1.0 / 3.0;
constexpr double TBT = 2.0 / 3.0;

// value / derivative arrays of the tangent state
struct TanState {
    const double2 *xy_t, *nrm_t;  // derivatives of (x, y) and (nx, ny)
    const Dual *obc;              // outer points: 8 Duals per point
    R4 *pv[2], *pt[2];            // prim
    R4 *qv[2], *qt[2];            // q
    double *dqv[2], *dqt[2];      // dq [n][8]
    double *qmv, *qmt;            // qm [n][8]
    double *dlv, *dlt;            // delta
    double *spv, *spt;            // spd
};

__device__ __forceinline__ void ld_dual4(const R4 *v, const R4 *t, int i, Dual out[4]) {
    const R4 a = v[i], b = t[i];
    out[0] = Dual(a.a, b.a);
    out[1] = Dual(a.b, b.b);
    out[2] = Dual(a.c, b.c);
    out[3] = Dual(a.d, b.d);
}
__device__ __forceinline__ void st_dual4(R4 *v, R4 *t, int i, const Dual x[4]) {
    v[i] = R4{x[0].v, x[1].v, x[2].v, x[3].v};
    t[i] = R4{x[0].d, x[1].d, x[2].d, x[3].d};
}
__device__ __forceinline__ void ld_dual8(const double *v, const double *t, int i, Dual a[4],
                                         Dual b[4]) {
    for (int m = 0; m < 4; ++m) {
        a[m] = Dual(v[8 * (size_t)i + m], t[8 * (size_t)i + m]);
        b[m] = Dual(v[8 * (size_t)i + 4 + m], t[8 * (size_t)i + 4 + m]);
    }
}
__device__ __forceinline__ void st_dual8(double *v, double *t, int i, const Dual a[4],
                                         const Dual b[4]) {
    for (int m = 0; m < 4; ++m) {
        v[8 * (size_t)i + m] = a[m].v;
        t[8 * (size_t)i + m] = a[m].d;
        v[8 * (size_t)i + 4 + m] = b[m].v;
        t[8 * (size_t)i + 4 + m] = b[m].d;
    }
}
__device__ __forceinline__ void xy_dual(const Geom &g, const TanState &s, int i, Dual &x,
                                        Dual &y) {
    const double2 p = g.xy[i], d = s.xy_t[i];
    x = Dual(p.x, d.x);
    y = Dual(p.y, d.y);
}

// q and spd of the initial state (its derivative is zero: prim_0 is held fixed)
__global__ void k_t_init(int n, TanState s, int cur, int qc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Dual P[4], q[4];
    ld_dual4(s.pv[cur], s.pt[cur], i, P);
    q_from_prim_t<Dual>(P[0], P[1], P[2], P[3], q);
    st_dual4(s.qv[qc], s.qt[qc], i, q);
    const Dual spd = sqrt(P[1] * P[1] + P[2] * P[2]) + Dual(3.0) * sqrt(P[3] / P[0]);
    s.spv[i] = spd.v;
    s.spt[i] = spd.d;
}

// eval_q_derivatives_d + func_delta_d (q_variables_d.F90, state_update_d.F90)
__global__ void __launch_bounds__(TB)
k_t_grad(Geom g, Consts c, TanState s, int qc, int with_delta) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.n) return;
    Dual xi, yi, qi[4];
    xy_dual(g, s, i, xi, yi);
    ld_dual4(s.qv[qc], s.qt[qc], i, qi);
    Dual qmax[4], qmin[4], sdxq[4], sdyq[4];
    for (int m = 0; m < 4; ++m) {
        qmax[m] = qi[m];
        qmin[m] = qi[m];
    }
    Dual sdx2, sdy2, sdxy, min_delt(1.0);
    const int nb = g.nbhs[i];
    for (int r = 0; r < nb; ++r) {
        const int k = g.conn[r * g.n + i];
        Dual xk, yk, qk[4];
        xy_dual(g, s, k, xk, yk);
        ld_dual4(s.qv[qc], s.qt[qc], k, qk);
        for (int m = 0; m < 4; ++m) {
            if (qk[m] > qmax[m]) qmax[m] = qk[m];
            if (qk[m] < qmin[m]) qmin[m] = qk[m];
        }
        const Dual delx = xk - xi, dely = yk - yi;
        const Dual dist = sqrt(delx * delx + dely * dely);
        sdx2 = sdx2 + delx * delx;
        sdy2 = sdy2 + dely * dely;
        sdxy = sdxy + delx * dely;
        for (int m = 0; m < 4; ++m) {
            sdxq[m] = sdxq[m] + delx * (qk[m] - qi[m]);
            sdyq[m] = sdyq[m] + dely * (qk[m] - qi[m]);
        }
        if (with_delta) {
            Dual delta_t = dist / Dual(s.spv[k], s.spt[k]);
            delta_t = Dual(c.cfl) * delta_t;
            if (min_delt > delta_t) min_delt = delta_t;
        }
    }
    const Dual one_by_det = Dual(1.0) / (sdx2 * sdy2 - sdxy * sdxy);
    Dual dx[4], dy[4];
    for (int m = 0; m < 4; ++m) {
        dx[m] = (sdxq[m] * sdy2 - sdyq[m] * sdxy) * one_by_det;
        dy[m] = (sdyq[m] * sdx2 - sdxq[m] * sdxy) * one_by_det;
    }
    st_dual8(s.dqv[0], s.dqt[0], i, dx, dy);
    st_dual8(s.qmv, s.qmt, i, qmax, qmin);
    if (with_delta) {
        s.dlv[i] = min_delt.v;
        s.dlt[i] = min_delt.d;
    }
}

// eval_q_inner_loop_d + eval_update_innerloop_d: dq buffer a -> a ^ 1
__global__ void __launch_bounds__(TB)
k_t_inner(Geom g, TanState s, int qc, int a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.n) return;
    Dual xi, yi, qi[4], dxi[4], dyi[4];
    xy_dual(g, s, i, xi, yi);
    ld_dual4(s.qv[qc], s.qt[qc], i, qi);
    ld_dual8(s.dqv[a], s.dqt[a], i, dxi, dyi);
    Dual sdx2, sdy2, sdxy, sdxq[4], sdyq[4];
    const int nb = g.nbhs[i];
    for (int r = 0; r < nb; ++r) {
        const int k = g.conn[r * g.n + i];
        Dual xk, yk, qk[4], dxk[4], dyk[4];
        xy_dual(g, s, k, xk, yk);
        ld_dual4(s.qv[qc], s.qt[qc], k, qk);
        ld_dual8(s.dqv[a], s.dqt[a], k, dxk, dyk);
        const Dual delx = xk - xi, dely = yk - yi;
        sdx2 = sdx2 + delx * delx;
        sdy2 = sdy2 + dely * dely;
        sdxy = sdxy + delx * dely;
        for (int m = 0; m < 4; ++m) {
            const Dual temp1 = qi[m] - Dual(0.5) * (delx * dxi[m] + dely * dyi[m]);
            const Dual temp2 = qk[m] - Dual(0.5) * (delx * dxk[m] + dely * dyk[m]);
            sdxq[m] = sdxq[m] + (delx * (temp2 - temp1));
            sdyq[m] = sdyq[m] + (dely * (temp2 - temp1));
        }
    }
    const Dual one_by_det = Dual(1.0) / (sdx2 * sdy2 - sdxy * sdxy);
    Dual dx[4], dy[4];
    for (int m = 0; m < 4; ++m) {
        dx[m] = one_by_det * (sdxq[m] * sdy2 - sdyq[m] * sdxy);
        dy[m] = one_by_det * (sdyq[m] * sdx2 - sdxq[m] * sdxy);
    }
    st_dual8(s.dqv[a ^ 1], s.dqt[a ^ 1], i, dx, dy);
}

// cal_flux_residual_d + state_update_d + eval_q_variables_d of the new state.
// Each list is summed over its slots in slot order (the reference's order);
// the states of a neighbour in two lists are recomputed per list.
__global__ void __launch_bounds__(TB)
k_t_flux(Geom g, Consts c, TanState s, int A, int B, int qc, int dqa, int rk, int last) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.n) return;
    const int kind = i < g.nw ? KIND_WALL : (i < g.nw + g.no ? KIND_OUTER : KIND_INTERIOR);
    Dual xi, yi;
    xy_dual(g, s, i, xi, yi);
    const Dual nx(g.nrm[i].x, s.nrm_t[i].x), ny(g.nrm[i].y, s.nrm_t[i].y);
    const Dual pi_c(c.pi), gm1(c.gm1), eps2i(g.eps2[i]);
    Dual qi[4], dxi[4], dyi[4], qmaxi[4], qmini[4];
    ld_dual4(s.qv[qc], s.qt[qc], i, qi);
    ld_dual8(s.dqv[dqa], s.dqt[dqa], i, dxi, dyi);
    ld_dual8(s.qmv, s.qmt, i, qmaxi, qmini);
    const int nb = g.nbhs[i];
    const unsigned long long mx = g.mx[i], my = g.my[i];
    const Dual s2q(kind == KIND_WALL ? -1.0 : 1.0);
    const Dual tx = ny, ty = -nx;
    Dual G[4][4];
    for (int L = 0; L < 4; ++L) {
        if ((kind == KIND_WALL && L == 2) || (kind == KIND_OUTER && L == 3)) continue;
        const unsigned long long bits = ((L < 2) ? mx : my) >> ((L & 1) ? 32 : 0);
        const Dual sg((L & 1) ? -1.0 : 1.0);
        Dual sdx2, sdy2, sdxy, fx[4], fy[4];
        for (int r = 0; r < nb; ++r) {
            if (!((bits >> r) & 1ull)) continue;
            const int k = g.conn[r * g.n + i];
            Dual xk, yk;
            xy_dual(g, s, k, xk, yk);
            const Dual delx = xk - xi, dely = yk - yi;
            Dual qk[4], dxk[4], dyk[4], qmaxk[4], qmink[4];
            ld_dual4(s.qv[qc], s.qt[qc], k, qk);
            ld_dual8(s.dqv[dqa], s.dqt[dqa], k, dxk, dyk);
            ld_dual8(s.qmv, s.qmt, k, qmaxk, qmink);
            Dual u1, u2, rho, pr;
            reconstruct<Dual>(qk, dxk, dyk, qmaxk, qmink, Dual(g.eps2[k]), delx, dely, gm1, u1,
                              u2, rho, pr);
            const KStateT<Dual> sk = kstate<Dual>(u1, u2, rho, pr, nx, ny, pi_c);
            reconstruct<Dual>(qi, dxi, dyi, qmaxi, qmini, eps2i, delx, dely, gm1, u1, u2, rho,
                              pr);
            const KStateT<Dual> si = kstate<Dual>(u1, u2, rho, pr, nx, ny, pi_c);
            Dual Gi[4], Gk[4];
            if (L < 2) {
                if (kind == KIND_INTERIOR) {
                    flux_gx<Dual>(si, sg, Gi);
                    flux_gx<Dual>(sk, sg, Gk);
                } else {
                    flux_quad<Dual>(si, sg, s2q, Gi);
                    flux_quad<Dual>(sk, sg, s2q, Gk);
                }
            } else {
                flux_gy<Dual>(si, sg, Gi);
                flux_gy<Dual>(sk, sg, Gk);
            }
            const Dual dels = delx * tx + dely * ty;
            const Dual deln = delx * nx + dely * ny;
            sdx2 = sdx2 + dels * dels;
            sdy2 = sdy2 + deln * deln;
            sdxy = sdxy + dels * deln;
            for (int m = 0; m < 4; ++m) {
                const Dual d = Gk[m] - Gi[m];
                fx[m] = fx[m] + d * dels;
                fy[m] = fy[m] + d * deln;
            }
        }
        const Dual one_by_det = Dual(1.0) / (sdx2 * sdy2 - sdxy * sdxy);
        for (int m = 0; m < 4; ++m)
            G[L][m] = L < 2 ? (fx[m] * sdy2 - fy[m] * sdxy) * one_by_det
                            : (fy[m] * sdx2 - fx[m] * sdxy) * one_by_det;
    }
    // state_update_d (state_update_d.F90)
    const Dual delta(s.dlv[i], s.dlt[i]);
    Dual fr[4];
    for (int m = 0; m < 4; ++m) {
        if (kind == KIND_WALL) fr[m] = Dual(2.0) * delta * (G[0][m] + G[1][m] + G[3][m]);
        else if (kind == KIND_OUTER) fr[m] = delta * (G[0][m] + G[1][m] + G[2][m]);
        else fr[m] = delta * (G[0][m] + G[1][m] + G[2][m] + G[3][m]);
    }
    Dual P[4], U[4], Uo[4];
    ld_dual4(rk == 1 ? s.pv[A] : s.pv[B], rk == 1 ? s.pt[A] : s.pt[B], i, P);
    if (kind == KIND_OUTER) {
        const Dual *inf = s.obc + 8 * (size_t)(i - g.nw);
        conserved_ubar_t<Dual>(P[0], P[1], P[2], P[3], nx, ny, inf, pi_c, gm1, U);
        if (rk == 3) {
            Dual O[4];
            ld_dual4(s.pv[A], s.pt[A], i, O);
            conserved_ubar_t<Dual>(O[0], O[1], O[2], O[3], nx, ny, inf, pi_c, gm1, Uo);
        }
    } else {
        prim_to_conserved_t<Dual>(P[0], P[1], P[2], P[3], nx, ny, U);
        if (rk == 3) {
            Dual O[4];
            ld_dual4(s.pv[A], s.pt[A], i, O);
            prim_to_conserved_t<Dual>(O[0], O[1], O[2], O[3], nx, ny, Uo);
        }
    }
    for (int m = 0; m < 4; ++m) {
        if (rk != 3) U[m] = U[m] - (Dual(0.5 * c.euler) * fr[m]);
        else U[m] = Dual(TBT) * Uo[m] + Dual(OBT) * (U[m] - Dual(0.5) * fr[m]);
    }
    if (kind == KIND_WALL) U[2] = Dual(0.0);
    const Dual U2_rot = U[1], U3_rot = U[2];
    U[1] = U2_rot * ny + U3_rot * nx;
    U[2] = U3_rot * ny - U2_rot * nx;
    Dual out[4], qn[4];
    out[0] = U[0];
    const Dual temp = Dual(1.0) / U[0];
    out[1] = U[1] * temp;
    out[2] = U[2] * temp;
    out[3] = Dual(0.4) * (U[3] - (Dual(0.5) * temp) * (U[1] * U[1] + U[2] * U[2]));
    st_dual4(s.pv[B], s.pt[B], i, out);
    q_from_prim_t<Dual>(out[0], out[1], out[2], out[3], qn);
    st_dual4(s.qv[qc ^ 1], s.qt[qc ^ 1], i, qn);
    if (last) {
        const Dual spd = sqrt(out[1] * out[1] + out[2] * out[2]) + Dual(3.0) * sqrt(out[3] / out[0]);
        s.spv[i] = spd.v;
        s.spt[i] = spd.d;
    }
}

struct TanShape {
    int npts, shapes;
    const int *idx, *left, *right, *shape;
};

// compute_cl_cd_cm_d (compute_force_coeffs_d.F90), one thread, shape points
// in grid order: out[0] = J, out[1] = dJ/de.
__global__ void k_t_forces(Geom g, TanState s, TanShape t, int cur, double mach, double cos_t,
                           double sin_t, int objective, double *out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double pr_inf = 1.0 / 1.4;
    const Dual temp(0.5 * 1.0 * mach * mach);
    Dual J;
    for (int sh = 0; sh < t.shapes; ++sh) {
        Dual H, V;
        for (int j = 0; j < t.npts; ++j) {
            if (t.shape[j] != sh) continue;
            const int m = t.idx[j], l = t.left[j], r = t.right[j];
            Dual lx, ly, mxx, myy, rx, ry;
            xy_dual(g, s, l, lx, ly);
            xy_dual(g, s, m, mxx, myy);
            xy_dual(g, s, r, rx, ry);
            const Dual ds1 = sqrt((mxx - lx) * (mxx - lx) + (myy - ly) * (myy - ly));
            const Dual ds2 = sqrt((rx - mxx) * (rx - mxx) + (ry - myy) * (ry - myy));
            const Dual ds = Dual(0.5) * (ds1 + ds2);
            const Dual nx(g.nrm[m].x, s.nrm_t[m].x), ny(g.nrm[m].y, s.nrm_t[m].y);
            Dual cp = Dual(s.pv[cur][m].d, s.pt[cur][m].d) - Dual(pr_inf);
            cp = -cp / temp;
            H = H + cp * nx * ds;
            V = V + cp * ny * ds;
        }
        const Dual cl = V * Dual(cos_t) - H * Dual(sin_t);
        const Dual cd = H * Dual(cos_t) + V * Dual(sin_t);
        J = J + (objective == 1 ? cd : cl);
    }
    out[0] = J.v;
    out[1] = J.d;
}

// Per-point terms of the secondary objectives (compute_entropy.F90:21-27,
// compute_enstrophy.F90:27-79, stagnation_values.F90:60-67), as Duals.
__global__ void k_t_obj_terms(Geom g, TanState s, int cur, int kind, double gamma_power,
                              double p0_inf, double *__restrict__ tv, double *__restrict__ td) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.n) return;
    const Dual gamma(1.4), pr_inf(1.0 / 1.4);
    Dual P[4];
    ld_dual4(s.pv[cur], s.pt[cur], i, P);
    Dual t;
    if (kind == MFCFD_OBJ_ENTROPY) {
        // rho**gamma = exp(gamma log rho)
        Dual temp1 = exp(gamma * log(P[0]));
        temp1 = P[3] / temp1;
        temp1 = log(temp1);
        t = fabs(temp1 - log(pr_inf));
    } else if (kind == MFCFD_OBJ_STAGNATION) {
        const Dual m2 = (P[1] * P[1] + P[2] * P[2]) / (gamma * P[3] / P[0]);
        const Dual A = Dual(1.0) + Dual((1.4 - 1) / 2) * m2;
        const Dual d = Dual(p0_inf) - P[3] * exp(Dual(gamma_power) * log(A));
        t = d * d;
    } else {
        Dual xi, yi;
        xy_dual(g, s, i, xi, yi);
        Dual sxx, syy, sxy, sxu1, sxu2, syu1, syu2;
        const int nb = g.nbhs[i];
        for (int r = 0; r < nb; ++r) {
            const int k = g.conn[r * g.n + i];
            Dual xk, yk, Q[4];
            xy_dual(g, s, k, xk, yk);
            ld_dual4(s.pv[cur], s.pt[cur], k, Q);
            const Dual delx = xk - xi, dely = yk - yi;
            sxx = sxx + delx * delx;
            syy = syy + dely * dely;
            sxy = sxy + delx * dely;
            sxu1 = sxu1 + delx * (Q[1] - P[1]);
            sxu2 = sxu2 + delx * (Q[2] - P[2]);
            syu1 = syu1 + dely * (Q[1] - P[1]);
            syu2 = syu2 + dely * (Q[2] - P[2]);
        }
        const Dual one_by_det = Dual(1.0) / (sxx * syy - sxy * sxy);
        const Dual w = (sxu2 * syy - syu2 * sxy) * one_by_det - (syu1 * sxx - sxu1 * sxy) * one_by_det;
        t = w * w;
    }
    tv[i] = t.v;
    td[i] = t.d;
}

inline int nblk(int n, int b) { return (n + b - 1) / b; }

}  // namespace

extern "C" int mfcfd_tangent(mfcfd_t *h, int objective, int n_iters, const double *dx,
                             const double *dy, double *J, double *dJ) {
    if (!h) return MFCFD_ERR_ARG;
    if (objective < MFCFD_OBJ_CL || objective > MFCFD_OBJ_STAGNATION)
        return fail(h, MFCFD_ERR_ARG, "objective must be 0..4");
    if (n_iters < 0) return fail(h, MFCFD_ERR_ARG, "n_iters < 0");
    if (h->fp32 || h->p.power != 0.0)
        return fail(h, MFCFD_ERR_ARG, "mfcfd_tangent needs an FP64 handle with power = 0");
    const int n = h->n, nw = h->nw, no = h->no, m = h->p.inner_iterations, rks = h->p.rks;
    CK(cudaStreamSynchronize(h->stream));
    std::vector<int> inv(n);
    for (int p = 0; p < n; ++p) inv[h->perm[p]] = p;
    // seed and geometry derivatives (point_normals_d.F90 on the host)
    std::vector<double2> hxy(n), hnrm(n), xy_t(n), nrm_t(n, make_double2(0.0, 0.0));
    CK(cudaMemcpy(hxy.data(), h->d_xy, n * sizeof(double2), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(hnrm.data(), h->d_nrm, n * sizeof(double2), cudaMemcpyDeviceToHost));
    for (int p = 0; p < n; ++p)
        xy_t[p] = make_double2(dx ? dx[h->perm[p]] : 0.0, dy ? dy[h->perm[p]] : 0.0);
    auto X = [&](int p) { return Dual(hxy[p].x, xy_t[p].x); };
    auto Y = [&](int p) { return Dual(hxy[p].y, xy_t[p].y); };
    std::vector<Dual> obc((size_t)8 * std::max(no, 1));
    const double pi = h->pi;
    for (int p = 0; p < nw + no; ++p) {
        const int l = inv[h->left0[h->perm[p]] - 1], r = inv[h->right0[h->perm[p]] - 1];
        const Dual nx1 = Y(p) - Y(l), nx2 = Y(r) - Y(p), ny1 = X(p) - X(l), ny2 = X(r) - X(p);
        const Dual vx = Dual(0.5) * (nx1 + nx2), vy = Dual(0.5) * (ny1 + ny2);
        const Dual det = sqrt(vx * vx + vy * vy);
        const Dual nx = -vx / det, ny = vy / det;
        nrm_t[p] = make_double2(nx.d, ny.d);
        if (p >= nw) {
            // state_update.F90:248-263, the freestream half of Ubar
            const double pr_inf = 1.0 / 1.4, rho_inf = 1.0, gamma = 1.4;
            const Dual u1_inf(h->q_inf[1]), u2_inf(h->q_inf[2]);
            const Dual tx = Dual(hnrm[p].y, nrm_t[p].y), ty = -Dual(hnrm[p].x, nrm_t[p].x);
            const Dual nxd(hnrm[p].x, nrm_t[p].x), nyd(hnrm[p].y, nrm_t[p].y);
            const Dual u1r = u1_inf * tx + u2_inf * ty;
            const Dual u2r = u1_inf * nxd + u2_inf * nyd;
            const Dual temp1 = (u1r * u1r + u2r * u2r);
            const Dual e_inf = Dual(pr_inf / (rho_inf * (gamma - 1.0))) + Dual(0.5) * temp1;
            const double beta = (0.5 * rho_inf) / pr_inf;
            const Dual S2 = u2r * Dual(::sqrt(beta));
            const Dual B2_inf = exp(-S2 * S2) / Dual(2.0 * ::sqrt(pi * beta));
            const Dual A2n_inf = Dual(0.5) * (Dual(1.0) - erf(S2));
            Dual *o = &obc[(size_t)8 * (p - nw)];
            o[0] = u1r;
            o[1] = u2r;
            o[2] = e_inf;
            o[3] = A2n_inf;
            o[4] = B2_inf;
        }
    }
    // shape points in grid order
    std::vector<int> si, sl, sr, ss;
    for (int i = 0; i < n; ++i) {
        if (h->flag2_0[i] <= 0) continue;
        si.push_back(inv[i]);
        sl.push_back(inv[h->left0[i] - 1]);
        sr.push_back(inv[h->right0[i] - 1]);
        ss.push_back(h->flag2_0[i] - 1);
    }
    const size_t ns = std::max<size_t>(si.size(), 1);

    // device buffers (freed on return)
    std::vector<void *> owned;
    auto take = [&](auto **p, size_t cnt) -> cudaError_t {
        cudaError_t e = dmalloc(p, cnt);
        if (e == cudaSuccess) owned.push_back(*p);
        return e;
    };
    int st = MFCFD_OK;
    TanState s{};
    double2 *d_xyt = nullptr, *d_nrmt = nullptr;
    Dual *d_obc = nullptr;
    int *d_si = nullptr, *d_sl = nullptr, *d_sr = nullptr, *d_ss = nullptr;
    double *d_out = nullptr;
    cudaError_t e = take(&d_xyt, n);
    if (e == cudaSuccess) e = take(&d_nrmt, n);
    if (e == cudaSuccess) e = take(&d_obc, obc.size());
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
        e = take(&s.pv[b], n);
        if (e == cudaSuccess) e = take(&s.pt[b], n);
        if (e == cudaSuccess) e = take(&s.qv[b], n);
        if (e == cudaSuccess) e = take(&s.qt[b], n);
        if (e == cudaSuccess) e = take(&s.dqv[b], (size_t)8 * n);
        if (e == cudaSuccess) e = take(&s.dqt[b], (size_t)8 * n);
    }
    if (e == cudaSuccess) e = take(&s.qmv, (size_t)8 * n);
    if (e == cudaSuccess) e = take(&s.qmt, (size_t)8 * n);
    if (e == cudaSuccess) e = take(&s.dlv, n);
    if (e == cudaSuccess) e = take(&s.dlt, n);
    if (e == cudaSuccess) e = take(&s.spv, n);
    if (e == cudaSuccess) e = take(&s.spt, n);
    if (e == cudaSuccess) e = take(&d_si, ns);
    if (e == cudaSuccess) e = take(&d_sl, ns);
    if (e == cudaSuccess) e = take(&d_sr, ns);
    if (e == cudaSuccess) e = take(&d_ss, ns);
    if (e == cudaSuccess) e = take(&d_out, 2);
    if (e != cudaSuccess) st = cuda_fail(h, e, "mfcfd_tangent cudaMalloc");
    auto up = [&](void *d, const void *src, size_t bytes) {
        if (st == MFCFD_OK && bytes) {
            cudaError_t u = cudaMemcpy(d, src, bytes, cudaMemcpyHostToDevice);
            if (u != cudaSuccess) st = cuda_fail(h, u, "mfcfd_tangent cudaMemcpy");
        }
    };
    up(d_xyt, xy_t.data(), n * sizeof(double2));
    up(d_nrmt, nrm_t.data(), n * sizeof(double2));
    up(d_obc, obc.data(), obc.size() * sizeof(Dual));
    up(d_si, si.data(), si.size() * sizeof(int));
    up(d_sl, sl.data(), sl.size() * sizeof(int));
    up(d_sr, sr.data(), sr.size() * sizeof(int));
    up(d_ss, ss.data(), ss.size() * sizeof(int));
    if (st == MFCFD_OK) {
        s.xy_t = d_xyt;
        s.nrm_t = d_nrmt;
        s.obc = d_obc;
        cudaStream_t str = h->stream;
        // the handle's state (held fixed: derivative 0)
        cudaError_t c1 = cudaMemcpyAsync(s.pv[0], h->d_prim[h->cur], sizeof(R4) * n,
                                         cudaMemcpyDeviceToDevice, str);
        if (c1 == cudaSuccess) c1 = cudaMemsetAsync(s.pt[0], 0, sizeof(R4) * n, str);
        if (c1 != cudaSuccess) st = cuda_fail(h, c1, "mfcfd_tangent state copy");
        int cur = 0, qc = 0;
        if (st == MFCFD_OK) k_t_init<<<nblk(n, 256), 256, 0, str>>>(n, s, cur, qc);
        for (int it = 0; it < n_iters && st == MFCFD_OK; ++it) {
            const int A = cur, B = cur ^ 1;
            for (int rk = 1; rk <= rks; ++rk) {
                k_t_grad<<<nblk(n, TB), TB, 0, str>>>(h->geom, h->consts, s, qc, rk == 1 ? 1 : 0);
                for (int t = 1; t <= m; ++t)
                    k_t_inner<<<nblk(n, TB), TB, 0, str>>>(h->geom, s, qc, (t - 1) & 1);
                k_t_flux<<<nblk(n, TB), TB, 0, str>>>(h->geom, h->consts, s, A, B, qc, m & 1, rk,
                                                     rk == rks ? 1 : 0);
                qc ^= 1;
                h->launches += 2 + m;
            }
            cur = B;
            cudaError_t le = cudaGetLastError();
            if (le != cudaSuccess) st = cuda_fail(h, le, "mfcfd_tangent launch");
        }
        if (st == MFCFD_OK && objective >= MFCFD_OBJ_ENTROPY) {
            // secondary objectives: per-point Dual terms, summed in caller order
            double *d_tv = nullptr, *d_td = nullptr;
            cudaError_t c2 = take(&d_tv, n);
            if (c2 == cudaSuccess) c2 = take(&d_td, n);
            const double gp = lskum_host::stagnation_gamma_power();
            const double p0_inf = lskum_host::stagnation_p0_inf(h->p.mach);
            if (c2 == cudaSuccess) {
                k_t_obj_terms<<<nblk(n, 256), 256, 0, str>>>(h->geom, s, cur, objective, gp, p0_inf,
                                                             d_tv, d_td);
                h->launches += 1;
                c2 = cudaGetLastError();
            }
            std::vector<double> tv(n), td(n);
            if (c2 == cudaSuccess)
                c2 = cudaMemcpyAsync(tv.data(), d_tv, sizeof(double) * n, cudaMemcpyDeviceToHost, str);
            if (c2 == cudaSuccess)
                c2 = cudaMemcpyAsync(td.data(), d_td, sizeof(double) * n, cudaMemcpyDeviceToHost, str);
            if (c2 == cudaSuccess) c2 = cudaStreamSynchronize(str);
            if (c2 != cudaSuccess) {
                st = cuda_fail(h, c2, "mfcfd_tangent objective");
            } else {
                Dual sum;
                for (int k = 0; k < n; ++k) sum = sum + Dual(tv[inv[k]], td[inv[k]]);
                if (objective == MFCFD_OBJ_STAGNATION) sum = sum * Dual(1 / (p0_inf * p0_inf * n));
                if (J) *J = sum.v;
                if (dJ) *dJ = sum.d;
            }
        } else if (st == MFCFD_OK) {
            TanShape ts{(int)si.size(), h->shapes, d_si, d_sl, d_sr, d_ss};
            k_t_forces<<<1, 32, 0, str>>>(h->geom, s, ts, cur, h->p.mach, h->cos_t, h->sin_t,
                                          objective, d_out);
            h->launches += 2;
            double o[2] = {0.0, 0.0};
            cudaError_t c2 = cudaMemcpyAsync(o, d_out, sizeof(o), cudaMemcpyDeviceToHost, str);
            if (c2 == cudaSuccess) c2 = cudaStreamSynchronize(str);
            if (c2 != cudaSuccess) st = cuda_fail(h, c2, "mfcfd_tangent result");
            if (J) *J = o[0];
            if (dJ) *dJ = o[1];
        }
    }
    cudaStreamSynchronize(h->stream);
    for (void *p : owned) cudaFree(p);
    return st;
}
