// Device-side building blocks of the LSKUM pseudo-time loop (FP64).
//
// Every function restates one reference routine of src_mpi_primal with the
// same expression association as the Fortran source (which evaluates
// a*b*c as (a*b)*c and a+b+c as (a+b)+c).  The split-flux routines are
// written once with sign arguments: a - b == a + (-1)*b exactly in IEEE
// arithmetic, so Gxp/Gxn (and GxI..GxIV) share one body.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace lskum {

enum PointKind { KIND_WALL = 0, KIND_INTERIOR = 1, KIND_OUTER = 2 };

// Limiter threshold: the literal 10e-6 in limiters.F90:78,81 is a
// default-real (single precision) constant promoted to double.
#define MFCFD_VENKAT_THR 9.99999974737875163555145263671875e-06

struct __align__(32) R4 {
    double a, b, c, d;
};

__device__ __forceinline__ R4 ld4(const R4 *p) {
    const double2 *q = reinterpret_cast<const double2 *>(p);
    double2 u = __ldg(q), v = __ldg(q + 1);
    return R4{u.x, u.y, v.x, v.y};
}
__device__ __forceinline__ void st4(R4 *p, double a, double b, double c, double d) {
    double2 *q = reinterpret_cast<double2 *>(p);
    q[0] = make_double2(a, b);
    q[1] = make_double2(c, d);
}

// Constant, renumbered geometry.  Wall points occupy [0, nw), outer points
// [nw, nw + no), interior points [nw + no, n).
struct Geom {
    int n, kp, nw, no;
    const double2 *xy;             // (x, y)
    const double2 *nrm;            // (nx, ny) as the reference sets them
    const double *eps2;            // (vl_const*min_dist)**3 squared
    const int *conn;               // [kp][n], 0-based renumbered indices
    const int *nbhs;               // [n]
    const unsigned long long *mx;  // bit r: slot r in xpos; bit 32+r: in xneg
    const unsigned long long *my;  // bit r: slot r in ypos; bit 32+r: in yneg
    const double *obc;             // outer points: u1_inf_rot, u2_inf_rot, e_inf, A2n_inf, B2_inf, 0,0,0
    // Tile halos of the D and I passes (nullptr: no halo, every row is
    // gathered directly).  The halo of a TILE-point tile is the sorted set of
    // rows its points read (the points themselves and their neighbours);
    // hoff[tile] .. hoff[tile + 1] index its rows in hrow (an empty range: the
    // tile's halo exceeds HALO_CAP and its rows are gathered directly).
    // hloc[p * hkp + r] is slot r's row within the tile's halo, hloc[p * hkp
    // + hkp - 1] the point's own; hc = the largest halo, the staging stride.
    const int *hoff = nullptr;
    const int *hrow = nullptr;
    const unsigned char *hloc = nullptr;
    int hkp = 0, hc = 0;
};
// rows a tile halo stages at most (its local row indices are bytes)
constexpr int HALO_CAP = 64;

struct Consts {
    double cfl, power, euler, pi, gm1;  // gm1 = gamma - 1
    int power_zero;                     // power == 0: weights are exactly 1
    int rks;
};

// ---------------------------------------------------------------------------
// q_variables.F90:8-37 eval_q_variables
template <class T>
__device__ __forceinline__ void q_from_prim_t(T rho, T u1, T u2, T pr, T q[4]) {
    T beta = T(0.5) * rho / pr;
    q[0] = (log(rho) + (log(beta) * T(2.5))) - beta * (u1 * u1 + u2 * u2);
    T two_times_beta = T(2.0) * beta;
    q[1] = two_times_beta * u1;
    q[2] = two_times_beta * u2;
    q[3] = -two_times_beta;
}
__device__ __forceinline__ void q_from_prim(double rho, double u1, double u2, double pr,
                                            double q[4]) {
    q_from_prim_t<double>(rho, u1, u2, pr, q);
}

// q_variables.F90:230-256 qtilde_to_primitive.  T is double on the FP64
// path and float on the FP32-mixed path; the literals keep their values.
template <class T>
__device__ __forceinline__ void qtilde_to_primitive(const T qt[4], T gm1, T &u1, T &u2, T &rho,
                                                    T &pr) {
    T beta = -qt[3] * T(0.5);
    T temp = T(0.5) / beta;
    u1 = qt[1] * temp;
    u2 = qt[2] * temp;
    T temp1 = qt[0] + beta * (u1 * u1 + u2 * u2);
    T temp2 = temp1 - (log(beta) / gm1);
    rho = exp(temp2);
    pr = rho * temp;
}

// limiters.F90:64-110 venkat_limiter, one component.
template <class T>
__device__ __forceinline__ T venkat_phi(T qtilde, T q, T qmax, T qmin, T eps2) {
    T del_neg = qtilde - q;
    if (fabs(del_neg) <= T(MFCFD_VENKAT_THR)) return T(1.0);
    T del_pos = del_neg > T(0.0) ? qmax - q : qmin - q;
    T num = (del_pos * del_pos) + eps2;
    num = num * del_neg + T(2.0) * del_neg * del_neg * del_pos;
    T den = del_pos * del_pos + T(2.0) * del_neg * del_neg;
    den = den + del_neg * del_pos + eps2;
    den = den * del_neg;
    T temp = num / den;
    return temp < T(1.0) ? temp : T(1.0);
}

// Limited reconstruction of one point towards one neighbour direction,
// straight to primitive variables (the qtilde lines of *_fluxes.F90, e.g.
// interior_fluxes.F90:158-172).  t = delx*dq(1,:) + dely*dq(2,:) is formed
// once and used for both the unlimited and the limited qtilde, exactly as the
// reference recomputes it.
template <class T>
__device__ __forceinline__ void reconstruct(const T q[4], const T dqx[4], const T dqy[4],
                                            const T qmax[4], const T qmin[4], T eps2, T delx,
                                            T dely, T gm1, T &u1, T &u2, T &rho, T &pr) {
    T qt[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        T t = delx * dqx[r] + dely * dqy[r];
        T phi = venkat_phi<T>(q[r] - T(0.5) * t, q[r], qmax[r], qmin[r], eps2);
        qt[r] = q[r] - T(0.5) * phi * t;
    }
    qtilde_to_primitive<T>(qt, gm1, u1, u2, rho, pr);
}

// The per-state part shared by split_fluxes.F90 and quadrant_fluxes.F90: the
// state in the point's (t, n) frame and the two Maxwellian half-moments.
template <class T>
struct KStateT {
    T rho, ut, un, pbr, usq, B1, B2, e1, e2;
};
using KState = KStateT<double>;

template <class T>
__device__ __forceinline__ KStateT<T> kstate(T u1, T u2, T rho, T pr, T nx, T ny, T pi) {
    KStateT<T> s;
    T tx = ny, ty = -nx;
    s.ut = u1 * tx + u2 * ty;
    s.un = u1 * nx + u2 * ny;
    T beta = T(0.5) * rho / pr;
    T sb = sqrt(beta);
    T S1 = s.ut * sb;
    T S2 = s.un * sb;
    T spb = sqrt(pi * beta);
    s.B1 = T(0.5) * exp(-S1 * S1) / spb;
    s.B2 = T(0.5) * exp(-S2 * S2) / spb;
    s.e1 = erf(S1);
    s.e2 = erf(S2);
    s.pbr = pr / rho;
    s.usq = s.ut * s.ut + s.un * s.un;
    s.rho = rho;
    return s;
}

// erf(x) given exp(-x*x).  FP64: the library erf.  FP32: Abramowitz &
// Stegun 7.1.26 (after Hastings), erf(|x|) = 1 - t (a1 + t (a2 + t (a3 + t
// (a4 + t a5)))) exp(-x^2), t = 1 / (1 + p |x|), absolute error below
// 1.5e-7 (5.3e-7 evaluated in FP32; tests/test_erf32.py) -- the split
// fluxes use erf only in 1 +- erf, so the absolute error is what counts --
// reusing the exponential the Maxwellian moments take anyway (C2: FP32 flux pass 0.316 -> 0.304 ms; |dCl| against the FP64
// loop after 50 iterations 1.0e-7 with the library erff, 6e-9 with this).
template <class T>
__device__ __forceinline__ T erf_with_exp(T x, T) {
    return erf(x);
}
template <>
__device__ __forceinline__ float erf_with_exp<float>(float x, float e) {
    const float ax = fabsf(x);
    const float t = 1.0f / (1.0f + 0.3275911f * ax);
    float p = 1.061405429f;
    p = p * t - 1.453152027f;
    p = p * t + 1.421413741f;
    p = p * t - 0.284496736f;
    p = p * t + 0.254829592f;
    return copysignf(1.0f - (p * t) * e, x);
}

// reconstruct + kstate in one, for the flux passes: the kinetic state of the
// limited reconstruction towards one neighbour.  beta and p/rho come from
// qtilde itself (beta = -qtilde_4/2, p/rho = 1/(2 beta)), which the
// reference's 0.5 rho/p and p/rho of the same state equal in exact
// arithmetic; 0.5/sqrt(pi beta) is formed as (p/rho) sqrt(beta) / sqrt(pi)
// and beta**(-1/(gamma-1)) without a log (below).  Five divisions and one
// reciprocal square root per state instead of ten divisions, two square
// roots and a log; the results differ from reconstruct + kstate by rounding
// only.
template <class T>
__device__ __forceinline__ KStateT<T> reconstruct_kstate(const T q[4], const T dqx[4],
                                                         const T dqy[4], const T qmax[4],
                                                         const T qmin[4], T eps2, T delx, T dely,
                                                         T inv_gm1, T nx, T ny, T inv_sqrt_pi,
                                                         T *u_out = nullptr) {
    T qt[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        T t = delx * dqx[r] + dely * dqy[r];
        T phi = venkat_phi<T>(q[r] - T(0.5) * t, q[r], qmax[r], qmin[r], eps2);
        qt[r] = q[r] - T(0.5) * phi * t;
    }
    const T beta = -qt[3] * T(0.5);
    const T temp = T(0.5) / beta;  // p / rho
    const T u1 = qt[1] * temp, u2 = qt[2] * temp;
    if (u_out) {  // the adjoint's tape keeps the reconstructed velocity
        u_out[0] = u1;
        u_out[1] = u2;
    }
    const T temp1 = qt[0] + beta * (u1 * u1 + u2 * u2);
    KStateT<T> s;
    // rho = exp(temp1 - log(beta)/(gamma-1)) with gamma = 1.4, a constant of
    // the reference (parameter.F90:10): beta**(-1/(gamma-1)) = beta**(-2.5)
    // = (1/beta)**2 / sqrt(beta), 1/beta = 2 p/rho -- no log, and sqrt(beta)
    // from the same reciprocal square root (C2: 0.705 -> 0.649 ms a flux
    // pass).  inv_gm1 is kept in the signature for the callers.
    const T rb = rsqrt(beta);
    const T sb = beta * rb;
    s.rho = exp(temp1) * ((T(4.0) * temp * temp) * rb);
    (void)inv_gm1;
    const T tx = ny, ty = -nx;
    s.ut = u1 * tx + u2 * ty;
    s.un = u1 * nx + u2 * ny;
    const T S1 = s.ut * sb, S2 = s.un * sb;
    const T h = temp * sb * inv_sqrt_pi;  // 0.5 / sqrt(pi beta)
    const T E1 = exp(-S1 * S1), E2 = exp(-S2 * S2);
    s.B1 = E1 * h;
    s.B2 = E2 * h;
    s.e1 = erf_with_exp(S1, E1);
    s.e2 = erf_with_exp(S2, E2);
    s.pbr = temp;
    s.usq = s.ut * s.ut + s.un * s.un;
    return s;
}

// split_fluxes.F90:8-96 flux_Gxp (s1 = +1) / flux_Gxn (s1 = -1)
template <class T>
__device__ __forceinline__ void flux_gx(const KStateT<T> &s, T s1, T G[4]) {
    T A1 = T(0.5) * (T(1.0) + s1 * s.e1);
    G[0] = s.rho * (s.ut * A1 + s1 * s.B1);
    T temp1 = s.pbr + s.ut * s.ut;
    T temp2 = temp1 * A1 + s1 * (s.ut * s.B1);
    G[1] = s.rho * temp2;
    temp1 = s.ut * s.un * A1 + s1 * (s.un * s.B1);
    G[2] = s.rho * temp1;
    temp1 = (T(7.0) * s.pbr) + s.usq;
    temp2 = T(0.5) * s.ut * temp1 * A1;
    temp1 = (T(6.0) * s.pbr) + s.usq;
    G[3] = s.rho * (temp2 + s1 * (T(0.5) * temp1 * s.B1));
}

// split_fluxes.F90:99-190 flux_Gyp (s2 = +1) / flux_Gyn (s2 = -1)
template <class T>
__device__ __forceinline__ void flux_gy(const KStateT<T> &s, T s2, T G[4]) {
    T A2 = T(0.5) * (T(1.0) + s2 * s.e2);
    G[0] = s.rho * (s.un * A2 + s2 * s.B2);
    T temp1 = s.pbr + s.un * s.un;
    T temp2 = temp1 * A2 + s2 * (s.un * s.B2);
    G[2] = s.rho * temp2;
    temp1 = s.ut * s.un * A2 + s2 * (s.ut * s.B2);
    G[1] = s.rho * temp1;
    temp1 = (T(7.0) * s.pbr) + s.usq;
    temp2 = T(0.5) * s.un * temp1 * A2;
    temp1 = (T(6.0) * s.pbr) + s.usq;
    G[3] = s.rho * (temp2 + s2 * (T(0.5) * temp1 * s.B2));
}

// quadrant_fluxes.F90:12-248: GxI (s1=-1,s2=-1), GxII (+1,-1), GxIII (+1,+1),
// GxIV (-1,+1).
template <class T>
__device__ __forceinline__ void flux_quad(const KStateT<T> &s, T s1, T s2, T G[4]) {
    T A1 = T(0.5) * (T(1.0) + s1 * s.e1);
    T A2 = T(0.5) * (T(1.0) + s2 * s.e2);
    T rA2 = s.rho * A2;
    T a1b = s.ut * A1 + s1 * s.B1;
    G[0] = rA2 * a1b;
    T temp1 = s.pbr + s.ut * s.ut;
    T temp2 = temp1 * A1 + s1 * (s.ut * s.B1);
    G[1] = rA2 * temp2;
    temp2 = s.un * A2 + s2 * s.B2;
    G[2] = s.rho * a1b * temp2;
    temp1 = (T(7.0) * s.pbr) + s.usq;
    temp2 = T(0.5) * s.ut * temp1 * A1;
    temp1 = (T(6.0) * s.pbr) + s.usq;
    T temp3 = T(0.5) * s.B1 * temp1;
    T temp4 = T(0.5) * s.rho * s.un * s.B2 * a1b;
    G[3] = rA2 * (temp2 + s1 * temp3) + s2 * temp4;
}

// state_update.F90:144-163 primitive_to_conserved
template <class T>
__device__ __forceinline__ void prim_to_conserved_t(T rho, T u1, T u2, T pr, T nx, T ny, T U[4]) {
    U[0] = rho;
    T temp1 = rho * u1;
    T temp2 = rho * u2;
    U[3] = T(2.5) * pr + T(0.5) * (temp1 * temp1 + temp2 * temp2) / rho;
    U[1] = temp1 * ny - temp2 * nx;
    U[2] = temp1 * nx + temp2 * ny;
}
__device__ __forceinline__ void prim_to_conserved(double rho, double u1, double u2, double pr,
                                                  double nx, double ny, double U[4]) {
    prim_to_conserved_t<double>(rho, u1, u2, pr, nx, ny, U);
}

// state_update.F90:239-294 conserved_vector_Ubar.  The freestream half
// (inf[0..4] = u1_inf_rot, u2_inf_rot, e_inf, A2n_inf, B2_inf) depends only on
// the geometry and is computed once on the host.
template <class T>
__device__ __forceinline__ void conserved_ubar_t(T rho, T u1, T u2, T pr, T nx, T ny,
                                                 const T *inf, T pi, T gm1, T Ubar[4]) {
    const T rho_inf = T(1.0);
    T u1_inf_rot = inf[0], u2_inf_rot = inf[1], e_inf = inf[2], A2n_inf = inf[3],
      B2_inf = inf[4];
    T tx = ny, ty = -nx;
    T u1_rot = u1 * tx + u2 * ty;
    T u2_rot = u1 * nx + u2 * ny;
    T temp1 = (u1_rot * u1_rot + u2_rot * u2_rot);
    T e = pr / (rho * gm1) + T(0.5) * (temp1);
    T beta = (rho) / (T(2.0) * pr);
    T S2 = u2_rot * sqrt(beta);
    T B2 = exp(-S2 * S2) / (T(2.0) * sqrt(pi * beta));
    T A2p = T(0.5) * (T(1.0) + erf(S2));
    Ubar[0] = (rho_inf * A2n_inf) + (rho * A2p);
    Ubar[1] = (rho_inf * u1_inf_rot * A2n_inf) + (rho * u1_rot * A2p);
    temp1 = rho_inf * (u2_inf_rot * A2n_inf - B2_inf);
    T temp2 = rho * (u2_rot * A2p + B2);
    Ubar[2] = temp1 + temp2;
    temp1 = (rho_inf * A2n_inf * e_inf - T(0.5) * rho_inf * u2_inf_rot * B2_inf);
    temp2 = (rho * A2p * e + T(0.5) * rho * u2_rot * B2);
    Ubar[3] = temp1 + temp2;
}
__device__ __forceinline__ void conserved_ubar(double rho, double u1, double u2, double pr,
                                               double nx, double ny, const double *inf,
                                               double pi, double gm1, double Ubar[4]) {
    conserved_ubar_t<double>(rho, u1, u2, pr, nx, ny, inf, pi, gm1, Ubar);
}

}  // namespace lskum
