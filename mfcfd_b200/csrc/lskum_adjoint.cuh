// Reverse-mode (adjoint) building blocks of the LSKUM pseudo-time loop, FP64.
//
// Each function is the hand-written reverse of the forward function of the
// same name in lskum_device.cuh: given the adjoint of the forward outputs
// (suffix _b) it accumulates the adjoints of the inputs.  Branches (limiter
// thresholds, split-list membership, max/min selection) are held at the
// forward outcome, as the reference's Tapenade-generated code does
// (e.g. src_mpi_adjoint/sensitivity_files/limiters_b.F90:43-165).
#pragma once

#include "lskum_device.cuh"

namespace lskum {

#define MFCFD_TWO_OVER_SQRT_PI 1.12837916709551257390

struct KStateB {
    double rho, ut, un, pbr, usq, B1, B2, e1, e2;
};

__device__ __forceinline__ void kzero(KStateB &b) {
    b.rho = b.ut = b.un = b.pbr = b.usq = b.B1 = b.B2 = b.e1 = b.e2 = 0.0;
}

// split_fluxes_b: flux_Gxp / flux_Gxn (s1 = +-1)
__device__ __forceinline__ void flux_gx_b(const KState &s, double s1, const double Gb[4],
                                          KStateB &b) {
    const double A1 = 0.5 * (1.0 + s1 * s.e1);
    double A1b = 0.0;
    const double t1 = s.pbr + s.ut * s.ut;
    const double t2 = t1 * A1 + s1 * (s.ut * s.B1);
    const double t3 = s.ut * s.un * A1 + s1 * (s.un * s.B1);
    const double t7 = (7.0 * s.pbr) + s.usq;
    const double t4 = 0.5 * s.ut * t7 * A1;
    const double t6 = (6.0 * s.pbr) + s.usq;
    b.rho += Gb[0] * (s.ut * A1 + s1 * s.B1) + Gb[1] * t2 + Gb[2] * t3 +
             Gb[3] * (t4 + s1 * (0.5 * t6 * s.B1));
    const double a0 = s.rho * Gb[0];
    b.ut += a0 * A1;
    A1b += a0 * s.ut;
    b.B1 += a0 * s1;
    const double a1 = s.rho * Gb[1];
    const double t1b = a1 * A1;
    A1b += a1 * t1;
    b.ut += a1 * s1 * s.B1 + 2.0 * s.ut * t1b;
    b.B1 += a1 * s1 * s.ut;
    b.pbr += t1b;
    const double a2 = s.rho * Gb[2];
    b.ut += a2 * s.un * A1;
    b.un += a2 * (s.ut * A1 + s1 * s.B1);
    A1b += a2 * s.ut * s.un;
    b.B1 += a2 * s1 * s.un;
    const double a3 = s.rho * Gb[3];
    const double t7b = a3 * 0.5 * s.ut * A1;
    const double t6b = a3 * s1 * 0.5 * s.B1;
    b.ut += a3 * 0.5 * t7 * A1;
    A1b += a3 * 0.5 * s.ut * t7;
    b.B1 += a3 * s1 * 0.5 * t6;
    b.pbr += 7.0 * t7b + 6.0 * t6b;
    b.usq += t7b + t6b;
    b.e1 += 0.5 * s1 * A1b;
}

// split_fluxes_b: flux_Gyp / flux_Gyn (s2 = +-1)
__device__ __forceinline__ void flux_gy_b(const KState &s, double s2, const double Gb[4],
                                          KStateB &b) {
    const double A2 = 0.5 * (1.0 + s2 * s.e2);
    double A2b = 0.0;
    const double t1 = s.pbr + s.un * s.un;
    const double t2 = t1 * A2 + s2 * (s.un * s.B2);
    const double t3 = s.ut * s.un * A2 + s2 * (s.ut * s.B2);
    const double t7 = (7.0 * s.pbr) + s.usq;
    const double t4 = 0.5 * s.un * t7 * A2;
    const double t6 = (6.0 * s.pbr) + s.usq;
    b.rho += Gb[0] * (s.un * A2 + s2 * s.B2) + Gb[2] * t2 + Gb[1] * t3 +
             Gb[3] * (t4 + s2 * (0.5 * t6 * s.B2));
    const double a0 = s.rho * Gb[0];
    b.un += a0 * A2;
    A2b += a0 * s.un;
    b.B2 += a0 * s2;
    const double a2 = s.rho * Gb[2];
    const double t1b = a2 * A2;
    A2b += a2 * t1;
    b.un += a2 * s2 * s.B2 + 2.0 * s.un * t1b;
    b.B2 += a2 * s2 * s.un;
    b.pbr += t1b;
    const double a1 = s.rho * Gb[1];
    b.un += a1 * s.ut * A2;
    b.ut += a1 * (s.un * A2 + s2 * s.B2);
    A2b += a1 * s.ut * s.un;
    b.B2 += a1 * s2 * s.ut;
    const double a3 = s.rho * Gb[3];
    const double t7b = a3 * 0.5 * s.un * A2;
    const double t6b = a3 * s2 * 0.5 * s.B2;
    b.un += a3 * 0.5 * t7 * A2;
    A2b += a3 * 0.5 * s.un * t7;
    b.B2 += a3 * s2 * 0.5 * t6;
    b.pbr += 7.0 * t7b + 6.0 * t6b;
    b.usq += t7b + t6b;
    b.e2 += 0.5 * s2 * A2b;
}

// quadrant_fluxes_b: GxI..GxIV
__device__ __forceinline__ void flux_quad_b(const KState &s, double s1, double s2,
                                            const double Gb[4], KStateB &b) {
    const double A1 = 0.5 * (1.0 + s1 * s.e1);
    const double A2 = 0.5 * (1.0 + s2 * s.e2);
    const double rA2 = s.rho * A2;
    const double a1b = s.ut * A1 + s1 * s.B1;
    const double t1 = s.pbr + s.ut * s.ut;
    const double t2 = t1 * A1 + s1 * (s.ut * s.B1);
    const double c2 = s.un * A2 + s2 * s.B2;
    const double t7 = (7.0 * s.pbr) + s.usq;
    const double t4 = 0.5 * s.ut * t7 * A1;
    const double t6 = (6.0 * s.pbr) + s.usq;
    const double t3 = 0.5 * s.B1 * t6;
    double A1b = 0.0, A2b = 0.0;
    const double rA2b = Gb[0] * a1b + Gb[1] * t2 + Gb[3] * (t4 + s1 * t3);
    const double a1bb = Gb[0] * rA2 + Gb[2] * s.rho * c2 + s2 * Gb[3] * (0.5 * s.rho * s.un * s.B2);
    // G1 = rA2 * t2
    const double t2b = Gb[1] * rA2;
    const double t1b = t2b * A1;
    A1b += t2b * t1;
    b.ut += t2b * s1 * s.B1 + 2.0 * s.ut * t1b;
    b.B1 += t2b * s1 * s.ut;
    b.pbr += t1b;
    // G2 = rho * a1b * c2
    b.rho += Gb[2] * a1b * c2;
    const double c2b = Gb[2] * s.rho * a1b;
    b.un += c2b * A2;
    A2b += c2b * s.un;
    b.B2 += c2b * s2;
    // G3 = rA2 * (t4 + s1 t3) + s2 * 0.5 rho un B2 a1b
    const double t4b = Gb[3] * rA2;
    const double t3b = Gb[3] * rA2 * s1;
    const double t5b = Gb[3] * s2;
    b.ut += t4b * 0.5 * t7 * A1;
    const double t7b = t4b * 0.5 * s.ut * A1;
    A1b += t4b * 0.5 * s.ut * t7;
    b.B1 += t3b * 0.5 * t6;
    const double t6b = t3b * 0.5 * s.B1;
    b.rho += t5b * 0.5 * s.un * s.B2 * a1b;
    b.un += t5b * 0.5 * s.rho * s.B2 * a1b;
    b.B2 += t5b * 0.5 * s.rho * s.un * a1b;
    b.pbr += 7.0 * t7b + 6.0 * t6b;
    b.usq += t7b + t6b;
    // a1b = ut A1 + s1 B1
    b.ut += a1bb * A1;
    A1b += a1bb * s.ut;
    b.B1 += a1bb * s1;
    // rA2 = rho A2
    b.rho += rA2b * A2;
    A2b += rA2b * s.rho;
    b.e1 += 0.5 * s1 * A1b;
    b.e2 += 0.5 * s2 * A2b;
}

// kstate_b: adjoint of the kinetic state w.r.t. (u1, u2, rho, pr) and the
// point's normal (nx, ny), which sets the (t, n) frame.
__device__ __forceinline__ void kstate_b(double u1, double u2, double rho, double pr, double nx,
                                         double ny, double pi, KStateB sb_, double &u1b,
                                         double &u2b, double &rhob, double &prb, double &nxb,
                                         double &nyb) {
    const double ut = u1 * ny - u2 * nx;
    const double un = u1 * nx + u2 * ny;
    const double beta = 0.5 * rho / pr;
    const double sb = sqrt(beta);
    const double S1 = ut * sb, S2 = un * sb;
    const double spb = sqrt(pi * beta);
    const double E1 = exp(-S1 * S1), E2 = exp(-S2 * S2);
    const double B1 = 0.5 * E1 / spb, B2 = 0.5 * E2 / spb;
    double utb = sb_.ut + 2.0 * ut * sb_.usq;
    double unb = sb_.un + 2.0 * un * sb_.usq;
    prb += sb_.pbr / rho;
    rhob += sb_.rho - sb_.pbr * (pr / rho) / rho;
    const double S1b = sb_.e1 * MFCFD_TWO_OVER_SQRT_PI * E1 + sb_.B1 * B1 * (-2.0 * S1);
    const double S2b = sb_.e2 * MFCFD_TWO_OVER_SQRT_PI * E2 + sb_.B2 * B2 * (-2.0 * S2);
    const double spbb = -(sb_.B1 * B1 + sb_.B2 * B2) / spb;
    double betab = spbb * pi / (2.0 * spb);
    utb += S1b * sb;
    unb += S2b * sb;
    const double sbb = S1b * ut + S2b * un;
    betab += sbb / (2.0 * sb);
    rhob += betab * 0.5 / pr;
    prb += -betab * beta / pr;
    u1b += utb * ny + unb * nx;
    u2b += -utb * nx + unb * ny;
    nxb += -utb * u2 + unb * u1;
    nyb += utb * u1 + unb * u2;
}

// kstate_b from the forward's own kinetic state s (its rho, ut, un, p/rho,
// B1, B2): exp(-S^2) / sqrt(pi beta) = 2 B and (2/sqrt(pi)) exp(-S^2) =
// 4 B sqrt(beta), so the adjoint needs one square root and two divisions
// instead of kstate_b's two exponentials, two square roots and seven
// divisions.  (u1, u2) is the state's velocity.
__device__ __forceinline__ void kstate_b_s(const KState &s, double u1, double u2, double nx,
                                           double ny, const KStateB &sb_, double &u1b,
                                           double &u2b, double &rhob, double &prb, double &nxb,
                                           double &nyb) {
    const double ut = s.ut, un = s.un, pbr = s.pbr;
    const double beta = 0.5 / pbr;
    const double ir = 1.0 / s.rho;
    const double sb = sqrt(beta);
    const double S1 = ut * sb, S2 = un * sb;
    double utb = sb_.ut + 2.0 * ut * sb_.usq;
    double unb = sb_.un + 2.0 * un * sb_.usq;
    prb += sb_.pbr * ir;
    rhob += sb_.rho - sb_.pbr * pbr * ir;
    const double S1b = s.B1 * (4.0 * sb * sb_.e1 - 2.0 * S1 * sb_.B1);
    const double S2b = s.B2 * (4.0 * sb * sb_.e2 - 2.0 * S2 * sb_.B2);
    double betab = -(sb_.B1 * s.B1 + sb_.B2 * s.B2) * pbr;
    utb += S1b * sb;
    unb += S2b * sb;
    betab += (S1b * ut + S2b * un) * sb * pbr;  // d sqrt(beta) / d beta = sqrt(beta) p/rho
    // beta = rho / (2 pr): d/drho = beta / rho, d/dpr = -beta / pr = -2 beta^2 / rho
    rhob += betab * beta * ir;
    prb += -betab * 2.0 * beta * beta * ir;
    u1b += utb * ny + unb * nx;
    u2b += -utb * nx + unb * ny;
    nxb += -utb * u2 + unb * u1;
    nyb += utb * u1 + unb * u2;
}

// qtilde_to_primitive_b (one division: 1/beta; 1/gm1 is loop-invariant
// where this is inlined)
__device__ __forceinline__ void qtilde_to_primitive_b(const double qt[4], double gm1, double rho,
                                                      double u1b, double u2b, double rhob,
                                                      double prb, double qtb[4]) {
    const double beta = -qt[3] * 0.5;
    const double ib = 1.0 / beta;
    const double igm1 = 1.0 / gm1;
    const double temp = 0.5 * ib;
    const double u1 = qt[1] * temp, u2 = qt[2] * temp;
    rhob += prb * temp;
    double tempb = prb * rho;
    const double temp2b = rhob * rho;
    const double temp1b = temp2b;
    double betab = -temp2b * ib * igm1;
    qtb[0] += temp1b;
    betab += temp1b * (u1 * u1 + u2 * u2);
    u1b += temp1b * 2.0 * beta * u1;
    u2b += temp1b * 2.0 * beta * u2;
    qtb[1] += u1b * temp;
    qtb[2] += u2b * temp;
    tempb += u1b * qt[1] + u2b * qt[2];
    betab += -tempb * temp * ib;
    qtb[3] += -0.5 * betab;
}

// reconstruct_b: adjoint of the limited reconstruction to primitive
// variables.  The Venkatakrishnan limiter of each component (its forward
// value and venkat_limiter_b) shares one reciprocal of its denominator:
// phi = num (1/den), num_b = phi_b (1/den), den_b = -phi_b phi (1/den).
__device__ __forceinline__ void reconstruct_b(const double q[4], const double dqx[4],
                                              const double dqy[4], const double qmax[4],
                                              const double qmin[4], double eps2, double delx,
                                              double dely, double gm1, double rho, double u1b,
                                              double u2b, double rhob, double prb, double qb[4],
                                              double dqxb[4], double dqyb[4], double qmaxb[4],
                                              double qminb[4], double &delxb, double &delyb) {
    double qt[4], t[4], phi[4], idn[4];
    unsigned active = 0;  // bit r: the limiter of component r is below 1
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        t[r] = delx * dqx[r] + dely * dqy[r];
        const double dn = (q[r] - 0.5 * t[r]) - q[r];
        phi[r] = 1.0;
        idn[r] = 0.0;
        if (fabs(dn) > MFCFD_VENKAT_THR) {
            const double dp = dn > 0.0 ? qmax[r] - q[r] : qmin[r] - q[r];
            const double num = ((dp * dp) + eps2) * dn + 2.0 * dn * dn * dp;
            const double den = ((dp * dp + 2.0 * dn * dn) + dn * dp + eps2) * dn;
            const double id = 1.0 / den;
            const double temp = num * id;
            if (temp < 1.0) {
                phi[r] = temp;
                idn[r] = id;
                active |= 1u << r;
            }
        }
        qt[r] = q[r] - 0.5 * phi[r] * t[r];
    }
    double qtb[4] = {0.0, 0.0, 0.0, 0.0};
    qtilde_to_primitive_b(qt, gm1, rho, u1b, u2b, rhob, prb, qtb);
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        qb[r] += qtb[r];
        double tb = -0.5 * phi[r] * qtb[r];
        if ((active >> r) & 1u) {
            // venkat_limiter_b of component r
            const double phib = -0.5 * t[r] * qtb[r];
            const double dn = (q[r] - 0.5 * t[r]) - q[r];
            const bool up = dn > 0.0;
            const double dp = up ? qmax[r] - q[r] : qmin[r] - q[r];
            const double num1 = (dp * dp) + eps2;
            const double den1 = dp * dp + 2.0 * dn * dn;
            const double den2 = den1 + dn * dp + eps2;
            const double numb = phib * idn[r];
            const double denb = -phib * phi[r] * idn[r];
            const double den2b = denb * dn;
            double dnb = denb * den2;
            const double den1b = den2b;
            dnb += den2b * dp;
            double dpb = den2b * dn;
            dpb += den1b * 2.0 * dp;
            dnb += den1b * 4.0 * dn;
            const double num1b = numb * dn;
            dnb += numb * (num1 + 4.0 * dn * dp);
            dpb += numb * 2.0 * dn * dn;
            dpb += num1b * 2.0 * dp;
            if (up) qmaxb[r] += dpb;
            else qminb[r] += dpb;
            qb[r] -= dpb;
            // dn = qt0 - q with qt0 = q - t/2: q's two shares of dnb cancel
            tb += -0.5 * dnb;
        }
        delxb += tb * dqx[r];
        delyb += tb * dqy[r];
        dqxb[r] += tb * delx;
        dqyb[r] += tb * dely;
    }
}

// primitive_to_conserved_b (state_update.F90:144-163)
__device__ __forceinline__ void prim_to_conserved_b(double rho, double u1, double u2, double pr,
                                                    double nx, double ny, const double Ub[4],
                                                    double pb[4], double &nxb, double &nyb) {
    const double t1 = rho * u1, t2 = rho * u2;
    const double t1b = Ub[1] * ny + Ub[2] * nx + Ub[3] * (t1 / rho);
    const double t2b = -Ub[1] * nx + Ub[2] * ny + Ub[3] * (t2 / rho);
    nxb += -Ub[1] * t2 + Ub[2] * t1;
    nyb += Ub[1] * t1 + Ub[2] * t2;
    pb[3] += 2.5 * Ub[3];
    pb[0] += Ub[0] - Ub[3] * 0.5 * (t1 * t1 + t2 * t2) / (rho * rho) + t1b * u1 + t2b * u2;
    pb[1] += t1b * rho;
    pb[2] += t2b * rho;
}

// conserved_vector_Ubar_b (state_update.F90:239-294): the point half w.r.t.
// prim and (nx, ny), and the freestream half w.r.t. (nx, ny).
__device__ __forceinline__ void conserved_ubar_b(double rho, double u1, double u2, double pr,
                                                 double nx, double ny, const double qinf[4],
                                                 double pi, double gm1, const double Ub[4],
                                                 double pb[4], double &nxb, double &nyb) {
    // point half
    const double u1r = u1 * ny - u2 * nx;
    const double u2r = u1 * nx + u2 * ny;
    const double e = pr / (rho * gm1) + 0.5 * (u1r * u1r + u2r * u2r);
    const double beta = rho / (2.0 * pr);
    const double sb = sqrt(beta);
    const double S2 = u2r * sb;
    const double spb = sqrt(pi * beta);
    const double E2 = exp(-S2 * S2);
    const double B2 = E2 / (2.0 * spb);
    const double A2p = 0.5 * (1.0 + erf(S2));
    double rhob = Ub[0] * A2p + Ub[1] * u1r * A2p + Ub[2] * (u2r * A2p + B2) +
                  Ub[3] * (A2p * e + 0.5 * u2r * B2);
    const double A2pb = Ub[0] * rho + Ub[1] * rho * u1r + Ub[2] * rho * u2r + Ub[3] * rho * e;
    double u1rb = Ub[1] * rho * A2p;
    double u2rb = Ub[2] * rho * A2p + Ub[3] * 0.5 * rho * B2;
    const double B2b = Ub[2] * rho + Ub[3] * 0.5 * rho * u2r;
    const double eb = Ub[3] * rho * A2p;
    double prb = eb / (rho * gm1);
    rhob += -eb * pr / (rho * rho * gm1);
    u1rb += eb * u1r;
    u2rb += eb * u2r;
    double S2b = A2pb * 0.5 * MFCFD_TWO_OVER_SQRT_PI * E2 + B2b * B2 * (-2.0 * S2);
    const double spbb = -B2b * B2 / spb;
    u2rb += S2b * sb;
    const double sbb = S2b * u2r;
    double betab = sbb / (2.0 * sb) + spbb * pi / (2.0 * spb);
    rhob += betab / (2.0 * pr);
    prb += -betab * beta / pr;
    pb[0] += rhob;
    pb[1] += u1rb * ny + u2rb * nx;
    pb[2] += -u1rb * nx + u2rb * ny;
    pb[3] += prb;
    nxb += -u1rb * u2 + u2rb * u1;
    nyb += u1rb * u1 + u2rb * u2;
    // freestream half
    const double rho_inf = qinf[0], u1i = qinf[1], u2i = qinf[2], pr_inf = qinf[3];
    const double u1ri = u1i * ny - u2i * nx;
    const double u2ri = u1i * nx + u2i * ny;
    const double e_inf = pr_inf / (rho_inf * gm1) + 0.5 * (u1ri * u1ri + u2ri * u2ri);
    const double beti = (0.5 * rho_inf) / pr_inf;
    const double sbi = sqrt(beti);
    const double S2i = u2ri * sbi;
    const double B2i = exp(-S2i * S2i) / (2.0 * sqrt(pi * beti));
    const double A2ni = 0.5 * (1.0 - erf(S2i));
    const double A2nib = rho_inf * (Ub[0] + Ub[1] * u1ri + Ub[2] * u2ri + Ub[3] * e_inf);
    const double e_infb = Ub[3] * rho_inf * A2ni;
    const double u1rib = Ub[1] * rho_inf * A2ni + e_infb * u1ri;
    double u2rib = Ub[2] * rho_inf * A2ni - Ub[3] * 0.5 * rho_inf * B2i + e_infb * u2ri;
    const double B2ib = -Ub[2] * rho_inf - Ub[3] * 0.5 * rho_inf * u2ri;
    const double S2ib = -A2nib * 0.5 * MFCFD_TWO_OVER_SQRT_PI * exp(-S2i * S2i) +
                        B2ib * B2i * (-2.0 * S2i);
    u2rib += S2ib * sbi;
    nxb += -u1rib * u2i + u2rib * u1i;
    nyb += u1rib * u1i + u2rib * u2i;
}

// q_variables_b (q_variables.F90:8-37)
__device__ __forceinline__ void q_from_prim_b(double rho, double u1, double u2, double pr,
                                              const double qb[4], double pb[4]) {
    const double beta = 0.5 * rho / pr;
    double betab = qb[0] * (2.5 / beta - (u1 * u1 + u2 * u2)) +
                   2.0 * (qb[1] * u1 + qb[2] * u2 - qb[3]);
    pb[0] += qb[0] / rho + betab * 0.5 / pr;
    pb[3] += -betab * beta / pr;
    pb[1] += -qb[0] * 2.0 * beta * u1 + qb[1] * 2.0 * beta;
    pb[2] += -qb[0] * 2.0 * beta * u2 + qb[2] * 2.0 * beta;
}

}  // namespace lskum
