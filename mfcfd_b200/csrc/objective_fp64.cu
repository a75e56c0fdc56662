// The reference's secondary objectives (present in src_mpi_primal, called
// from objective_function only in commented-out lines):
//   total entropy     compute_entropy.F90:10-40    sum |log(p/rho^gamma) - log(pr_inf)|
//   total enstrophy   compute_enstrophy.F90:9-89   sum (du2/dx - du1/dy)^2, the
//                     velocity gradient by least squares over the stencil
//   stagnation-pressure loss  stagnation_values.F90:43-76
//                     sum (p0_inf - p0)^2 / (p0_inf^2 N)
// as the value (mfcfd_objective) and as seeds of the reverse sweep: the
// adjoint of J with respect to the final state and, for the enstrophy, the
// coordinates.  Per-point terms are evaluated on the device; the sums run on
// the host over the caller's point order, the reference's loop order.
#include <cuda_runtime.h>

#include <vector>

#include "adjoint.h"
#include "handle.h"
#include "objective.h"

using namespace lskum;
using lskum_host::cuda_fail;
using lskum_host::dmalloc;
using lskum_host::fail;

namespace {

constexpr double GAMMA = 1.4;
constexpr double PR_INF = 1.0 / 1.4;

__device__ __forceinline__ double entropy_term(const R4 &P) {
    double temp1 = pow(P.a, GAMMA);
    temp1 = P.d / temp1;
    temp1 = log(temp1);
    return fabs(temp1 - log(PR_INF));
}

// p0 of stagnation_values.F90:63-66; mach_t^2 formed as |u|^2 / (gamma p / rho)
__device__ __forceinline__ double stagnation_p0(const R4 &P, double gamma_power) {
    const double angle = sqrt(GAMMA * P.d / P.a);
    const double mach_t = sqrt(P.b * P.b + P.c * P.c) / angle;
    return P.d * pow(1 + ((GAMMA - 1) / 2) * mach_t * mach_t, gamma_power);
}

// least-squares velocity gradient terms of compute_enstrophy.F90:27-67
struct Vort {
    double sxx, syy, sxy, sxu1, sxu2, syu1, syu2;
};
__device__ __forceinline__ Vort vort_sums(const Geom &g, const Consts &c, const R4 *prim, int i) {
    Vort v{0, 0, 0, 0, 0, 0, 0};
    const double2 pi_ = g.xy[i];
    const R4 Pi = ld4(prim + i);
    const int nb = g.nbhs[i];
    for (int r = 0; r < nb; ++r) {
        const int k = g.conn[r * g.n + i];
        const double2 pk = g.xy[k];
        const R4 Pk = ld4(prim + k);
        const double delx = pk.x - pi_.x, dely = pk.y - pi_.y;
        const double w = c.power_zero ? 1.0 : pow(sqrt(delx * delx + dely * dely), c.power);
        v.sxx = v.sxx + delx * delx * w;
        v.syy = v.syy + dely * dely * w;
        v.sxy = v.sxy + delx * dely * w;
        v.sxu1 = v.sxu1 + w * delx * (Pk.b - Pi.b);
        v.sxu2 = v.sxu2 + w * delx * (Pk.c - Pi.c);
        v.syu1 = v.syu1 + w * dely * (Pk.b - Pi.b);
        v.syu2 = v.syu2 + w * dely * (Pk.c - Pi.c);
    }
    return v;
}

__global__ void k_obj_terms(Geom g, Consts c, const R4 *__restrict__ prim, int kind,
                            double gamma_power, double p0_inf, double *__restrict__ term) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.n) return;
    const R4 P = ld4(prim + i);
    if (kind == MFCFD_OBJ_ENTROPY) {
        term[i] = entropy_term(P);
    } else if (kind == MFCFD_OBJ_STAGNATION) {
        const double d = p0_inf - stagnation_p0(P, gamma_power);
        term[i] = d * d;
    } else {
        const Vort v = vort_sums(g, c, prim, i);
        const double one_by_det = 1.0 / (v.sxx * v.syy - v.sxy * v.sxy);
        const double du2_dx = (v.sxu2 * v.syy - v.syu2 * v.sxy) * one_by_det;
        const double du1_dy = (v.syu1 * v.sxx - v.sxu1 * v.sxy) * one_by_det;
        const double temp = du2_dx - du1_dy;
        term[i] = temp * temp;
    }
}

// Seeds of the reverse sweep (the adjoints of the Tapenade _b routines of
// the objectives): pb += dJ/dprim of each point; for the enstrophy also the
// coordinates (xb, yb of the point itself, and per stencil slot a
// contribution record for the neighbour: fields 4..7 its prim adjoint, 8..9
// its x, y adjoint, added by the gather in the transposed-stencil order).
__global__ void k_obj_seed_b(Geom g, const R4 *__restrict__ prim, int kind, double gamma_power,
                             double p0_inf, double scale, double *__restrict__ pb,
                             double *__restrict__ xb, double *__restrict__ yb,
                             double *__restrict__ contrib) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.n) return;
    const R4 P = ld4(prim + i);
    if (kind == MFCFD_OBJ_ENTROPY) {
        // t = log(p / rho^gamma); term = |t - log(pr_inf)|
        const double t = log(P.d / pow(P.a, GAMMA)) - log(PR_INF);
        const double s = t >= 0.0 ? 1.0 : -1.0;
        pb[4 * (size_t)i + 0] += -s * GAMMA / P.a;
        pb[4 * (size_t)i + 3] += s / P.d;
    } else if (kind == MFCFD_OBJ_STAGNATION) {
        // p0 = p A^gp, A = 1 + g2 M^2, M^2 = rho |u|^2 / (gamma p)
        const double g2 = (GAMMA - 1) / 2;
        const double m2 = P.a * (P.b * P.b + P.c * P.c) / (GAMMA * P.d);
        const double A = 1 + g2 * m2;
        const double Agm1 = pow(A, gamma_power - 1.0);
        const double p0 = P.d * Agm1 * A;
        const double p0b = scale * -2.0 * (p0_inf - p0);
        const double f = gamma_power * Agm1 * g2;  // d p0 / d(M^2), over p
        pb[4 * (size_t)i + 0] += p0b * f * m2 * P.d / P.a;
        pb[4 * (size_t)i + 1] += p0b * f * 2.0 * P.b * P.a / GAMMA;
        pb[4 * (size_t)i + 2] += p0b * f * 2.0 * P.c * P.a / GAMMA;
        pb[4 * (size_t)i + 3] += p0b * Agm1 * (A - gamma_power * g2 * m2);
    } else {
        // enstrophy: J = sum w^2, w = du2/dx - du1/dy (weights 1: power 0)
        Consts c0{};
        c0.power_zero = 1;
        const Vort v = vort_sums(g, c0, prim, i);
        const double obd = 1.0 / (v.sxx * v.syy - v.sxy * v.sxy);
        const double du2_dx = (v.sxu2 * v.syy - v.syu2 * v.sxy) * obd;
        const double du1_dy = (v.syu1 * v.sxx - v.sxu1 * v.sxy) * obd;
        const double wb = 2.0 * (du2_dx - du1_dy);
        const double du2_dxb = wb, du1_dyb = -wb;
        double sxu2b = du2_dxb * v.syy * obd, syu2b = -du2_dxb * v.sxy * obd;
        double syyb = du2_dxb * v.sxu2 * obd, sxyb = -du2_dxb * v.syu2 * obd;
        double obdb = du2_dxb * (v.sxu2 * v.syy - v.syu2 * v.sxy);
        const double syu1b = du1_dyb * v.sxx * obd, sxu1b = -du1_dyb * v.sxy * obd;
        double sxxb = du1_dyb * v.syu1 * obd;
        sxyb += -du1_dyb * v.sxu1 * obd;
        obdb += du1_dyb * (v.syu1 * v.sxx - v.sxu1 * v.sxy);
        const double detb = -obdb * obd * obd;
        sxxb += detb * v.syy;
        syyb += detb * v.sxx;
        sxyb += -2.0 * detb * v.sxy;
        const double2 pi_ = g.xy[i];
        double u1ib = 0.0, u2ib = 0.0, xib = 0.0, yib = 0.0;
        const int nb = g.nbhs[i];
        for (int r = 0; r < nb; ++r) {
            const int k = g.conn[r * g.n + i];
            const double2 pk = g.xy[k];
            const R4 Pk = ld4(prim + k);
            const double dx = pk.x - pi_.x, dy = pk.y - pi_.y;
            const double du1 = Pk.b - P.b, du2 = Pk.c - P.c;
            const double dxb = 2.0 * dx * sxxb + dy * sxyb + du1 * sxu1b + du2 * sxu2b;
            const double dyb = 2.0 * dy * syyb + dx * sxyb + du1 * syu1b + du2 * syu2b;
            const double du1b = dx * sxu1b + dy * syu1b;
            const double du2b = dx * sxu2b + dy * syu2b;
            double *cb = contrib + ((size_t)i * g.kp + r) * ADJ_CW;
            cb[0] = cb[1] = cb[2] = cb[3] = 0.0;
            cb[4] = 0.0;
            cb[5] = du1b;
            cb[6] = du2b;
            cb[7] = 0.0;
            cb[8] = dxb;
            cb[9] = dyb;
            u1ib -= du1b;
            u2ib -= du2b;
            xib -= dxb;
            yib -= dyb;
        }
        pb[4 * (size_t)i + 1] += u1ib;
        pb[4 * (size_t)i + 2] += u2ib;
        xb[i] += xib;
        yb[i] += yib;
    }
}

}  // namespace

namespace lskum_host {

double stagnation_gamma_power() { return GAMMA / (GAMMA - 1); }
double stagnation_p0_inf(double mach) {
    const double gp = GAMMA / (GAMMA - 1);
    return PR_INF * pow(1 + ((GAMMA - 1) / 2) * mach * mach, gp);
}

int objective_value(mfcfd_t *h, int kind, const R4 *prim, double *J) {
    const int n = h->n;
    if (kind == MFCFD_OBJ_CL || kind == MFCFD_OBJ_CD) {
        std::vector<double> cl(h->shapes), cd(h->shapes), cm(h->shapes);
        int st = mfcfd_forces(h, cl.data(), cd.data(), cm.data(), nullptr);
        if (st) return st;
        double s = 0.0;
        for (int k = 0; k < h->shapes; ++k) s += kind == MFCFD_OBJ_CD ? cd[k] : cl[k];
        *J = s;
        return MFCFD_OK;
    }
    double *d_term = nullptr;
    CK(dmalloc(&d_term, n));
    const double gp = stagnation_gamma_power(), p0_inf = stagnation_p0_inf(h->p.mach);
    k_obj_terms<<<(n + 255) / 256, 256, 0, h->stream>>>(h->geom, h->consts, prim, kind, gp, p0_inf,
                                                        d_term);
    h->launches += 1;
    std::vector<double> term(n);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(term.data(), d_term, sizeof(double) * n, cudaMemcpyDeviceToHost,
                            h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(d_term);
    if (e != cudaSuccess) return cuda_fail(h, e, "objective terms");
    std::vector<int> inv(n);
    for (int p = 0; p < n; ++p) inv[h->perm[p]] = p;
    double s = 0.0;
    for (int k = 0; k < n; ++k) s = s + term[inv[k]];
    if (kind == MFCFD_OBJ_STAGNATION) s = s * (1 / (p0_inf * p0_inf * h->n));
    *J = s;
    return MFCFD_OK;
}

void launch_objective_b(mfcfd_t *h, int kind, const R4 *prim, double *pb, double *xb, double *yb,
                        double *contrib, cudaStream_t s) {
    const double gp = stagnation_gamma_power(), p0_inf = stagnation_p0_inf(h->p.mach);
    const double scale = 1 / (p0_inf * p0_inf * h->n);
    k_obj_seed_b<<<(h->n + 255) / 256, 256, 0, s>>>(h->geom, prim, kind, gp, p0_inf, scale, pb,
                                                    xb, yb, contrib);
    h->launches += 1;
}

}  // namespace lskum_host

extern "C" int mfcfd_objective(mfcfd_t *h, int objective, double *J) {
    if (!h || !J) return MFCFD_ERR_ARG;
    if (objective < MFCFD_OBJ_CL || objective > MFCFD_OBJ_STAGNATION)
        return fail(h, MFCFD_ERR_ARG, "objective must be 0..4");
    CK(cudaStreamSynchronize(h->stream));
    const R4 *prim = h->d_prim[h->cur];
    if (h->fp32) {
        launch_widen(h->f_prim[h->cur], h->d_prim[0], h->n, h->stream);
        h->launches += 1;
        prim = h->d_prim[0];
    }
    return lskum_host::objective_value(h, objective, prim, J);
}
