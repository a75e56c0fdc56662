// mfcfd_output_fields: the CUDA tree's post-processing fields of the state.
//
//   Mach number   src_cuda/post_processing.F90:24-27, sqrt(|u|^2 / c) as the
//                 reference forms it (|u| squared over the sound speed)
//   entropy       src_cuda/compute_entropy.F90:10-30, |log(p/rho^gamma) - log(pr_inf)|
//   sensor        src_cuda/adaptation_sensors.F90:7-101, the largest D2
//                 distance to a stencil neighbour, normalised by its maximum
//
// One thread per point evaluates the three fields on the device; the sum of
// the entropy and the maximum of the D2 distance run on the host over the
// caller's point order, the reference's loop order.
#include <cuda_runtime.h>

#include <vector>

#include "handle.h"

using namespace lskum;
using lskum_host::cuda_fail;
using lskum_host::dmalloc;
using lskum_host::fail;

namespace {

__global__ void k_output_fields(Geom g, const R4 *__restrict__ prim, double *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.n) return;
    const double gamma = 1.4, pr_inf = 1.0 / 1.4;
    const R4 P = ld4(prim + i);
    const double rho_i = P.a, u1_i = P.b, u2_i = P.c, pr_i = P.d;
    const double sos = sqrt(gamma * pr_i / rho_i);
    const double vel_mag = u1_i * u1_i + u2_i * u2_i;
    double temp1 = pow(rho_i, gamma);
    temp1 = pr_i / temp1;
    temp1 = log(temp1);
    double maxi = 0.0;
    const int nb = g.nbhs[i];
    for (int r = 0; r < nb; ++r) {
        const R4 Q = ld4(prim + g.conn[r * g.n + i]);
        const double rho_j = Q.a, u1_j = Q.b, u2_j = Q.c, pr_j = Q.d;
        double t1 = (pr_i * pr_i * rho_j) / (pr_j * pr_j * rho_i);
        t1 = log(t1);
        t1 = (rho_j - rho_i) * t1;
        const double u_sqr = (u1_j - u1_i) * (u1_j - u1_i) + (u2_j - u2_i) * (u2_j - u2_i);
        double t2 = (rho_j / rho_i) + (pr_i * rho_j) / (pr_j * rho_i);
        t2 = t2 * u_sqr;
        t2 = (0.5 * rho_i * rho_i / pr_i) * t2;
        double t3 = rho_i * (((pr_i * rho_j) / (pr_j * rho_i)) - 1.0);
        t3 = t3 + rho_j * (((pr_j * rho_i) / (pr_i * rho_j)) - 1.0);
        t3 = 2.0 * t3;
        const double d2 = t1 + t2 + t3;
        if (d2 > maxi) maxi = d2;
    }
    out[3 * (size_t)i] = sqrt(vel_mag / sos);
    out[3 * (size_t)i + 1] = fabs(temp1 - log(pr_inf));
    out[3 * (size_t)i + 2] = maxi;
}

}  // namespace

extern "C" int mfcfd_output_fields(mfcfd_t *h, double *mach, double *entropy, double *sensor,
                                   double *total_entropy) {
    if (!h) return MFCFD_ERR_ARG;
    const int n = h->n;
    const R4 *prim = h->d_prim[h->cur];
    if (h->fp32) {
        launch_widen(h->f_prim[h->cur], h->d_prim[0], n, h->stream);
        h->launches += 1;
        prim = h->d_prim[0];
    }
    double *d_out = nullptr;
    CK(dmalloc(&d_out, (size_t)3 * n));
    k_output_fields<<<(n + 255) / 256, 256, 0, h->stream>>>(h->geom, prim, d_out);
    h->launches += 1;
    std::vector<double> o((size_t)3 * n);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(o.data(), d_out, o.size() * sizeof(double), cudaMemcpyDeviceToHost,
                            h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(d_out);
    if (e != cudaSuccess) return cuda_fail(h, e, "mfcfd_output_fields");
    // caller order: point k of the caller is renumbered point inv[k]
    std::vector<int> inv(n);
    for (int p = 0; p < n; ++p) inv[h->perm[p]] = p;
    double total = 0.0, max_sensor = 0.0;
    for (int k = 0; k < n; ++k) {
        const double *r = &o[3 * (size_t)inv[k]];
        if (mach) mach[k] = r[0];
        if (entropy) entropy[k] = r[1];
        total = total + r[1];
        if (r[2] >= max_sensor) max_sensor = r[2];
    }
    if (sensor)
        for (int k = 0; k < n; ++k) sensor[k] = o[3 * (size_t)inv[k] + 2] / max_sensor;
    if (total_entropy) *total_entropy = total;
    return MFCFD_OK;
}
