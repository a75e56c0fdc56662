// Forward-mode (tangent) scalar: a value and its directional derivative.
//
// The primal device templates (reconstruct, kstate, split and quadrant
// fluxes, q_from_prim, prim_to_conserved, conserved_ubar) instantiated on
// Dual give the tangent of the reference's routines, like the Tapenade
// `_d` routines of src_mpi_forward/sensitivity_files (q_lskum_d.F90:28-89).
// Comparisons act on values, so a branch (limiter threshold, max/min, the
// time-step minimum) passes the derivative of the branch taken.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace lskum {

struct Dual {
    double v, d;
    __host__ __device__ Dual() : v(0.0), d(0.0) {}
    __host__ __device__ Dual(double x) : v(x), d(0.0) {}  // NOLINT: constants are duals
    __host__ __device__ Dual(double x, double dx) : v(x), d(dx) {}
};

__host__ __device__ inline Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
__host__ __device__ inline Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
__host__ __device__ inline Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
__host__ __device__ inline Dual operator*(Dual a, Dual b) {
    return Dual(a.v * b.v, a.d * b.v + a.v * b.d);
}
__host__ __device__ inline Dual operator/(Dual a, Dual b) {
    const double q = a.v / b.v;
    return Dual(q, (a.d - q * b.d) / b.v);
}
__host__ __device__ inline Dual &operator+=(Dual &a, Dual b) { return a = a + b; }
__host__ __device__ inline Dual &operator-=(Dual &a, Dual b) { return a = a - b; }
__host__ __device__ inline bool operator<(Dual a, Dual b) { return a.v < b.v; }
__host__ __device__ inline bool operator>(Dual a, Dual b) { return a.v > b.v; }
__host__ __device__ inline bool operator<=(Dual a, Dual b) { return a.v <= b.v; }
__host__ __device__ inline bool operator>=(Dual a, Dual b) { return a.v >= b.v; }

__host__ __device__ inline Dual fabs(Dual a) { return a.v < 0.0 ? -a : a; }
__host__ __device__ inline Dual sqrt(Dual a) {
    const double s = ::sqrt(a.v);
    return Dual(s, a.d / (2.0 * s));
}
__host__ __device__ inline Dual exp(Dual a) {
    const double e = ::exp(a.v);
    return Dual(e, e * a.d);
}
__host__ __device__ inline Dual log(Dual a) { return Dual(::log(a.v), a.d / a.v); }
// d erf(x)/dx = 2/sqrt(pi) exp(-x^2)
__host__ __device__ inline Dual erf(Dual a) {
    const double two_by_sqrt_pi = 1.1283791670955126;
    return Dual(::erf(a.v), two_by_sqrt_pi * ::exp(-a.v * a.v) * a.d);
}

}  // namespace lskum
