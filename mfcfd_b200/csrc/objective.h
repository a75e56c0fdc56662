// Internal: values and reverse seeds of the objectives (objective_fp64.cu).
#pragma once

#include "handle.h"

namespace lskum_host {
// gamma/(gamma-1) and p0_inf of stagnation_values.F90:56-57
double stagnation_gamma_power();
double stagnation_p0_inf(double mach);
// J of objective `kind` (MFCFD_OBJ_*) for the state prim (renumbered rows)
int objective_value(mfcfd_t *h, int kind, const lskum::R4 *prim, double *J);
// seeds pb (and for the enstrophy xb, yb and the contribution records) with
// dJ/d(prim, x, y) of objective kind 2..4 at the state prim
void launch_objective_b(mfcfd_t *h, int kind, const lskum::R4 *prim, double *pb, double *xb,
                        double *yb, double *contrib, cudaStream_t s);
}  // namespace lskum_host
