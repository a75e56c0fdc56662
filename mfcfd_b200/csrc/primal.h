// Internal interface between the C ABI (api.cu) and the kernel launchers.
#pragma once

#include <cuda_runtime.h>

#include "lskum_device.cuh"

namespace lskum {

// Control block in device memory (one per handle).
struct Ctl {
    int it;           // iteration number the next residual belongs to
    int it_first;     // first iteration of the current mfcfd_run call
    int halted;       // 1 once a residue was NaN: later kernels return at once
    int done;         // iterations completed in the current call
    int restart;      // reference `restart` flag
    int plen;         // points in the residual norm
    double res_old;   // residual norm the residue is measured against
};

// Buffers one pseudo-time stage reads and writes.
struct StageBufs {
    const R4 *prim_in;   // state the stage starts from
    R4 *prim_out;        // updated state (may alias prim_in)
    const R4 *prim_old;  // state at the start of the iteration (rk == 3)
    const R4 *q_in;      // q of prim_in
    R4 *q_out;           // q of prim_out
    const double *dq;    // [n][8] final dq of the stage (dq/dx 1..4, dq/dy 1..4)
    const double *qm;    // [n][8] max 1..4, min 1..4
    const double *delta; // local time step
    double *spd;         // |u| + 3 sqrt(p/rho) of prim_out (last stage)
    double *res_part;    // per-block sums of res_sqr (last stage)
    double *flux_dbg;    // [n][4] flux_res, or nullptr
};

// D pass: qm and dq (eval_q_derivatives); with_delta also computes the
// local time step (func_delta) from spd of the neighbours.
void launch_grad(const Geom &g, const Consts &c, const R4 *q, const double *spd, double *dq,
                 double *qm, double *delta, bool with_delta, const Ctl *ctl, cudaStream_t s);
// I pass: one inner iteration (eval_q_inner_loop + eval_update_innerloop).
void launch_inner(const Geom &g, const Consts &c, const R4 *q, const double *dq_in,
                  double *dq_out, const Ctl *ctl, cudaStream_t s);
// One-time kernel attributes (before any stream capture).
cudaError_t init_kernels();
// F pass: flux residual + state update of stage rk (1-based).
int flux_blocks(int n);
void launch_flux(const Geom &g, const Consts &c, const StageBufs &b, int rk, bool last,
                 const Ctl *ctl, cudaStream_t s);
// residual norm / residue of one iteration; writes hist[it - it_first].
void launch_residual(const double *res_part, int nparts, Ctl *ctl, double *hist,
                     cudaStream_t s);
// q and spd from prim (set_state)
void launch_init_state(const Geom &g, const R4 *prim, R4 *q, double *spd, cudaStream_t s);

// FP32-mixed stage buffers: FP32 prim/q/dq/qm, FP64 delta/spd/partials.
struct StageBufs32 {
    const float4 *prim_in;
    float4 *prim_out;
    const float4 *prim_old;
    const float4 *q_in;
    float4 *q_out;
    const float *dq;     // [n][8]
    const float *qm;     // [n][8]
    const float *eps2f;  // eps2 rounded to FP32
    const double *delta;
    double *spd;
    double *res_part;
    double *flux_dbg;
};
cudaError_t init_kernels32();
void launch_grad32(const Geom &g, const Consts &c, const float4 *q, const double *spd, float *dq,
                   float *qm, double *delta, bool with_delta, const Ctl *ctl, cudaStream_t s);
void launch_inner32(const Geom &g, const Consts &c, const float4 *q, const float *dq_in,
                    float *dq_out, const Ctl *ctl, cudaStream_t s);
void launch_flux32(const Geom &g, const Consts &c, const StageBufs32 &b, int rk, bool last,
                   const Ctl *ctl, cudaStream_t s);
void launch_init_state32(const Geom &g, const float4 *prim, float4 *q, double *spd,
                         cudaStream_t s);
// float4 prim -> FP64 rows (for the force sums and diagnostics)
void launch_widen(const float4 *in, R4 *out, int n, cudaStream_t s);

// Shape-point force sums (compute_cl_cd_cm), serial in grid order.
struct ShapeTab {
    int npts, shapes;
    const int *idx;        // renumbered point
    const int *shape;      // 0-based shape number
    const double *geo;     // [npts][4]: nx, ny, ds, mx ; my in geo2
    const double *my;      // [npts]
};
void launch_forces(const ShapeTab &t, const R4 *prim, double mach, double cos_t, double sin_t,
                   double *out /* 3*shapes cl,cd,cm then npts cp */, cudaStream_t s);

}  // namespace lskum
