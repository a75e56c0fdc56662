// Internal interface between the C ABI (api.cu) and the kernel launchers.
#pragma once

#include <cuda_runtime.h>

#include "lskum_device.cuh"

namespace lskum {

// Control block in device memory (one per handle).
struct Ctl {
    int it;           // iteration number the next residual belongs to
    int it_first;     // first iteration of the current run call
    int halted;       // 1 once a residue was NaN
    int done;         // iterations completed in the current call
    int active;       // 1 while the instance is scheduled (0 after it retires)
    int state;        // BatchState the instance retired with
    int restart;      // reference `restart` flag
    int plen;         // points in the residual norm
    double res_old;   // residual norm the residue is measured against
};
// Ctl fields a run call resets from the host (it .. state); the rest stays
// on the device between calls.
constexpr size_t CTL_RESET_BYTES = 6 * sizeof(int);

// Batched runs ------------------------------------------------------------
constexpr int TILE = 16;        // points per schedule tile (= points per flux block)
constexpr int MAX_BATCH = 256;  // instances per batch
enum BatchState { BATCH_RUNNING = 0, BATCH_CONVERGED = 1, BATCH_MAX_ITERS = 2,
                  BATCH_NONFINITE = 3 };

// One instance inside the concatenated point set (all counts in points
// except tile0/ntiles).
struct InstInfo {
    int base;     // first global point (a multiple of TILE)
    int n, nw, no;
    int obc_off;  // first row of the instance's outer points in Geom::obc
    int tile0;    // base / TILE
    int ntiles;   // ceil(n / TILE)
    int pad;
};

// Schedule of the running instances, one int block in device memory:
// [nact, ticket counter, pre[MAX_BATCH + 1], act[MAX_BATCH]] -- pre[a] = tiles
// before running slot a (pre[nact] = total), act[a] = its instance.  Written
// by the host at the start of a run and by the residual kernel after every
// iteration.
constexpr int SCHED_NACT = 0, SCHED_COUNTER = 1, SCHED_PRE = 2, SCHED_ACT = 3 + MAX_BATCH;
constexpr int SCHED_INTS = 3 + 2 * MAX_BATCH;
struct Sched {
    const InstInfo *inst;  // [n_inst]
    const int *pre;
    const int *act;
    const int *nact;
};
inline Sched sched_view(const InstInfo *inst, const int *blk) {
    return Sched{inst, blk + SCHED_PRE, blk + SCHED_ACT, blk + SCHED_NACT};
}
// Host: the schedule of the instances with active[i] != 0, in instance order.
inline void sched_fill(int *blk, const InstInfo *inst, const int *active, int n_inst) {
    int na = 0, pre = 0;
    for (int i = 0; i < n_inst; ++i)
        if (active[i]) {
            blk[SCHED_PRE + na] = pre;
            blk[SCHED_ACT + na] = i;
            pre += inst[i].ntiles;
            ++na;
        }
    blk[SCHED_PRE + na] = pre;
    blk[SCHED_NACT] = na;
    blk[SCHED_COUNTER] = 0;
}

// Retirement rule of the current batched run (device memory, read by
// kb_residual, so the captured graphs need no update).
struct BatchRun {
    double tol;     // retire once residue <= tol
    int max_iters;  // retire after this many iterations of the run
    int pad;
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
    // per (point, slot) the two reconstructed kinetic states and velocities
    // ([n][kp][KS_TAPE], the adjoint's tape), or nullptr
    double *kstape = nullptr;
};
// doubles per (point, slot) in the kinetic-state tape: for the point's and
// then the neighbour's reconstruction rho p/rho B1 B2 erf1 erf2 u1 u2
constexpr int KS_TAPE = 16;

// The passes of one stage.  Each is a grid-stride kernel over the tiles of
// the scheduled instances; `block` threads per block for the point passes
// and `grid` blocks (0 = one wave of resident blocks).
// D pass: qm and dq (eval_q_derivatives); with_delta also computes the
// local time step (func_delta) from spd of the neighbours.
void launch_grad(const Geom &g, const Consts &c, const Sched &s, const R4 *q, const double *spd,
                 double *dq, double *qm, double *delta, bool with_delta, int block, int grid,
                 cudaStream_t st);
// I pass: one inner iteration (eval_q_inner_loop + eval_update_innerloop).
// dq0: the stage's D-pass derivatives (kept through its inner iterations;
// the FP64 dq buffers rotate as dq_src / dq_dst say).
void launch_inner(const Geom &g, const Consts &c, const Sched &s, const double *dq0,
                  const double *dq_in, double *dq_out, int block, int grid, cudaStream_t st);
// F pass: flux residual + state update of stage rk (1-based).
void launch_flux(const Geom &g, const Consts &c, const Sched &s, const StageBufs &b, int rk,
                 bool last, int grid, cudaStream_t st);
// Residual norm and residue of one iteration per instance (hist row i, entry
// it - it_first), retirement, and the schedule of the next iteration.
void launch_residual(const InstInfo *inst, int n_inst, const double *res_part, Ctl *ctl,
                     double *hist, int hist_ld, const BatchRun *run, int *sched,
                     cudaStream_t st);
// One-time kernel attributes (before any stream capture).
cudaError_t init_kernels();
// tiles (TILE-point schedule units) of n points
int flux_blocks(int n);
// flux-pass blocks beyond which some warps would find no chunk of two tiles
int flux_grid_blocks(int n);
// resident blocks per SM (kind: 0 D pass, 1 I pass, 2 F pass; fp32 selects
// the FP32-mixed kernels)
int batch_occupancy(int kind, bool fp32, int block, size_t smem);
int batch_occupancy32(int kind, int block, size_t smem);
// dynamic shared memory of the flux passes for stencils of kp slots
size_t flux_smem_bytes(int kp);
size_t flux32_smem_bytes(int kp);
// blocks of one wave of resident blocks of a pass on device dev (for the
// point passes their own staging memory replaces `smem`)
int wave_blocks(int dev, int kind, int block, size_t smem, bool fp32);
// threads per block of the point passes (their staging buffers take up to
// 512 B of shared memory a thread)
inline int default_point_block(bool) { return 128; }
// q and spd from prim (set_state)
void launch_init_state(const Geom &g, const R4 *prim, R4 *q, double *spd, cudaStream_t s);
// q and spd of rows [i0, i1) only (the ghost rows of a partitioned grid)
void launch_init_rows(const Geom &g, const R4 *prim, R4 *q, double *spd, int i0, int i1,
                      cudaStream_t s);
// *out = the sum of nparts tile partials, in a fixed order
void launch_sum_parts(const double *part, int nparts, double *out, cudaStream_t s);

// FP32-mixed geometry, precomputed once per grid in FP64 and rounded:
// offsets to the stencil neighbours [slot][point] (and weights when power
// != 0, else w == nullptr), the inverse normal matrix of each point's full
// stencil (a, b, c: dx = a Sx + b Sy, dy = b Sx + c Sy) and per split list
// the two coefficients of the flux solve ([2i] lists 0-1, [2i+1] lists 2-3).
struct Geom32 {
    const float2 *dxy;
    const float *w;
    const float4 *lsq;
    const float4 *flsq;
};

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
    Geom32 f;
};
cudaError_t init_kernels32();
void launch_grad32(const Geom &g, const Consts &c, const Geom32 &f, const Sched &s,
                   const float4 *q, const double *spd, float *dq, float *qm, double *delta,
                   bool with_delta, int block, int grid, cudaStream_t st);
// dq0: the D pass's derivatives of the stage, kept through its inner
// iterations (the FP32 buffers rotate as dq32_src / dq32_dst say)
void launch_inner32(const Geom &g, const Consts &c, const Geom32 &f, const Sched &s,
                    const float *dq0, const float *dq_in, float *dq_out, int block, int grid,
                    cudaStream_t st);
// FP32 dq buffers of a stage: 0 holds the D pass's result for the whole
// stage; inner iteration t (1-based) reads dq32_src(t), writes dq32_dst(t);
// the flux pass reads dq32_final(m).
inline int dq32_src(int t) { return t == 1 ? 0 : 1 + ((t - 2) & 1); }
inline int dq32_dst(int t) { return 1 + ((t - 1) & 1); }
inline int dq32_final(int m) { return m == 0 ? 0 : dq32_dst(m); }
// the FP64 dq buffers of a stage rotate the same way
inline int dq_src(int t) { return dq32_src(t); }
inline int dq_dst(int t) { return dq32_dst(t); }
inline int dq_final(int m) { return dq32_final(m); }
void launch_flux32(const Geom &g, const Consts &c, const Sched &s, const StageBufs32 &b, int rk,
                   bool last, int grid, cudaStream_t st);
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
