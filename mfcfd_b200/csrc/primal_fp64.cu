// FP64 kernels of the LSKUM pseudo-time loop on sm_100a.
//
// Per pseudo-time stage (fpi_solver.F90:27-53):
//   kb_grad_h   D pass  -- eval_q_derivatives (+ func_delta on the first stage)
//   kb_inner_h  I pass  -- eval_q_inner_loop + eval_update_innerloop, rearranged
//                          (dq buffers rotate; the D pass's result is kept)
//   kb_flux   F pass  -- cal_flux_residual + state_update + eval_q_variables of
//                        the new state (+ res_sqr partials on the last stage)
// and per iteration kb_residual (fpi_solver.F90:57-70).
//
// Every pass walks a schedule of instances (batch.cuh): a single grid is a
// schedule of one instance, a batch of independent grids one of many, and
// both run the same compiled kernels, so an instance's results do not depend
// on what it is batched with.
//
// Layout in HBM (renumbered points: wall | outer | interior): one 32-byte
// row per point for prim and q, 64-byte rows for dq and qm, 16-byte rows for
// (x, y) and (nx, ny); stencils as ELL columns conn[slot][point] so the
// thread-per-point passes read them coalesced.
#include <cuda_runtime.h>

#include <algorithm>

#include "batch.cuh"
#include "halo.cuh"
#include "primal.h"

namespace lskum {

namespace {

constexpr int GRAD_BLOCK = 256;  // blocks of the per-point set-up kernels
constexpr int LPP = 8;                   // lanes per point in the flux pass
constexpr int FLUX_BLOCK = 128;          // four independent warps
constexpr int REC = 19;                  // dGxp[4] dGxn[4] dGyp[4] dGyn[4] dels deln w
#ifndef FLUX_MIN_BLOCKS
#define FLUX_MIN_BLOCKS 4                // <= 128 registers; shared memory allows 4 blocks
#endif
constexpr double OBT = 1.0 / 3.0;        // state_update.F90:19-20
constexpr double TBT = 2.0 / 3.0;

// Rows in 256-bit read-only loads (ld.global.nc.v4.f64, sm_100): a 32-byte
// q row in one load, a 64-byte dq row in two (the D and I passes' rows of
// tiles without a staged halo, the I pass's dq0 row).  R4 rows and dq rows
// are 32-byte aligned.  The flux pass uses them for its 64-byte dq and qm
// rows only: its 32-byte q rows in the wide form made it spill.
__device__ __forceinline__ R4 ld4w(const R4 *p) {
    R4 r;
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
        : "=d"(r.a), "=d"(r.b), "=d"(r.c), "=d"(r.d)
        : "l"(p));
    return r;
}

__device__ __forceinline__ void ld8w(const double *p, double a[4], double b[4]) {
    const R4 u = ld4w(reinterpret_cast<const R4 *>(p));
    const R4 v = ld4w(reinterpret_cast<const R4 *>(p + 4));
    a[0] = u.a; a[1] = u.b; a[2] = u.c; a[3] = u.d;
    b[0] = v.a; b[1] = v.b; b[2] = v.c; b[3] = v.d;
}

// Row sources of the per-point sums of the D and I passes: the rows of a
// point's stencil gathered from global memory, or from its tile's halo
// staged in shared memory (kb_grad_h, kb_inner_h).  Both give the same
// values, so the sums below do not depend on where their rows come from.
struct GlobalRows {
    const Geom &g;
    const R4 *q;
    const double *dq;   // I pass: dq_in
    const double *spd;  // D pass
    int i;
    __device__ __forceinline__ int self() const { return i; }
    __device__ __forceinline__ int nbr(int r) const { return g.conn[r * g.n + i]; }
    __device__ __forceinline__ double2 xy(int k) const { return g.xy[k]; }
    __device__ __forceinline__ void qrow(int k, double v[4]) const {
        const R4 a = ld4w(q + k);
        v[0] = a.a; v[1] = a.b; v[2] = a.c; v[3] = a.d;
    }
    __device__ __forceinline__ void dqrow(int k, double x[4], double y[4]) const {
        ld8w(dq + 8 * (size_t)k, x, y);
    }
    __device__ __forceinline__ double spdv(int k) const { return spd[k]; }
};

// Shared-memory arrays of a staged tile halo, hc rows each (hc is the
// staging stride, one more than a multiple of eight, so that the arrays of a
// row start on different banks): D pass q[0..1], q[2..3], (x, y), (spd, -);
// I pass (x, y), dq/dx[0..1], dq/dx[2..3], dq/dy[0..1], dq/dy[2..3].  One
// 16-byte array per pair keeps a warp's reads of neighbouring rows on
// distinct banks.
constexpr int HA_I = 5, HA_D = 4;
constexpr int HALO_BLOCK = 128;  // four warps, a half-warp per tile
// resident blocks per SM the register budget allows, measured at C2: the D
// pass 0.090 ms at 4 (128 registers), 0.102 at 5, 0.132 at 6; the I pass
// 0.119 ms at 4, 0.087 at 5 (96 registers), 0.092 at 6
#ifndef HALO_MIN_BLOCKS_D
#define HALO_MIN_BLOCKS_D 4
#endif
#ifndef HALO_MIN_BLOCKS_I
#define HALO_MIN_BLOCKS_I 5
#endif

template <int nA>
struct HaloRows {
    static constexpr int OXY = nA == HA_I ? 0 : 2, ODQ = 1, OSPD = 3;
    const double2 *sm;
    int hc;
    HaloLoc loc;
    // i < 0: no point (nothing is loaded)
    __device__ __forceinline__ HaloRows(const Geom &g, const double2 *sm_, int i)
        : sm(sm_), hc(g.hc), loc(g, i) {}
    __device__ __forceinline__ int self() const { return loc.own; }
    __device__ __forceinline__ int nbr(int r) const { return loc.slot(r); }
    __device__ __forceinline__ double2 xy(int l) const { return sm[OXY * hc + l]; }
    __device__ __forceinline__ void qrow(int l, double v[4]) const {
        const double2 a = sm[l], b = sm[hc + l];
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    }
    __device__ __forceinline__ void dqrow(int l, double x[4], double y[4]) const {
        const double2 a = sm[ODQ * hc + l], b = sm[(ODQ + 1) * hc + l],
                      e = sm[(ODQ + 2) * hc + l], f = sm[(ODQ + 3) * hc + l];
        x[0] = a.x; x[1] = a.y; x[2] = b.x; x[3] = b.y;
        y[0] = e.x; y[1] = e.y; y[2] = f.x; y[3] = f.y;
    }
    __device__ __forceinline__ double spdv(int l) const { return sm[OSPD * hc + l].x; }
};

// q_variables.F90:41-112 eval_q_derivatives and state_update.F90:190-236
// func_delta over the rows of R, in slot order.
template <class Rows>
__device__ __forceinline__ void grad_sums(const Consts &c, const Rows &R, int nb, int with_delta,
                                          double dx[4], double dy[4], double qmax[4],
                                          double qmin[4], double &min_delt) {
    const int me = R.self();
    const double2 pi_ = R.xy(me);
    double qi[4];
    R.qrow(me, qi);
#pragma unroll
    for (int m = 0; m < 4; ++m) qmax[m] = qmin[m] = qi[m];
    double sdx2 = 0.0, sdy2 = 0.0, sdxy = 0.0;
    double sdxq[4] = {0.0, 0.0, 0.0, 0.0}, sdyq[4] = {0.0, 0.0, 0.0, 0.0};
    min_delt = 1.0;
    for (int r = 0; r < nb; ++r) {
        const int k = R.nbr(r);
        double qk[4];
        R.qrow(k, qk);
        const double2 pk = R.xy(k);
#pragma unroll
        for (int mm = 0; mm < 4; ++mm) {
            if (qk[mm] > qmax[mm]) qmax[mm] = qk[mm];
            if (qk[mm] < qmin[mm]) qmin[mm] = qk[mm];
        }
        double delx = pk.x - pi_.x, dely = pk.y - pi_.y;
        double dist = sqrt(delx * delx + dely * dely);
        double w = c.power_zero ? 1.0 : pow(dist, c.power);
        sdx2 = sdx2 + delx * delx * w;
        sdy2 = sdy2 + dely * dely * w;
        sdxy = sdxy + delx * dely * w;
#pragma unroll
        for (int mm = 0; mm < 4; ++mm) {
            sdxq[mm] = sdxq[mm] + w * delx * (qk[mm] - qi[mm]);
            sdyq[mm] = sdyq[mm] + w * dely * (qk[mm] - qi[mm]);
        }
        if (with_delta) {
            double delta_t = dist / R.spdv(k);
            delta_t = c.cfl * delta_t;
            if (min_delt > delta_t) min_delt = delta_t;
        }
    }
    double det = sdx2 * sdy2 - sdxy * sdxy;
    double one_by_det = 1.0 / det;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        dx[m] = (sdxq[m] * sdy2 - sdyq[m] * sdxy) * one_by_det;
        dy[m] = (sdyq[m] * sdx2 - sdxq[m] * sdxy) * one_by_det;
    }
}

// q_variables.F90:115-227 eval_q_inner_loop + eval_update_innerloop over the
// rows of R, rearranged.  q is fixed within a stage, so the reference's
// L sum_k w d (qtilde_k - qtilde_i), with qtilde = q - d.dq/2 and L the
// inverse of the stencil's normal matrix M = sum_k w d d^T, equals
//     dq0 + dq_i / 2 - L sum_k w d (d . dq_k) / 2,
// dq0 = L sum_k w d (q_k - q_i) being the D pass's result (kept through the
// stage's inner iterations) and L M dq_i = dq_i: the same value up to
// rounding, from the neighbours' dq and (x, y) alone (no q gathers).  dq0x,
// dq0y: the point's D-pass derivatives; the point's own dq_i and the
// neighbours' come through R.
template <class Rows>
__device__ __forceinline__ void inner_sums(const Consts &c, const Rows &R, int nb,
                                           const double dq0x[4], const double dq0y[4],
                                           double dx[4], double dy[4]) {
    const int me = R.self();
    const double2 pi_ = R.xy(me);
    double sdx2 = 0.0, sdy2 = 0.0, sdxy = 0.0;
    double sA[4] = {0.0, 0.0, 0.0, 0.0}, sB[4] = {0.0, 0.0, 0.0, 0.0};
    for (int r = 0; r < nb; ++r) {
        const int k = R.nbr(r);
        double dxk[4], dyk[4];
        R.dqrow(k, dxk, dyk);
        const double2 pk = R.xy(k);
        double delx = pk.x - pi_.x, dely = pk.y - pi_.y;
        double w = 1.0;
        if (!c.power_zero) w = pow(sqrt(delx * delx + dely * dely), c.power);
        sdx2 = sdx2 + delx * delx * w;
        sdy2 = sdy2 + dely * dely * w;
        sdxy = sdxy + delx * dely * w;
        const double wx = w * delx, wy = w * dely;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const double t = delx * dxk[m] + dely * dyk[m];
            sA[m] = sA[m] + wx * t;
            sB[m] = sB[m] + wy * t;
        }
    }
    double dxi[4], dyi[4];
    R.dqrow(me, dxi, dyi);
    double det = sdx2 * sdy2 - sdxy * sdxy;
    double one_by_det = 1.0 / det;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        const double Lx = one_by_det * (sA[m] * sdy2 - sB[m] * sdxy);
        const double Ly = one_by_det * (sB[m] * sdx2 - sA[m] * sdxy);
        dx[m] = (dq0x[m] + 0.5 * dxi[m]) - 0.5 * Lx;
        dy[m] = (dq0y[m] + 0.5 * dyi[m]) - 0.5 * Ly;
    }
}

// 64-byte rows in two 256-bit stores (st.global.v4.f64, sm_100): a warp's
// store of 32 rows touches each 128-byte line once per store instead of
// once per 16-byte piece.
__device__ __forceinline__ void st8w(double *p, const double a[4], const double b[4]) {
    asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(a[0]), "d"(a[1]),
                 "d"(a[2]), "d"(a[3]) : "memory");
    asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p + 4), "d"(b[0]), "d"(b[1]),
                 "d"(b[2]), "d"(b[3]) : "memory");
}

// Copies the halo rows of a warp's two tiles (hrow ranges [h0, h0 + hn0) and
// [h1, h1 + hn1), row u of the pair being row u of the first tile's halo or
// row u - hn0 of the second's) into their shared-memory arrays sm0 / sm1.
// Consecutive lanes copy consecutive 16-byte pieces of a row array -- the
// pieces of one row, then those of the next row in the halo's ascending
// order -- so that runs of neighbouring rows come in whole 128-byte lines.
// Lane l first loads the row indices of pair rows l, l + 32, l + 64 and
// l + 96; a copy takes its row index from the lane holding it (a shuffle
// whose source register is the same for the whole warp).  nA = HA_I copies
// q, (x, y) and dq; nA = HA_D copies q, (x, y) and, with spd != nullptr, spd.
// Stages a chunk's halo rows: the D pass q (two pieces a row), (x, y) and,
// with spd != nullptr, spd; the I pass (x, y) and dq (four pieces a row).
template <int nA>
__device__ __forceinline__ void stage_halo(const Geom &g, const R4 *q, const double *dq,
                                           const double *spd, const HaloIdx &x, int lane,
                                           double2 *sm0, double2 *sm1) {
    using H = HaloRows<nA>;
    if (nA == HA_D) stage_array<2>(q, 32, x, lane, sm0, sm1, g.hc, 0);
    stage_array<1>(g.xy, 16, x, lane, sm0, sm1, g.hc, H::OXY);
    if (nA == HA_I) stage_array<4>(dq, 64, x, lane, sm0, sm1, g.hc, H::ODQ);
    else if (spd) stage_array8(spd, x, lane, sm0, sm1, g.hc, H::OSPD);
}

// The D and I passes with tile halos (halo.cuh): a warp stages two tiles'
// halo rows, waits, and computes one point per lane from shared memory; a
// tile whose halo was too large to stage reads its rows directly.  No block
// barrier but the schedule load; the lanes of a warp meet at __syncwarp
// before the rows are read and before they are overwritten.
__global__ void __launch_bounds__(HALO_BLOCK, HALO_MIN_BLOCKS_I)
kb_inner_h(Geom g, Consts c, Sched s, const double *__restrict__ dq0,
           const double *__restrict__ dq_in, double *__restrict__ dq_out) {
    extern __shared__ double2 hsm[];
    __shared__ SchedSmem ss;
    load_sched(s, ss);
    const int ntiles = ss.pre[ss.nact];
    const int wpb = blockDim.x / 32, warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int half = lane / TILE, stride = gridDim.x * wpb;
    double2 *sm0 = hsm + (size_t)(2 * warp) * HA_I * g.hc, *sm1 = sm0 + HA_I * g.hc;
    HaloChunk cur;
    for (int ch = blockIdx.x * wpb + warp; 2 * ch < ntiles; ch += stride) {
        halo_chunk(g, s, ss, ntiles, ch, lane, cur);
        stage_halo<HA_I>(g, nullptr, dq_in, nullptr, cur.x, lane, sm0, sm1);
        const HaloRows<HA_I> hr(g, half ? sm1 : sm0, cur.hn > 0 ? cur.i : -1);
        double ax[4], ay[4];
        if (cur.i >= 0) ld8w(dq0 + 8 * (size_t)cur.i, ax, ay);
        halo_wait();
        __syncwarp();
        if (cur.i >= 0) {
            double dx[4], dy[4];
            if (cur.hn > 0) inner_sums(c, hr, cur.nb, ax, ay, dx, dy);
            else
                inner_sums(c, GlobalRows{g, nullptr, dq_in, nullptr, cur.i}, cur.nb, ax, ay, dx,
                           dy);
            st8w(dq_out + 8 * (size_t)cur.i, dx, dy);
        }
        __syncwarp();
    }
}

__global__ void __launch_bounds__(HALO_BLOCK, HALO_MIN_BLOCKS_D)
kb_grad_h(Geom g, Consts c, Sched s, const R4 *__restrict__ q, const double *__restrict__ spd,
          double *__restrict__ dq, double *__restrict__ qm, double *__restrict__ delta,
          int with_delta) {
    extern __shared__ double2 hsm[];
    __shared__ SchedSmem ss;
    load_sched(s, ss);
    const int ntiles = ss.pre[ss.nact];
    const int wpb = blockDim.x / 32, warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int half = lane / TILE, stride = gridDim.x * wpb;
    double2 *sm0 = hsm + (size_t)(2 * warp) * HA_D * g.hc, *sm1 = sm0 + HA_D * g.hc;
    HaloChunk cur;
    for (int ch = blockIdx.x * wpb + warp; 2 * ch < ntiles; ch += stride) {
        halo_chunk(g, s, ss, ntiles, ch, lane, cur);
        stage_halo<HA_D>(g, q, nullptr, with_delta ? spd : nullptr, cur.x, lane, sm0, sm1);
        const HaloRows<HA_D> hr(g, half ? sm1 : sm0, cur.hn > 0 ? cur.i : -1);
        halo_wait();
        __syncwarp();
        if (cur.i >= 0) {
            double dx[4], dy[4], qmax[4], qmin[4], min_delt;
            if (cur.hn > 0) grad_sums(c, hr, cur.nb, with_delta, dx, dy, qmax, qmin, min_delt);
            else
                grad_sums(c, GlobalRows{g, q, nullptr, spd, cur.i}, cur.nb, with_delta, dx, dy,
                          qmax, qmin, min_delt);
            st8w(dq + 8 * (size_t)cur.i, dx, dy);
            st8w(qm + 8 * (size_t)cur.i, qmax, qmin);
            if (with_delta) delta[cur.i] = min_delt;
        }
        __syncwarp();
    }
}

// flux_residual.F90:14-73 cal_flux_residual + state_update.F90:10-141 +
// q_variables.F90:8-37 on the new state.
//
// Work split: a warp owns CHUNK = 32 consecutive points (two tiles) end to
// end, with no block barrier.  It computes their list derivatives in rounds
// of PPW = 4 points, eight lanes per point (flux_group), leaving each point's
// sixteen list derivatives in the warp's shared memory, then updates the 32
// points with one lane each (update_point) and writes the two tiles'
// residual partials.
//
// In flux_group lane l of a point takes stencil slots l, l+8, l+16.  For its
// neighbour k it reconstructs both states once (limiter + qtilde -> kinetic
// state, reconstruct_kstate; the reference repeats this per direction list
// with identical inputs, so sharing it is exact), evaluates the split fluxes
// of every list the neighbour belongs to, and stores G_k - G_i with the
// geometry in a record.  Lane pair (2L, 2L+1) then sums list L in slot order
// -- the reference's loop order -- for components (0,1) and (2,3).  Slots
// are taken eight at a time: the records of one round of slots are summed
// before the next round overwrites them, the running sums waiting in shared
// memory between rounds, so shared memory does not grow with the stencil.
constexpr int PPW = 32 / LPP;          // points per warp round
constexpr int CHUNK = 2 * TILE;        // points a warp owns (two tiles)
constexpr int GST = 17;                // stride of a point's list derivatives (odd: no bank conflicts)
constexpr int FLUX_WARPS = FLUX_BLOCK / 32;
// doubles per warp: per point of a round its records and its lanes' parked
// sums, then the chunk's list derivatives and residual terms
// (one double of padding puts the four point groups' records on different
// banks: at 208 doubles, a multiple of 128 bytes, the list-sum reads of the
// four groups met in the same banks; C2 0.587 -> 0.575 ms)
constexpr int GROUP_SMEM = LPP * REC + 7 * LPP + 1;
constexpr int WARP_SMEM = PPW * GROUP_SMEM + CHUNK * GST + CHUNK;

// TAPE: also write both reconstructed kinetic states of every slot to
// b.kstape (the adjoint's taped re-run; the primal runs TAPE = false).
template <bool TAPE>
__device__ __forceinline__ void
flux_group(const Geom &g, const Consts &c, const StageBufs &b, int i, bool valid, int kind0,
           double *rec, double *Gout) {
    const int lane = threadIdx.x % LPP;
    const double inv_gm1 = 1.0 / c.gm1, inv_sqrt_pi = 1.0 / sqrt(c.pi);

    int nb = 0, kind = KIND_INTERIOR;
    unsigned long long mx = 0, my = 0;
    double nx = 0.0, ny = 1.0;
    if (valid) {
        nb = g.nbhs[i];
        kind = kind0;
        mx = g.mx[i];
        my = g.my[i];
        const double2 nn = g.nrm[i];
        nx = nn.x;
        ny = nn.y;
    }
    // x-list flux signs: interior Gxp/Gxn; wall GxII/GxI (A2neg); outer
    // GxIII/GxIV (A2pos).  y lists: Gyp (+1) / Gyn (-1).
    const double s2q = kind == KIND_WALL ? -1.0 : 1.0;
    const int nbw = __reduce_max_sync(0xffffffffu, nb);  // slot rounds of the warp
    // list-sum role of this lane: list L, components c0, c0+1
    const int L = lane >> 1, c0 = (lane & 1) * 2;
    const bool used =
        valid && !((kind == KIND_WALL && L == 2) || (kind == KIND_OUTER && L == 3));
    double sdx2 = 0.0, sdy2 = 0.0, sdxy = 0.0;
    double fx0 = 0.0, fx1 = 0.0, fy0 = 0.0, fy1 = 0.0;
    double *park = rec + LPP * REC + 7 * lane;  // running sums across slot rounds
    for (int r0 = 0; r0 < nbw; r0 += LPP) {
        if (r0 > 0) {
            // stencils of more than eight slots: the sums wait in shared
            // memory while the next round's records are computed
            park[0] = sdx2; park[1] = sdy2; park[2] = sdxy;
            park[3] = fx0; park[4] = fx1; park[5] = fy0; park[6] = fy1;
        }
        const int r = r0 + lane;
        if (r < nb) {
            const int k = g.conn[r * g.n + i];
            const double2 pi_ = g.xy[i];
            const double2 pk = g.xy[k];
            const double delx = pk.x - pi_.x, dely = pk.y - pi_.y;
            // neighbour state first (its gathers are the long-latency loads),
            // then the point's own state, re-read per slot from L1 so nothing
            // but the neighbour's kinetic state stays live across the two
            KState sk, si;
            double uk[2], ui[2];
            {
                const R4 kv = ld4(b.q_in + k);
                const double qk[4] = {kv.a, kv.b, kv.c, kv.d};
                double dxk[4], dyk[4], qmaxk[4], qmink[4];
                ld8w(b.dq + 8 * (size_t)k, dxk, dyk);
                ld8w(b.qm + 8 * (size_t)k, qmaxk, qmink);
                sk = reconstruct_kstate(qk, dxk, dyk, qmaxk, qmink, g.eps2[k], delx, dely,
                                        inv_gm1, nx, ny, inv_sqrt_pi, TAPE ? uk : nullptr);
            }
            {
                const R4 qv = ld4(b.q_in + i);
                const double qi[4] = {qv.a, qv.b, qv.c, qv.d};
                double dxi[4], dyi[4], qmaxi[4], qmini[4];
                ld8w(b.dq + 8 * (size_t)i, dxi, dyi);
                ld8w(b.qm + 8 * (size_t)i, qmaxi, qmini);
                si = reconstruct_kstate(qi, dxi, dyi, qmaxi, qmini, g.eps2[i], delx, dely,
                                        inv_gm1, nx, ny, inv_sqrt_pi, TAPE ? ui : nullptr);
            }
            if (TAPE) {
                // per state rho, p/rho, B1, B2, e1, e2, u1, u2 (ut, un and
                // |u|^2 follow from u and the point's normal)
                const double v[KS_TAPE] = {si.rho, si.pbr, si.B1, si.B2, si.e1, si.e2, ui[0],
                                           ui[1],  sk.rho, sk.pbr, sk.B1, sk.B2, sk.e1, sk.e2,
                                           uk[0],  uk[1]};
                double2 *tp = reinterpret_cast<double2 *>(
                    b.kstape + ((size_t)i * g.kp + r) * KS_TAPE);
#pragma unroll
                for (int h = 0; h < KS_TAPE / 2; ++h) tp[h] = make_double2(v[2 * h], v[2 * h + 1]);
            }
            const double tx = ny, ty = -nx;
            const double dels = delx * tx + dely * ty;
            const double deln = delx * nx + dely * ny;
            double w = 1.0;
            if (!c.power_zero) w = pow(sqrt(dels * dels + deln * deln), c.power);
            double *e = rec + lane * REC;
            // Per direction the neighbour is in one list of the pair (in both
            // only when its projection is exactly 0): one evaluation with the
            // list's sign taken per lane keeps the warp converged where
            // neighbours fall in different lists of the pair.
            double Gi[4], Gk[4];
#pragma unroll
            for (int d = 0; d < 2; ++d) {
                const unsigned long long bits = d == 0 ? mx : my;
                const bool in0 = (bits >> r) & 1ull, in1 = (bits >> (r + 32)) & 1ull;
#pragma unroll
                for (int pass = 0; pass < 2; ++pass) {
                    // pass 0: the first list holding the neighbour; pass 1:
                    // the second list of a neighbour in both
                    if (pass == 0 ? !(in0 || in1) : !(in0 && in1)) continue;
                    const int Lx = 2 * d + ((pass == 1 || !in0) ? 1 : 0);
                    const double sg = (Lx & 1) ? -1.0 : 1.0;
                    if (d == 0) {
                        if (kind == KIND_INTERIOR) {
                            flux_gx(si, sg, Gi);
                            flux_gx(sk, sg, Gk);
                        } else {
                            flux_quad(si, sg, s2q, Gi);
                            flux_quad(sk, sg, s2q, Gk);
                        }
                    } else {
                        flux_gy(si, sg, Gi);
                        flux_gy(sk, sg, Gk);
                    }
#pragma unroll
                    for (int m = 0; m < 4; ++m) e[4 * Lx + m] = Gk[m] - Gi[m];
                }
            }
            e[16] = dels;
            e[17] = deln;
            e[18] = w;
        }
        __syncwarp();
        if (r0 > 0) {
            sdx2 = park[0]; sdy2 = park[1]; sdxy = park[2];
            fx0 = park[3]; fx1 = park[4]; fy0 = park[5]; fy1 = park[6];
        }
        // list sums of this round's slots, in slot order
        if (used) {
            // the list's slots of this round in slot order (lowest bit first):
            // a lane loops over its own members only
            const unsigned long long lbits = ((L < 2) ? mx : my) >> ((L & 1) ? 32 : 0);
            // (a point with fewer slots than r0 has none in this round)
            const int cnt = min(nb, r0 + LPP) - r0;
            unsigned rb = cnt > 0 ? (unsigned)(lbits >> r0) & ((1u << cnt) - 1u) : 0u;
            while (rb) {
                const int rr = r0 + __ffs(rb) - 1;
                rb &= rb - 1u;
                const double *e = rec + (rr - r0) * REC;
                double dels = e[16], deln = e[17], w = e[18];
                double dels_w = dels * w, deln_w = deln * w;
                sdx2 = sdx2 + dels * dels_w;
                sdy2 = sdy2 + deln * deln_w;
                sdxy = sdxy + dels * deln_w;
                double d0 = e[4 * L + c0], d1 = e[4 * L + c0 + 1];
                fx0 = fx0 + d0 * dels_w;
                fy0 = fy0 + d0 * deln_w;
                fx1 = fx1 + d1 * dels_w;
                fy1 = fy1 + d1 * deln_w;
            }
        }
        __syncwarp();  // the next round overwrites the records
    }
    double Gv0 = 0.0, Gv1 = 0.0;
    if (used) {
        double det = sdx2 * sdy2 - sdxy * sdxy;
        double one_by_det = 1.0 / det;
        if (L < 2) {
            Gv0 = (fx0 * sdy2 - fy0 * sdxy) * one_by_det;
            Gv1 = (fx1 * sdy2 - fy1 * sdxy) * one_by_det;
        } else {
            Gv0 = (fy0 * sdx2 - fx0 * sdxy) * one_by_det;
            Gv1 = (fy1 * sdx2 - fx1 * sdxy) * one_by_det;
        }
    }
    // lane 2L+h holds G[L][2h], G[L][2h+1]
    Gout[2 * lane] = Gv0;
    Gout[2 * lane + 1] = Gv1;
}

// state_update.F90:10-141 of one point from its four list derivatives
// Gs[4L+m]; returns its res_sqr term.
__device__ __forceinline__ double
update_point(const Geom &g, const Consts &c, const StageBufs &b, int rk, int last, int i,
             int kind, int orow, const double *Gs) {
    double G[4][4];
#pragma unroll
    for (int L = 0; L < 4; ++L)
#pragma unroll
        for (int m = 0; m < 4; ++m) G[L][m] = Gs[4 * L + m];
    const double2 nn = g.nrm[i];
    const double nx = nn.x, ny = nn.y;
    double res_sqr = 0.0;
    {
        const double delta = b.delta[i];
        double fr[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            if (kind == KIND_WALL) fr[m] = 2.0 * delta * (G[0][m] + G[1][m] + G[3][m]);
            else if (kind == KIND_OUTER) fr[m] = delta * (G[0][m] + G[1][m] + G[2][m]);
            else fr[m] = delta * (G[0][m] + G[1][m] + G[2][m] + G[3][m]);
        }
        if (b.flux_dbg) st4(reinterpret_cast<R4 *>(b.flux_dbg) + i, fr[0], fr[1], fr[2], fr[3]);
        R4 P = ld4(b.prim_in + i);
        double U[4], Uo[4] = {0.0, 0.0, 0.0, 0.0};
        if (kind == KIND_OUTER) {
            const double *inf = g.obc + 8 * (size_t)orow;
            conserved_ubar(P.a, P.b, P.c, P.d, nx, ny, inf, c.pi, c.gm1, U);
            if (rk == 3) {
                R4 O = ld4(b.prim_old + i);
                conserved_ubar(O.a, O.b, O.c, O.d, nx, ny, inf, c.pi, c.gm1, Uo);
            }
        } else {
            prim_to_conserved(P.a, P.b, P.c, P.d, nx, ny, U);
            if (rk == 3) {
                R4 O = ld4(b.prim_old + i);
                prim_to_conserved(O.a, O.b, O.c, O.d, nx, ny, Uo);
            }
        }
        double temp = U[0];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            if (rk != 3) U[m] = U[m] - (0.5 * c.euler * fr[m]);
            else U[m] = TBT * Uo[m] + OBT * (U[m] - 0.5 * fr[m]);
        }
        if (kind == KIND_WALL) U[2] = 0.0;
        double U2_rot = U[1], U3_rot = U[2];
        U[1] = U2_rot * ny + U3_rot * nx;
        U[2] = U3_rot * ny - U2_rot * nx;
        if (kind != KIND_OUTER) res_sqr = (U[0] - temp) * (U[0] - temp);
        double rho = U[0];
        temp = 1.0 / U[0];
        double u1 = U[1] * temp;
        double u2 = U[2] * temp;
        double pr = 0.4 * (U[3] - (0.5 * temp) * (U[1] * U[1] + U[2] * U[2]));
        st4(b.prim_out + i, rho, u1, u2, pr);
        double qn[4];
        q_from_prim(rho, u1, u2, pr, qn);
        st4(b.q_out + i, qn[0], qn[1], qn[2], qn[3]);
        if (last) b.spd[i] = sqrt(u1 * u1 + u2 * u2) + 3.0 * sqrt(pr / rho);
    }
    return res_sqr;
}

// F pass: each warp walks chunks of two scheduled tiles with a stride of all
// warps of the grid.  A tile never straddles two instances and its partial
// lands in slot (instance's first tile + tile number), summed over its 16
// points in point order, so an instance's residual sums do not depend on the
// other instances or on the launch shape.
template <bool TAPE>
__global__ void __launch_bounds__(FLUX_BLOCK, FLUX_MIN_BLOCKS)
kb_flux(Geom g, Consts c, Sched s, StageBufs b, int rk, int last) {
    __shared__ double sm[FLUX_WARPS * WARP_SMEM];
#ifdef FLUX_SCHED_GLOBAL
    // the schedule stays in global memory: 2 KB more shared memory per block
    // for the records (one more resident block per SM)
    const int ntiles = __ldg(s.pre + __ldg(s.nact));
#define FLUX_TILE(v) sched_tile_global(s, v)
#else
    __shared__ SchedSmem ss;
    load_sched(s, ss);  // the kernel's only block barrier
    const int ntiles = ss.pre[ss.nact];
#define FLUX_TILE(v) sched_tile(s, ss, v)
#endif
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    double *rec = sm + warp * WARP_SMEM;       // PPW groups of GROUP_SMEM
    double *wG = rec + PPW * GROUP_SMEM;       // CHUNK points x GST
    double *wres = wG + CHUNK * GST;           // CHUNK residual terms
    const int nchunks = (ntiles + 1) / 2;
    for (int ch = blockIdx.x * FLUX_WARPS + warp; ch < nchunks; ch += gridDim.x * FLUX_WARPS) {
        const bool has1 = 2 * ch + 1 < ntiles;
        for (int rnd = 0; rnd < CHUNK / PPW; ++rnd) {
            const int pj = rnd * PPW + lane / LPP;  // point of the chunk
            const int v = 2 * ch + (pj < TILE ? 0 : 1);
            bool valid = false;
            int i = 0, kind = KIND_INTERIOR;
            if (v < ntiles) {
                const TileRef t = FLUX_TILE(v);
                const int j = t.j0 + (pj % TILE);
                valid = j < t.n;
                i = t.base + j;
                kind = j < t.nw ? KIND_WALL : (j < t.nw + t.no ? KIND_OUTER : KIND_INTERIOR);
            }
            flux_group<TAPE>(g, c, b, i, valid, kind, rec + (lane / LPP) * GROUP_SMEM,
                             wG + GST * pj);
        }
        __syncwarp();
        // the chunk's state updates, one point per lane
        const int v = 2 * ch + (lane < TILE ? 0 : 1);
        const TileRef t = FLUX_TILE(v < ntiles ? v : 2 * ch);
        const int j = t.j0 + (lane % TILE);
        const bool valid = v < ntiles && j < t.n;
        double rs = 0.0;
        if (valid) {
            const int kind = j < t.nw ? KIND_WALL : (j < t.nw + t.no ? KIND_OUTER : KIND_INTERIOR);
            rs = update_point(g, c, b, rk, last, t.base + j, kind, t.obc_off + j - t.nw,
                              wG + GST * lane);
        }
        if (last) {
            wres[lane] = rs;
            __syncwarp();
            if ((lane % TILE) == 0 && (lane < TILE || has1)) {
                double acc = 0.0;
                for (int q = 0; q < TILE; ++q) acc = acc + wres[lane + q];
                b.res_part[t.tile] = acc;
            }
        }
        __syncwarp();  // the next chunk reuses wG and wres
    }
#undef FLUX_TILE
}

// Sum of nparts tile partials in a fixed order (deterministic, independent
// of the launch shape of the passes that wrote them): thread t of a block of
// 1024 keeps eight accumulators over partials t + 1024 j (j mod 8 picks the
// accumulator, so the loads of one thread are independent), adds them
// pairwise, and a tree over the block adds the threads.  The result is in
// s[0] for every thread.
__device__ __forceinline__ void sum_parts_block(const double *__restrict__ part, int nparts,
                                                double *s) {
    constexpr int U = 8;
    const int T = blockDim.x;
    double acc[U] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    int t = threadIdx.x;
    for (; t + (U - 1) * T < nparts; t += U * T) {
#pragma unroll
        for (int j = 0; j < U; ++j) acc[j] = acc[j] + __ldg(part + t + j * T);
    }
#pragma unroll
    for (int j = 0; j < U; ++j)
        if (t + j * T < nparts) acc[j] = acc[j] + __ldg(part + t + j * T);
    s[threadIdx.x] = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) s[threadIdx.x] = s[threadIdx.x] + s[threadIdx.x + w];
        __syncthreads();
    }
}

// fpi_solver.F90:57-70: res_new = sqrt(sum res_sqr)/plen and the residue.
// Whole block of 1024 threads; the residue is returned on thread 0.
__device__ __forceinline__ double residual_block(const double *__restrict__ part, int nparts,
                                                 Ctl *ctl, double *hist, double *s) {
    sum_parts_block(part, nparts, s);
    if (threadIdx.x == 0) {
        double res_new = sqrt(s[0]) / ctl->plen;
        int it = ctl->it;
        double residue;
        if (it <= 2 && ctl->restart == 0) {
            ctl->res_old = res_new;
            residue = 0.0;
        } else {
            residue = log10(res_new / ctl->res_old);
        }
        hist[it - ctl->it_first] = residue;
        ctl->it = it + 1;
        ctl->done = ctl->done + 1;
        if (isnan(residue)) ctl->halted = 1;
        return residue;
    }
    return 0.0;
}

// Sum of nparts tile partials in the fixed order of residual_block (one
// block of 1024 threads): a partitioned grid's share of the residual, which
// the host adds over the ranks before the norm.
__global__ void __launch_bounds__(1024)
k_sum_parts(const double *__restrict__ part, int nparts, double *out) {
    __shared__ double s[1024];
    sum_parts_block(part, nparts, s);
    if (threadIdx.x == 0) *out = s[0];
}

// Per-instance residual (block b = instance b): the instance's tile partials
// are reduced in the order of residual_block, then the retirement rule of the
// run is applied (NaN residue, residue <= tol, max_iters iterations).  The
// last block to finish (threadfence + ticket, no waiting) rebuilds the
// schedule from Ctl::active for the next iteration's passes: a stable
// compaction of the running instances and the prefix sums of their tile
// counts (Hillis-Steele scans over MAX_BATCH slots).
__global__ void __launch_bounds__(1024)
kb_residual(const InstInfo *__restrict__ inst, int n_inst, const double *__restrict__ part,
            Ctl *ctl, double *hist, int hist_ld, const BatchRun *__restrict__ run,
            int *sched) {
    __shared__ double s[1024];
    __shared__ int s_active, s_last;
    __shared__ int cnt[MAX_BATCH], til[MAX_BATCH];
    Ctl *c = ctl + blockIdx.x;
    if (threadIdx.x == 0) s_active = c->active;
    __syncthreads();
    if (s_active) {
        const InstInfo in = inst[blockIdx.x];
        const double residue =
            residual_block(part + in.tile0, in.ntiles, c, hist + (size_t)blockIdx.x * hist_ld, s);
        if (threadIdx.x == 0) {
            if (isnan(residue)) {
                c->active = 0;
                c->state = BATCH_NONFINITE;
            } else if (residue <= run->tol) {
                c->active = 0;
                c->state = BATCH_CONVERGED;
            } else if (c->done >= run->max_iters) {
                c->active = 0;
                c->state = BATCH_MAX_ITERS;
            }
        }
    }
    int *counter = sched + SCHED_COUNTER;
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(counter, 1) == (int)gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const int t = threadIdx.x;
    int a = 0, nt = 0;
    if (t < MAX_BATCH) {
        a = (t < n_inst && reinterpret_cast<volatile const int *>(&ctl[t].active)[0]) ? 1 : 0;
        nt = a ? inst[t].ntiles : 0;
        cnt[t] = a;
        til[t] = nt;
    }
    __syncthreads();
    for (int off = 1; off < MAX_BATCH; off <<= 1) {
        int x = 0, y = 0;
        if (t < MAX_BATCH && t >= off) {
            x = cnt[t - off];
            y = til[t - off];
        }
        __syncthreads();
        if (t < MAX_BATCH) {
            cnt[t] += x;
            til[t] += y;
        }
        __syncthreads();
    }
    int *pre = sched + SCHED_PRE, *act = sched + SCHED_ACT;
    if (a) {
        act[cnt[t] - 1] = t;
        pre[cnt[t] - 1] = til[t] - nt;
    }
    if (t == MAX_BATCH - 1) {
        sched[SCHED_NACT] = cnt[t];
        pre[cnt[t]] = til[t];
        *counter = 0;
    }
}

// q and spd of rows [i0, i1) from their prim (set_state: every row; a
// partitioned grid: the ghost rows after their exchange)
__global__ void k_init_state(Geom g, const R4 *__restrict__ prim, R4 *__restrict__ q,
                             double *__restrict__ spd, int i0, int i1) {
    int i = i0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= i1) return;
    R4 P = ld4(prim + i);
    double qn[4];
    q_from_prim(P.a, P.b, P.c, P.d, qn);
    st4(q + i, qn[0], qn[1], qn[2], qn[3]);
    spd[i] = sqrt(P.b * P.b + P.c * P.c) + 3.0 * sqrt(P.d / P.a);
}

// compute_force_coeffs.F90:11-102, one thread, shape points in grid order.
// One block of FORCE_BLOCK threads: per chunk of FORCE_BLOCK shape points the
// threads form cp and the point's three terms in parallel, then thread 0
// adds them to its shape's sums in point order (the reference's loop order),
// so the sums do not depend on the launch.
constexpr int FORCE_BLOCK = 1024;

__global__ void __launch_bounds__(FORCE_BLOCK)
k_forces(ShapeTab t, const R4 *__restrict__ prim, double mach, double cos_t, double sin_t,
         double *out) {
    __shared__ double th[FORCE_BLOCK], tv[FORCE_BLOCK], tm[FORCE_BLOCK];
    __shared__ int ts[FORCE_BLOCK];
    const double rho_inf = 1.0, pr_inf = 1.0 / 1.4;
    double *H = out, *V = out + t.shapes, *PM = out + 2 * t.shapes;
    double *cp_out = out + 3 * t.shapes;
    if (threadIdx.x == 0)
        for (int s = 0; s < t.shapes; ++s) H[s] = V[s] = PM[s] = 0.0;
    const double temp = 0.5 * rho_inf * mach * mach;
    for (int j0 = 0; j0 < t.npts; j0 += FORCE_BLOCK) {
        const int j = j0 + threadIdx.x;
        if (j < t.npts) {
            const int m = t.idx[j];
            const double nx = t.geo[4 * j], ny = t.geo[4 * j + 1], ds = t.geo[4 * j + 2];
            const double mx = t.geo[4 * j + 3], my = t.my[j];
            double cp = prim[m].d - pr_inf;
            cp = -cp / temp;
            cp_out[j] = cp;
            th[threadIdx.x] = cp * nx * ds;
            tv[threadIdx.x] = cp * ny * ds;
            tm[threadIdx.x] = -cp * ny * ds * (mx - 0.25) + cp * nx * ds * (my);
            ts[threadIdx.x] = t.shape[j];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const int nj = min(FORCE_BLOCK, t.npts - j0);
            for (int q = 0; q < nj; ++q) {
                const int s = ts[q];
                H[s] = H[s] + th[q];
                V[s] = V[s] + tv[q];
                PM[s] = PM[s] + tm[q];
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int s = 0; s < t.shapes; ++s) {
            double h = H[s], v = V[s];
            H[s] = v * cos_t - h * sin_t;  // Cl
            V[s] = h * cos_t + v * sin_t;  // Cd
        }
}

inline int nblk(int n, int b) { return (n + b - 1) / b; }

}  // namespace

int flux_blocks(int n) { return nblk(n, TILE); }
// blocks that give every warp of the flux pass one chunk of two tiles
int flux_grid_blocks(int n) { return nblk(nblk(n, TILE), 2 * FLUX_WARPS); }

// staging memory of a block of the halo kernels: two tiles a warp
size_t halo_smem_bytes(int kind, int hc) {
    return halo_bytes(HALO_BLOCK / 32, kind == 0 ? HA_D : HA_I, hc);
}

cudaError_t init_kernels() {
    cudaError_t e = cudaFuncSetAttribute(kb_grad_h, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)halo_smem_bytes(0, HALO_CAP + 1));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kb_inner_h, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)halo_smem_bytes(1, HALO_CAP + 1));
    return e;
}

int wave_blocks(int dev, int kind, int block, size_t smem, bool fp32) {
    // the D and I passes: their own staging memory (the halo kernels' at the
    // largest stride; the FP32 I pass none)
    if (kind == 0 || kind == 1) smem = 0;
    int sms = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return std::max(sms, 1) * std::max(1, batch_occupancy(kind, fp32, block, smem));
}

namespace {
// grid of a launch: `grid` blocks, or one wave of resident blocks (grid == 0)
int wave(int kind, int block, size_t smem, int grid) {
    if (grid > 0) return grid;
    int dev = 0;
    cudaGetDevice(&dev);
    return wave_blocks(dev, kind, block, smem, false);
}
}  // namespace

// the flux pass's shared memory is static (independent of the stencil size)
size_t flux_smem_bytes(int) { return 0; }

int batch_occupancy(int kind, bool fp32, int block, size_t smem) {
    if (fp32) return batch_occupancy32(kind, block, smem);
    int nb = 0;
    cudaError_t e = cudaErrorInvalidValue;
    // the D and I passes: their tile-halo kernels (blocks of HALO_BLOCK
    // threads, the largest staging stride), which every grid with halos runs
    if (kind == 0)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kb_grad_h, HALO_BLOCK,
                                                          halo_smem_bytes(0, HALO_CAP + 1));
    else if (kind == 1)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kb_inner_h, HALO_BLOCK,
                                                          halo_smem_bytes(1, HALO_CAP + 1));
    else e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kb_flux<false>, block, smem);
    return e == cudaSuccess ? nb : 1;
}

// one wave of resident blocks of a halo kernel (kind 0: D pass, 1: I pass)
int halo_wave(int kind, int hc) {
    int dev = 0, sms = 1, nb = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t smem = halo_smem_bytes(kind, hc);
    cudaError_t e = kind == 0
        ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kb_grad_h, HALO_BLOCK, smem)
        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kb_inner_h, HALO_BLOCK, smem);
    return std::max(sms, 1) * std::max(1, e == cudaSuccess ? nb : 1);
}

void launch_grad(const Geom &g, const Consts &c, const Sched &s, const R4 *q, const double *spd,
                 double *dq, double *qm, double *delta, bool with_delta, int block, int grid,
                 cudaStream_t st) {
    (void)block;  // the halo kernels' blocks are HALO_BLOCK threads
    kb_grad_h<<<grid > 0 ? grid : halo_wave(0, g.hc), HALO_BLOCK, halo_smem_bytes(0, g.hc), st>>>(
        g, c, s, q, spd, dq, qm, delta, with_delta ? 1 : 0);
}

void launch_inner(const Geom &g, const Consts &c, const Sched &s, const double *dq0,
                  const double *dq_in, double *dq_out, int block, int grid, cudaStream_t st) {
    (void)block;
    kb_inner_h<<<grid > 0 ? grid : halo_wave(1, g.hc), HALO_BLOCK, halo_smem_bytes(1, g.hc), st>>>(
        g, c, s, dq0, dq_in, dq_out);
}

void launch_flux(const Geom &g, const Consts &c, const Sched &s, const StageBufs &b, int rk,
                 bool last, int grid, cudaStream_t st) {
    const int gr = wave(2, FLUX_BLOCK, 0, grid);
    if (b.kstape) kb_flux<true><<<gr, FLUX_BLOCK, 0, st>>>(g, c, s, b, rk, last ? 1 : 0);
    else kb_flux<false><<<gr, FLUX_BLOCK, 0, st>>>(g, c, s, b, rk, last ? 1 : 0);
}

void launch_residual(const InstInfo *inst, int n_inst, const double *res_part, Ctl *ctl,
                     double *hist, int hist_ld, const BatchRun *run, int *sched,
                     cudaStream_t st) {
    kb_residual<<<n_inst, 1024, 0, st>>>(inst, n_inst, res_part, ctl, hist, hist_ld, run, sched);
}

void launch_init_state(const Geom &g, const R4 *prim, R4 *q, double *spd, cudaStream_t s) {
    k_init_state<<<nblk(g.n, GRAD_BLOCK), GRAD_BLOCK, 0, s>>>(g, prim, q, spd, 0, g.n);
}

void launch_init_rows(const Geom &g, const R4 *prim, R4 *q, double *spd, int i0, int i1,
                      cudaStream_t s) {
    if (i1 > i0)
        k_init_state<<<nblk(i1 - i0, GRAD_BLOCK), GRAD_BLOCK, 0, s>>>(g, prim, q, spd, i0, i1);
}

void launch_sum_parts(const double *part, int nparts, double *out, cudaStream_t s) {
    k_sum_parts<<<1, 1024, 0, s>>>(part, nparts, out);
}

void launch_forces(const ShapeTab &t, const R4 *prim, double mach, double cos_t, double sin_t,
                   double *out, cudaStream_t s) {
    k_forces<<<1, FORCE_BLOCK, 0, s>>>(t, prim, mach, cos_t, sin_t, out);
}

}  // namespace lskum
