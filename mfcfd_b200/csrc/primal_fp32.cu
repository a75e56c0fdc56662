// FP32-mixed kernels of the LSKUM pseudo-time loop on sm_100a.
//
// Stored per point in FP32: prim, q, dq, qm (half the FP64 gather traffic).
// Computed in FP32: the q-derivative sums of the D and I passes, the
// per-neighbour work of the flux pass -- limiter, qtilde -> primitive (log,
// exp), the Maxwellian moments (exp, erf, sqrt) and the split fluxes -- with
// the flux contributions summed by compensated (Kahan) FP32 addition in slot
// order.  The 2x2 least-squares normal matrices, ill-conditioned on
// stretched near-wall stencils, are pure geometry: they are formed and
// inverted once per grid in FP64 (Geom32) and only applied per iteration.
// The state update runs in FP32 too (the state is stored in FP32); kept in
// FP64: the local time step, the list derivatives and flux residual, the
// residual norm (from the FP64 increment) and the force coefficients.
#include <cuda_runtime.h>

#include <algorithm>

#include "batch.cuh"
#include "halo.cuh"
#include "primal.h"

namespace lskum {

namespace {

constexpr int GRAD_BLOCK = 256;
constexpr int LPP = 8;
constexpr int FLUX_BLOCK = 128;  // four independent warps
constexpr int FREC = 10;  // dGxp..dGyn as 16 floats, then each list's slot weight c_L (20 floats)
#ifndef FLUX32_MIN_BLOCKS
#define FLUX32_MIN_BLOCKS 7  // <= 72 registers (8 blocks: 64 registers with spills, 0.370 against 0.364 ms on C2)
#endif
constexpr double OBT = 1.0 / 3.0;
constexpr double TBT = 2.0 / 3.0;

// A 32-byte row (dq or qm of one point) in one 256-bit read-only load
// (ld.global.nc.v8.f32, sm_100); the rows are 32-byte aligned.
__device__ __forceinline__ void ldf8w(const float *p, float a[4], float b[4]) {
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(a[0]), "=f"(a[1]), "=f"(a[2]), "=f"(a[3]), "=f"(b[0]), "=f"(b[1]), "=f"(b[2]),
          "=f"(b[3])
        : "l"(p));
}

// A 32-byte row in one 256-bit store (st.global.v8.f32, sm_100).
__device__ __forceinline__ void stf8w(float *p, const float a[4], const float b[4]) {
    asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p),
                 "f"(a[0]), "f"(a[1]), "f"(a[2]), "f"(a[3]), "f"(b[0]), "f"(b[1]), "f"(b[2]),
                 "f"(b[3])
                 : "memory");
}

// eval_q_inner_loop + eval_update_innerloop (q_variables.F90:115-227) with
// FP32 sums, rearranged.  The reference's new derivative is
//   L sum_k w d (qt_k - qt_i),  qt = q - (d . dq)/2,  L = M^-1,  M = sum_k w d d^T
// (d = x_k - x_i).  q is fixed within a stage, so it splits into
//   dq0 + dq_i/2 - L sum_k w d (d . dq_k) / 2,
// where dq0 = L sum_k w d (q_k - q_i) is the D pass's result of this stage
// and L M = I turns the point's own term into dq_i/2.  Equal in exact
// arithmetic; only the neighbours' derivatives are gathered (no q).
__device__ __forceinline__ void
inner32_point(const Geom &g, const Geom32 &f, const float *__restrict__ dq0,
              const float *__restrict__ dq_in, float *__restrict__ dq_out, int i) {
    float tx[4] = {0.f, 0.f, 0.f, 0.f}, ty[4] = {0.f, 0.f, 0.f, 0.f};
    const int nb = g.nbhs[i];
    for (int r = 0; r < nb; ++r) {
        const int k = g.conn[r * g.n + i];
        const float2 d = __ldg(f.dxy + r * g.n + i);
        const float w = f.w ? __ldg(f.w + r * g.n + i) : 1.0f;
        float dxk[4], dyk[4];
        ldf8w(dq_in + 8 * (size_t)k, dxk, dyk);
        const float wdx = w * d.x, wdy = w * d.y;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const float pk = d.x * dxk[m] + d.y * dyk[m];
            tx[m] = tx[m] + wdx * pk;
            ty[m] = ty[m] + wdy * pk;
        }
    }
    float dxi[4], dyi[4], dx0[4], dy0[4];
    ldf8w(dq_in + 8 * (size_t)i, dxi, dyi);
    ldf8w(dq0 + 8 * (size_t)i, dx0, dy0);
    const float4 L = __ldg(f.lsq + i);
    float dx[4], dy[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        dx[m] = dx0[m] + 0.5f * dxi[m] - 0.5f * (L.x * tx[m] + L.y * ty[m]);
        dy[m] = dy0[m] + 0.5f * dyi[m] - 0.5f * (L.y * tx[m] + L.z * ty[m]);
    }
    stf8w(dq_out + 8 * (size_t)i, dx, dy);
}

__global__ void __launch_bounds__(GRAD_BLOCK)
kb_inner32(Geom g, Geom32 f, Sched s, const float *__restrict__ dq0,
           const float *__restrict__ dq_in, float *__restrict__ dq_out) {
    __shared__ SchedSmem ss;
    load_sched(s, ss);
    const int total = ss.pre[ss.nact] * TILE;
    for (int vp = blockIdx.x * blockDim.x + threadIdx.x; vp < total;
         vp += gridDim.x * blockDim.x) {
        const int i = sched_point(s, ss, vp);
        if (i >= 0) inner32_point(g, f, dq0, dq_in, dq_out, i);
    }
}

// The D pass with tile halos (halo.cuh).  The per-slot FP32 offsets come
// from the staged FP64 (x, y) rows, rounded as the host rounds the offsets
// it stores ((float)(x_k - x_i)), so the halo and the stored-offset forms
// see the same offsets.  Row sources: GlobalRows32 reads the stored offsets
// and the rows from global memory (tiles without a staged halo); HaloRows32
// reads the staged q (float4), (x, y) and spd.  (The I pass keeps its direct
// 256-bit gathers of the 32-byte dq rows: a halo I pass staging (x, y) and dq
// measured slower, 0.057 against 0.050 ms per C2 launch, and so did one
// staging only (x, y) and the row indices, 0.064 ms.)
constexpr int HALO32_BLOCK = 128;
constexpr int HA32 = 3;  // staged arrays
#ifndef HALO32_MIN_BLOCKS
#define HALO32_MIN_BLOCKS 8
#endif

struct GlobalRows32 {
    const Geom &g;
    const Geom32 &f;
    const float4 *q;
    const double *spd;
    int i;
    __device__ __forceinline__ void begin() {}
    __device__ __forceinline__ int self() const { return i; }
    __device__ __forceinline__ int nbr(int r) const { return g.conn[r * g.n + i]; }
    __device__ __forceinline__ float2 off(int r, int) const { return __ldg(f.dxy + r * g.n + i); }
    __device__ __forceinline__ float4 qrow(int k) const { return __ldg(q + k); }
    __device__ __forceinline__ double spdv(int k) const { return spd[k]; }
};

// staged arrays: q 0, (x, y) 1, spd 2
struct HaloRows32 {
    static constexpr int OQ = 0, OXY = 1, OSPD = 2;
    const double2 *sm;
    int hc;
    HaloLoc loc;
    double2 pi;
    __device__ __forceinline__ HaloRows32(const Geom &g, const double2 *sm_, int i)
        : sm(sm_), hc(g.hc), loc(g, i), pi(make_double2(0.0, 0.0)) {}
    __device__ __forceinline__ void begin() { pi = sm[OXY * hc + loc.own]; }
    __device__ __forceinline__ int self() const { return loc.own; }
    __device__ __forceinline__ int nbr(int r) const { return loc.slot(r); }
    __device__ __forceinline__ float2 off(int, int l) const {
        const double2 pk = sm[OXY * hc + l];
        return make_float2((float)(pk.x - pi.x), (float)(pk.y - pi.y));
    }
    __device__ __forceinline__ float4 qrow(int l) const {
        return *reinterpret_cast<const float4 *>(sm + OQ * hc + l);
    }
    __device__ __forceinline__ double spdv(int l) const { return sm[OSPD * hc + l].x; }
};

// grad32_point's sums over the rows of R (the same arithmetic)
template <class Rows>
__device__ __forceinline__ void grad32_sums(const Consts &c, const Geom32 &f, int n, Rows R,
                                            int nb, int with_delta, int i, float dx[4],
                                            float dy[4], float qmax[4], float qmin[4],
                                            double &min_delt) {
    R.begin();
    const float4 qv = R.qrow(R.self());
    const float qi[4] = {qv.x, qv.y, qv.z, qv.w};
#pragma unroll
    for (int m = 0; m < 4; ++m) qmax[m] = qmin[m] = qi[m];
    float sx[4] = {0.f, 0.f, 0.f, 0.f}, sy[4] = {0.f, 0.f, 0.f, 0.f};
    min_delt = 1.0;
    for (int r = 0; r < nb; ++r) {
        const int k = R.nbr(r);
        const float4 kv = R.qrow(k);
        const float2 gs = R.off(r, k);
        const float qk[4] = {kv.x, kv.y, kv.z, kv.w};
        const float w = f.w ? __ldg(f.w + r * n + i) : 1.0f;
#pragma unroll
        for (int mm = 0; mm < 4; ++mm) {
            if (qk[mm] > qmax[mm]) qmax[mm] = qk[mm];
            if (qk[mm] < qmin[mm]) qmin[mm] = qk[mm];
        }
        const float wdx = w * gs.x, wdy = w * gs.y;
#pragma unroll
        for (int mm = 0; mm < 4; ++mm) {
            const float dqm = qk[mm] - qi[mm];
            sx[mm] = sx[mm] + wdx * dqm;
            sy[mm] = sy[mm] + wdy * dqm;
        }
        if (with_delta) {
            const double dist = (double)sqrtf(gs.x * gs.x + gs.y * gs.y);
            double delta_t = dist / R.spdv(k);
            delta_t = c.cfl * delta_t;
            if (min_delt > delta_t) min_delt = delta_t;
        }
    }
    const float4 L = __ldg(f.lsq + i);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        dx[m] = L.x * sx[m] + L.y * sy[m];
        dy[m] = L.y * sx[m] + L.z * sy[m];
    }
}

__global__ void __launch_bounds__(HALO32_BLOCK, HALO32_MIN_BLOCKS)
kb_grad32_h(Geom g, Consts c, Geom32 f, Sched s, const float4 *__restrict__ q,
            const double *__restrict__ spd, float *__restrict__ dq, float *__restrict__ qm,
            double *__restrict__ delta, int with_delta) {
    extern __shared__ double2 hsm[];
    __shared__ SchedSmem ss;
    load_sched(s, ss);
    const int ntiles = ss.pre[ss.nact];
    const int wpb = blockDim.x / 32, warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int half = lane / TILE, stride = gridDim.x * wpb;
    using H = HaloRows32;
    double2 *sm0 = hsm + (size_t)(2 * warp) * HA32 * g.hc, *sm1 = sm0 + HA32 * g.hc;
    HaloChunk cur;
    for (int ch = blockIdx.x * wpb + warp; 2 * ch < ntiles; ch += stride) {
        halo_chunk(g, s, ss, ntiles, ch, lane, cur);
        stage_array<1>(q, 16, cur.x, lane, sm0, sm1, g.hc, H::OQ);
        stage_array<1>(g.xy, 16, cur.x, lane, sm0, sm1, g.hc, H::OXY);
        if (with_delta) stage_array8(spd, cur.x, lane, sm0, sm1, g.hc, H::OSPD);
        const H hr(g, half ? sm1 : sm0, cur.hn > 0 ? cur.i : -1);
        halo_wait();
        __syncwarp();
        if (cur.i >= 0) {
            float dx[4], dy[4], qmax[4], qmin[4];
            double min_delt;
            if (cur.hn > 0)
                grad32_sums(c, f, g.n, hr, cur.nb, with_delta, cur.i, dx, dy, qmax, qmin,
                            min_delt);
            else
                grad32_sums(c, f, g.n, GlobalRows32{g, f, q, spd, cur.i}, cur.nb,
                            with_delta, cur.i, dx, dy, qmax, qmin, min_delt);
            stf8w(dq + 8 * (size_t)cur.i, dx, dy);
            stf8w(qm + 8 * (size_t)cur.i, qmax, qmin);
            if (with_delta) delta[cur.i] = min_delt;
        }
        __syncwarp();
    }
}

// Compensated FP32 addition (Kahan): s += v with running correction cmp.
__device__ __forceinline__ void kahan_add(float &s, float &cmp, float v) {
    float y = __fsub_rn(v, cmp);
    float t = __fadd_rn(s, y);
    cmp = __fsub_rn(__fsub_rn(t, s), y);
    s = t;
}

// cal_flux_residual + state_update + eval_q_variables of the new state, with
// the per-neighbour work in FP32.  Work split as in the FP64 pass: a warp
// owns two tiles (32 points) end to end with no block barrier, computes
// their list derivatives in rounds of four points (eight lanes each, slots
// taken eight at a time with the lane pairs' Kahan sums parked in shared
// memory between slot rounds), then updates the 32 points one per lane.
#ifndef FLUX32_CT
#define FLUX32_CT 1  // tiles a warp owns: 1 (0.366 ms per C2 launch) or 2 (every lane updates a point; 0.375 ms)
#endif
// Arithmetic types of the flux pass: RT for the reconstruction to the
// kinetic state, FT for the split fluxes and their differences, UT for the
// state update.  The state is stored in FP32 throughout.  The update runs in
// FP64: its conversions prim -> U -> prim, four times an iteration, are what
// moved the FP32-mixed loop away from the FP64 loop (640x400 grid, 2,000
// iterations from freestream: |dCd| 1.1e-5 with an FP32 update, 2.2e-7 with
// an FP64 one, at 1.4 % of the pass's time), while FP64 reconstruction or
// fluxes changed nothing measurable (|dCd| 1.10-1.12e-5 with either).
#ifndef FLUX32_RT
#define FLUX32_RT float
#endif
#ifndef FLUX32_FT
#define FLUX32_FT float
#endif
#ifndef FLUX32_UT
#define FLUX32_UT double
#endif
using RT = FLUX32_RT;
using FT = FLUX32_FT;
using UT = FLUX32_UT;
template <class D, class S>
__device__ __forceinline__ KStateT<D> kcast(const KStateT<S> &s) {
    KStateT<D> d;
    d.rho = (D)s.rho; d.ut = (D)s.ut; d.un = (D)s.un; d.pbr = (D)s.pbr; d.usq = (D)s.usq;
    d.B1 = (D)s.B1; d.B2 = (D)s.B2; d.e1 = (D)s.e1; d.e2 = (D)s.e2;
    return d;
}
// the reconstructed kinetic state of point p along (dx, dy)
__device__ __forceinline__ KStateT<FT> kstate32(const StageBufs32 &b, int p, RT dx, RT dy, RT inv_gm1,
                                                RT nx, RT ny, RT inv_sqrt_pi) {
    const float4 v = __ldg(b.q_in + p);
    float dxf[4], dyf[4], qmaxf[4], qminf[4];
    ldf8w(b.dq + 8 * (size_t)p, dxf, dyf);
    ldf8w(b.qm + 8 * (size_t)p, qmaxf, qminf);
    const RT q[4] = {v.x, v.y, v.z, v.w};
    RT ddx[4], ddy[4], qmax[4], qmin[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        ddx[j] = dxf[j]; ddy[j] = dyf[j]; qmax[j] = qmaxf[j]; qmin[j] = qminf[j];
    }
    return kcast<FT>(reconstruct_kstate<RT>(q, ddx, ddy, qmax, qmin, (RT)b.eps2f[p], dx, dy,
                                            inv_gm1, nx, ny, inv_sqrt_pi));
}
constexpr int PPW = 32 / LPP;
constexpr int CT = FLUX32_CT;
constexpr int CHUNK = CT * TILE;
constexpr int GST = 17;                                  // odd: no bank conflicts
constexpr int FLUX_WARPS = FLUX_BLOCK / 32;
constexpr int GROUP_SMEM = LPP * FREC + 4 * LPP;         // records + parked sums (doubles)
constexpr int WARP_SMEM = PPW * GROUP_SMEM + CHUNK * GST + CHUNK;

__device__ __forceinline__ void
flux32_group(const Geom &g, const Consts &c, const StageBufs32 &b, int i, bool valid,
             int kind0, double *rec, double *Gout) {
    const int lane = threadIdx.x % LPP;
    int nb = 0, kind = KIND_INTERIOR;
    unsigned long long mx = 0, my = 0;
    RT nxf = 0, nyf = 1;
    if (valid) {
        nb = g.nbhs[i];
        kind = kind0;
        mx = g.mx[i];
        my = g.my[i];
        const double2 nn = g.nrm[i];
        nxf = (RT)nn.x;
        nyf = (RT)nn.y;
    }
    const RT inv_gm1 = (RT)(1.0 / c.gm1), inv_sqrt_pi = (RT)(1.0 / sqrt(c.pi));
    const FT s2q = kind == KIND_WALL ? FT(-1) : FT(1);
    const int nbw = __reduce_max_sync(0xffffffffu, nb);
    const int L = lane >> 1, c0 = (lane & 1) * 2;
    const bool used =
        valid && !((kind == KIND_WALL && L == 2) || (kind == KIND_OUTER && L == 3));
    // Kahan sums of the lane's two list components and their corrections
    float fx0 = 0.f, fx1 = 0.f, cx0 = 0.f, cx1 = 0.f;
    float *park = reinterpret_cast<float *>(rec + LPP * FREC) + 8 * lane;
    for (int r0 = 0; r0 < nbw; r0 += LPP) {
        if (r0 > 0) {
            park[0] = fx0; park[1] = fx1; park[2] = cx0; park[3] = cx1;
        }
        const int r = r0 + lane;
        if (r < nb) {
            const int k = g.conn[r * g.n + i];
            const float2 d = __ldg(b.f.dxy + r * g.n + i);
            const float dxf = d.x, dyf = d.y;
            const KStateT<FT> sk = kstate32(b, k, dxf, dyf, inv_gm1, nxf, nyf, inv_sqrt_pi);
            const KStateT<FT> si = kstate32(b, i, dxf, dyf, inv_gm1, nxf, nyf, inv_sqrt_pi);
            const float dels = dxf * nyf - dyf * nxf;
            const float deln = dxf * nxf + dyf * nyf;
            const float w = b.f.w ? __ldg(b.f.w + r * g.n + i) : 1.0f;
            float *ef = reinterpret_cast<float *>(rec + lane * FREC);
            FT Gi[4], Gk[4];
#pragma unroll
            for (int dd = 0; dd < 2; ++dd) {
                // one converged evaluation per direction, as in the FP64 pass
                const unsigned long long bits = dd == 0 ? mx : my;
                const bool in0 = (bits >> r) & 1ull, in1 = (bits >> (r + 32)) & 1ull;
#pragma unroll
                for (int pass = 0; pass < 2; ++pass) {
                    if (pass == 0 ? !(in0 || in1) : !(in0 && in1)) continue;
                    const int Lx = 2 * dd + ((pass == 1 || !in0) ? 1 : 0);
                    const FT sg = (Lx & 1) ? FT(-1) : FT(1);
                    if (dd == 0) {
                        if (kind == KIND_INTERIOR) {
                            flux_gx<FT>(si, sg, Gi);
                            flux_gx<FT>(sk, sg, Gk);
                        } else {
                            flux_quad<FT>(si, sg, s2q, Gi);
                            flux_quad<FT>(sk, sg, s2q, Gk);
                        }
                    } else {
                        flux_gy<FT>(si, sg, Gi);
                        flux_gy<FT>(sk, sg, Gk);
                    }
#pragma unroll
                    for (int m = 0; m < 4; ++m) ef[4 * Lx + m] = (float)(Gk[m] - Gi[m]);
                }
            }
            {
                // the list solves folded into the slot: list L's derivative is
                // sum_slots d * c_L with c_L = a_L dels w + b_L deln w (x lists)
                // or a_L deln w + b_L dels w (y lists)
                const float sw = dels * w, nw = deln * w;
                const float4 cx = __ldg(b.f.flsq + 2 * (size_t)i);
                const float4 cy = __ldg(b.f.flsq + 2 * (size_t)i + 1);
                ef[16] = cx.x * sw + cx.y * nw;
                ef[17] = cx.z * sw + cx.w * nw;
                ef[18] = cy.x * nw + cy.y * sw;
                ef[19] = cy.z * nw + cy.w * sw;
            }
        }
        __syncwarp();
        if (r0 > 0) {
            fx0 = park[0]; fx1 = park[1]; cx0 = park[2]; cx1 = park[3];
        }
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
                const float *ef = reinterpret_cast<const float *>(rec + (rr - r0) * FREC);
                const float d0 = ef[4 * L + c0], d1 = ef[4 * L + c0 + 1];
                const float cl = ef[16 + L];
                kahan_add(fx0, cx0, d0 * cl);
                kahan_add(fx1, cx1, d1 * cl);
            }
        }
        __syncwarp();  // the next round overwrites the records
    }
    double Gv0 = 0.0, Gv1 = 0.0;
    if (used) {
        Gv0 = (double)fx0 - cx0;
        Gv1 = (double)fx1 - cx1;
    }
    // lane 2L+h holds G[L][2h], G[L][2h+1]
    Gout[2 * lane] = Gv0;
    Gout[2 * lane + 1] = Gv1;
}

// state_update.F90:10-141 of one point from its four list derivatives
// Gs[4L+m]: FP32 state in and out, arithmetic in UT; returns its res_sqr
// term (FP64).
__device__ __forceinline__ double
update32_point(const Geom &g, const Consts &c, const StageBufs32 &b, int rk, int last, int i,
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
        // state_update in UT (the state is stored in FP32); the residual
        // from the increment itself, 0.5 euler fr(1), in FP64, which FP32
        // differences of U(1) would cancel (last stage: rk != 3)
        if (kind != KIND_OUTER) res_sqr = (0.5 * c.euler * fr[0]) * (0.5 * c.euler * fr[0]);
        const UT nxf = (UT)nx, nyf = (UT)ny, pif = (UT)c.pi, gm1f = (UT)c.gm1;
        UT frf[4] = {(UT)fr[0], (UT)fr[1], (UT)fr[2], (UT)fr[3]};
        const float4 P = b.prim_in[i];
        UT U[4], Uo[4] = {0, 0, 0, 0};
        if (kind == KIND_OUTER) {
            const double *inf = g.obc + 8 * (size_t)orow;
            const UT inff[5] = {(UT)inf[0], (UT)inf[1], (UT)inf[2], (UT)inf[3], (UT)inf[4]};
            conserved_ubar_t<UT>(P.x, P.y, P.z, P.w, nxf, nyf, inff, pif, gm1f, U);
            if (rk == 3) {
                const float4 O = b.prim_old[i];
                conserved_ubar_t<UT>(O.x, O.y, O.z, O.w, nxf, nyf, inff, pif, gm1f, Uo);
            }
        } else {
            prim_to_conserved_t<UT>(P.x, P.y, P.z, P.w, nxf, nyf, U);
            if (rk == 3) {
                const float4 O = b.prim_old[i];
                prim_to_conserved_t<UT>(O.x, O.y, O.z, O.w, nxf, nyf, Uo);
            }
        }
        const UT half_euler = (UT)(0.5 * c.euler);
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            if (rk != 3) U[m] = U[m] - half_euler * frf[m];
            else U[m] = (UT)TBT * Uo[m] + (UT)OBT * (U[m] - UT(0.5) * frf[m]);
        }
        if (kind == KIND_WALL) U[2] = 0;
        const UT U2_rot = U[1], U3_rot = U[2];
        U[1] = U2_rot * nyf + U3_rot * nxf;
        U[2] = U3_rot * nyf - U2_rot * nxf;
        const UT temp = UT(1) / U[0];
        const float rho = (float)U[0];
        const float u1 = (float)(U[1] * temp);
        const float u2 = (float)(U[2] * temp);
        const float pr = (float)(UT(0.4) * (U[3] - (UT(0.5) * temp) * (U[1] * U[1] + U[2] * U[2])));
        b.prim_out[i] = make_float4(rho, u1, u2, pr);
        float qn[4];
        q_from_prim_t<float>(rho, u1, u2, pr, qn);
        b.q_out[i] = make_float4(qn[0], qn[1], qn[2], qn[3]);
        if (last) b.spd[i] = (double)(sqrtf(u1 * u1 + u2 * u2) + 3.0f * sqrtf(pr / rho));
    }
    return res_sqr;
}

// Each warp walks chunks of two scheduled tiles with a stride of all warps of
// the grid; tile partials as in the FP64 pass.
__global__ void __launch_bounds__(FLUX_BLOCK, FLUX32_MIN_BLOCKS)
kb_flux32(Geom g, Consts c, Sched s, StageBufs32 b, int rk, int last) {
    __shared__ double sm[FLUX_WARPS * WARP_SMEM];
    __shared__ SchedSmem ss;
    load_sched(s, ss);  // the kernel's only block barrier
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    double *rec = sm + warp * WARP_SMEM;
    double *wG = rec + PPW * GROUP_SMEM;
    double *wres = wG + CHUNK * GST;
    const int ntiles = ss.pre[ss.nact];
    const int nchunks = (ntiles + CT - 1) / CT;
    for (int ch = blockIdx.x * FLUX_WARPS + warp; ch < nchunks; ch += gridDim.x * FLUX_WARPS) {
        for (int rnd = 0; rnd < CHUNK / PPW; ++rnd) {
            const int pj = rnd * PPW + lane / LPP;
            const int v = CT * ch + pj / TILE;
            bool valid = false;
            int i = 0, kind = KIND_INTERIOR;
            if (v < ntiles) {
                const TileRef t = sched_tile(s, ss, v);
                const int j = t.j0 + (pj % TILE);
                valid = j < t.n;
                i = t.base + j;
                kind = j < t.nw ? KIND_WALL : (j < t.nw + t.no ? KIND_OUTER : KIND_INTERIOR);
            }
            flux32_group(g, c, b, i, valid, kind, rec + (lane / LPP) * GROUP_SMEM, wG + GST * pj);
        }
        __syncwarp();
        const int v = CT * ch + lane / TILE;  // lanes past the chunk idle here
        const bool inchunk = lane < CHUNK && v < ntiles;
        const TileRef t = sched_tile(s, ss, inchunk ? v : CT * ch);
        const int j = t.j0 + (lane % TILE);
        const bool valid = inchunk && j < t.n;
        double rs = 0.0;
        if (valid) {
            const int kind = j < t.nw ? KIND_WALL : (j < t.nw + t.no ? KIND_OUTER : KIND_INTERIOR);
            rs = update32_point(g, c, b, rk, last, t.base + j, kind, t.obc_off + j - t.nw,
                                wG + GST * lane);
        }
        if (last) {
            if (lane < CHUNK) wres[lane] = rs;
            __syncwarp();
            if ((lane % TILE) == 0 && inchunk) {
                double acc = 0.0;
                for (int q = 0; q < TILE; ++q) acc = acc + wres[lane + q];
                b.res_part[t.tile] = acc;
            }
        }
        __syncwarp();  // the next chunk reuses wG and wres
    }
}

__global__ void k_init_state32(Geom g, const float4 *__restrict__ prim, float4 *__restrict__ q,
                               double *__restrict__ spd) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.n) return;
    float4 P = prim[i];
    double qn[4];
    q_from_prim((double)P.x, (double)P.y, (double)P.z, (double)P.w, qn);
    q[i] = make_float4((float)qn[0], (float)qn[1], (float)qn[2], (float)qn[3]);
    double u1 = P.y, u2 = P.z, rho = P.x, pr = P.w;
    spd[i] = sqrt(u1 * u1 + u2 * u2) + 3.0 * sqrt(pr / rho);
}

__global__ void k_widen(const float4 *__restrict__ in, R4 *__restrict__ out, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 v = in[i];
    st4(out + i, v.x, v.y, v.z, v.w);
}

inline int nblk(int n, int b) { return (n + b - 1) / b; }

}  // namespace


cudaError_t init_kernels32() {
    // the FP32 halo D pass stays below the default 48 KB of dynamic shared
    // memory (at most 25 KB); nothing to set
    return cudaSuccess;
}

namespace {
// dynamic shared memory of the halo kernels at staging stride hc
size_t halo32_smem(int hc) { return halo_bytes(HALO32_BLOCK / 32, HA32, hc); }
// one wave of resident blocks of a halo kernel (kind 0: D pass, 1: I pass)
int halo32_wave(int kind, int hc) {
    int dev = 0, sms = 1, nb = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    (void)kind;  // the D pass only
    cudaError_t e =
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kb_grad32_h, HALO32_BLOCK, halo32_smem(hc));
    return std::max(sms, 1) * std::max(1, e == cudaSuccess ? nb : 1);
}
}  // namespace

// the flux pass's shared memory is static (independent of the stencil size)
size_t flux32_smem_bytes(int) { return 0; }

int batch_occupancy32(int kind, int block, size_t smem) {
    int nb = 0;
    cudaError_t e = cudaErrorInvalidValue;
    // the D pass: its tile-halo kernel at the largest staging stride, which
    // every grid with halos runs
    if (kind == 0)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kb_grad32_h, HALO32_BLOCK,
                                                          halo32_smem(HALO_CAP + 1));
    else if (kind == 1)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kb_inner32, block, smem);
    else e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kb_flux32, block, smem);
    return e == cudaSuccess ? nb : 1;
}

namespace {
int wave32(int kind, int block, size_t smem, int grid) {
    if (grid > 0) return grid;
    int dev = 0;
    cudaGetDevice(&dev);
    return wave_blocks(dev, kind, block, smem, true);
}
}  // namespace

void launch_grad32(const Geom &g, const Consts &c, const Geom32 &f, const Sched &s,
                   const float4 *q, const double *spd, float *dq, float *qm, double *delta,
                   bool with_delta, int block, int grid, cudaStream_t st) {
    (void)block;  // the halo kernel's blocks are HALO32_BLOCK threads
    kb_grad32_h<<<grid > 0 ? grid : halo32_wave(0, g.hc), HALO32_BLOCK, halo32_smem(g.hc), st>>>(
        g, c, f, s, q, spd, dq, qm, delta, with_delta ? 1 : 0);
}

void launch_inner32(const Geom &g, const Consts &c, const Geom32 &f, const Sched &s,
                    const float *dq0, const float *dq_in, float *dq_out, int block, int grid,
                    cudaStream_t st) {
    (void)c;
    kb_inner32<<<wave32(1, block, 0, grid), block, 0, st>>>(g, f, s, dq0, dq_in, dq_out);
}

void launch_flux32(const Geom &g, const Consts &c, const Sched &s, const StageBufs32 &b,
                         int rk, bool last, int grid, cudaStream_t st) {
    kb_flux32<<<wave32(2, FLUX_BLOCK, 0, grid), FLUX_BLOCK, 0, st>>>(g, c, s, b, rk,
                                                                     last ? 1 : 0);
}

void launch_init_state32(const Geom &g, const float4 *prim, float4 *q, double *spd,
                         cudaStream_t s) {
    k_init_state32<<<nblk(g.n, GRAD_BLOCK), GRAD_BLOCK, 0, s>>>(g, prim, q, spd);
}

void launch_widen(const float4 *in, R4 *out, int n, cudaStream_t s) {
    k_widen<<<nblk(n, GRAD_BLOCK), GRAD_BLOCK, 0, s>>>(in, out, n);
}

}  // namespace lskum
