// Reverse (adjoint) kernels of the LSKUM pseudo-time loop, FP64.
//
// One pseudo-time stage reverses in the order
//   k_update_b   state_update_b      prim_out_b -> prim_in_b, prim_old_b, flux_res_b, n_b
//   k_flux_b     cal_flux_residual_b flux_res_b -> q_b, dq_b, qm_b, x_b, y_b, n_b, delta_b
//   k_inner_b    eval_q_inner_loop_b (per inner iteration, last first)
//   k_grad_b     eval_q_derivatives_b + func_delta_b (first stage)
//   k_qvar_b     eval_q_variables_b  q_b -> prim_in_b
// (the stage-by-stage order of the reference's FPI_SOLVER_B,
// src_mpi_adjoint/sensitivity_files/fpi_solver_b.F90:28-156).
//
// A point's adjoint flows to its neighbours, without atomics.  The q-
// derivative reverses write their contribution for neighbour slot r of
// point i into contrib[(i*kp + r)*CW + field] and k_gather adds them per
// neighbour in the fixed (i, r) order of the transposed stencil.  The flux
// reverse, whose neighbour side is most of the work, pulls instead:
// k_flux_b leaves a short record per slot and k_flux_b_nbr, one thread per
// neighbour, reverses the neighbour's reconstruction of each slot naming it
// in that same order.  Results are deterministic either way.
#include <cuda_runtime.h>

#include <algorithm>

#include "adjoint.h"
#include "lskum_adjoint.cuh"

namespace lskum {

namespace {

constexpr int BLK = 128;
constexpr int LPP = 8;
constexpr int GROUPS = BLK / LPP;
constexpr int BREC = 44;  // dG[16] dels deln si[9] sk[9] prim_i[4] prim_k[4]
constexpr double OBT = 1.0 / 3.0;
constexpr double TBT = 2.0 / 3.0;

__device__ __forceinline__ void ld8a(const double *p, double a[4], double b[4]) {
    const double2 *v = reinterpret_cast<const double2 *>(p);
    double2 t0 = v[0], t1 = v[1], t2 = v[2], t3 = v[3];
    a[0] = t0.x; a[1] = t0.y; a[2] = t1.x; a[3] = t1.y;
    b[0] = t2.x; b[1] = t2.y; b[2] = t3.x; b[3] = t3.y;
}

// Four doubles in one 256-bit read-only load (ld.global.nc.v4.f64, sm_100);
// p is 32-byte aligned and not written by the kernel that reads it.
__device__ __forceinline__ void ld4nc(const double *p, double v[4]) {
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
        : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3])
        : "l"(p));
}

__device__ __forceinline__ void kst_store(double *e, const KState &s) {
    e[0] = s.rho; e[1] = s.ut; e[2] = s.un; e[3] = s.pbr; e[4] = s.usq;
    e[5] = s.B1; e[6] = s.B2; e[7] = s.e1; e[8] = s.e2;
}
// A kinetic state from its tape entry (rho, p/rho, B1, B2, e1, e2, u1, u2)
// and the point's normal, as reconstruct_kstate forms ut, un and |u|^2.
__device__ __forceinline__ KState kst_taped(const double *v, double nx, double ny) {
    KState s;
    const double tx = ny, ty = -nx;
    s.rho = v[0];
    s.pbr = v[1];
    s.B1 = v[2];
    s.B2 = v[3];
    s.e1 = v[4];
    s.e2 = v[5];
    s.ut = v[6] * tx + v[7] * ty;
    s.un = v[6] * nx + v[7] * ny;
    s.usq = s.ut * s.ut + s.un * s.un;
    return s;
}
__device__ __forceinline__ KState kst_load(const double *e) {
    KState s;
    s.rho = e[0]; s.ut = e[1]; s.un = e[2]; s.pbr = e[3]; s.usq = e[4];
    s.B1 = e[5]; s.B2 = e[6]; s.e1 = e[7]; s.e2 = e[8];
    return s;
}

// state_update_b (state_update.F90:10-141, reverse)
// Stores n (even) doubles as 16-byte pairs; dst is 16-byte aligned (records
// are ADJ_CW = 22 doubles = 176 bytes from an aligned base).
__device__ __forceinline__ void st_pairs(double *dst, const double *v, int n) {
    double2 *d2 = reinterpret_cast<double2 *>(dst);
#pragma unroll
    for (int h = 0; h < n / 2; ++h) d2[h] = make_double2(v[2 * h], v[2 * h + 1]);
}

// dst[j] += v[j] for n (even) doubles, as 16-byte pairs (dst 16-byte aligned)
__device__ __forceinline__ void add_pairs(double *dst, const double *v, int n) {
    double2 *d2 = reinterpret_cast<double2 *>(dst);
#pragma unroll
    for (int h = 0; h < n / 2; ++h) {
        double2 t = d2[h];
        t.x = t.x + v[2 * h];
        t.y = t.y + v[2 * h + 1];
        d2[h] = t;
    }
}

#ifndef ADJ_MIN_BLOCKS
#define ADJ_MIN_BLOCKS 3
#endif
__global__ void __launch_bounds__(BLK, ADJ_MIN_BLOCKS)
k_update_b(Geom g, Consts c, AdjConsts a, const R4 *__restrict__ prim_in,
           const R4 *__restrict__ prim_old, const R4 *__restrict__ fr,
           const double *__restrict__ pb_out, double *__restrict__ pb_in,
           double *__restrict__ pb_old, double *__restrict__ frb, double *__restrict__ nxb,
           double *__restrict__ nyb, int rk) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.n) return;
    const int kind = i < g.nw ? KIND_WALL : (i < g.nw + g.no ? KIND_OUTER : KIND_INTERIOR);
    const double2 nn = g.nrm[i];
    const double nx = nn.x, ny = nn.y;
    const R4 P = ld4(prim_in + i);
    const R4 F = ld4(fr + i);
    const double frv[4] = {F.a, F.b, F.c, F.d};
    double U[4], Uo[4] = {0.0, 0.0, 0.0, 0.0};
    R4 O{0.0, 0.0, 0.0, 0.0};
    if (kind == KIND_OUTER) {
        const double *inf = g.obc + 8 * (size_t)(i - g.nw);
        conserved_ubar(P.a, P.b, P.c, P.d, nx, ny, inf, c.pi, c.gm1, U);
        if (rk == 3) {
            O = ld4(prim_old + i);
            conserved_ubar(O.a, O.b, O.c, O.d, nx, ny, inf, c.pi, c.gm1, Uo);
        }
    } else {
        prim_to_conserved(P.a, P.b, P.c, P.d, nx, ny, U);
        if (rk == 3) {
            O = ld4(prim_old + i);
            prim_to_conserved(O.a, O.b, O.c, O.d, nx, ny, Uo);
        }
    }
    double Up[4];
    for (int m = 0; m < 4; ++m) {
        if (rk != 3) Up[m] = U[m] - (0.5 * c.euler * frv[m]);
        else Up[m] = TBT * Uo[m] + OBT * (U[m] - 0.5 * frv[m]);
    }
    if (kind == KIND_WALL) Up[2] = 0.0;
    const double V1 = Up[1] * ny + Up[2] * nx;
    const double V2 = Up[2] * ny - Up[1] * nx;
    const double V0 = Up[0];
    const double tmp = 1.0 / V0;
    // reverse of prim_out = (V0, V1 tmp, V2 tmp, 0.4 (V3 - 0.5 tmp (V1^2 + V2^2)))
    const double *po = pb_out + 4 * (size_t)i;
    const double rb = po[0], u1b = po[1], u2b = po[2], pbv = po[3];
    const double inner = V1 * V1 + V2 * V2;
    const double V3b = 0.4 * pbv;
    double tmpb = -0.4 * 0.5 * inner * pbv;
    const double innerb = -0.4 * 0.5 * tmp * pbv;
    double V1b = 2.0 * V1 * innerb + u1b * tmp;
    double V2b = 2.0 * V2 * innerb + u2b * tmp;
    tmpb += u1b * V1 + u2b * V2;
    const double V0b = rb - tmpb * tmp * tmp;
    double Upb[4];
    Upb[0] = V0b;
    Upb[3] = V3b;
    Upb[1] = V1b * ny - V2b * nx;
    Upb[2] = V1b * nx + V2b * ny;
    double nxbv = V1b * Up[2] - V2b * Up[1];
    double nybv = V1b * Up[1] + V2b * Up[2];
    if (kind == KIND_WALL) Upb[2] = 0.0;
    double Ub[4], Uob[4], frbv[4];
    for (int m = 0; m < 4; ++m) {
        if (rk != 3) {
            Ub[m] = Upb[m];
            Uob[m] = 0.0;
            frbv[m] = -0.5 * c.euler * Upb[m];
        } else {
            Uob[m] = TBT * Upb[m];
            Ub[m] = OBT * Upb[m];
            frbv[m] = -0.5 * OBT * Upb[m];
        }
    }
    double pbi[4] = {0.0, 0.0, 0.0, 0.0}, pbo[4] = {0.0, 0.0, 0.0, 0.0};
    if (kind == KIND_OUTER) {
        conserved_ubar_b(P.a, P.b, P.c, P.d, nx, ny, a.q_inf, c.pi, c.gm1, Ub, pbi, nxbv, nybv);
        if (rk == 3)
            conserved_ubar_b(O.a, O.b, O.c, O.d, nx, ny, a.q_inf, c.pi, c.gm1, Uob, pbo, nxbv,
                             nybv);
    } else {
        prim_to_conserved_b(P.a, P.b, P.c, P.d, nx, ny, Ub, pbi, nxbv, nybv);
        if (rk == 3) prim_to_conserved_b(O.a, O.b, O.c, O.d, nx, ny, Uob, pbo, nxbv, nybv);
    }
    double *pin = pb_in + 4 * (size_t)i;
    for (int m = 0; m < 4; ++m) pin[m] += pbi[m];
    if (rk == 3) {
        double *pold = pb_old + 4 * (size_t)i;
        for (int m = 0; m < 4; ++m) pold[m] += pbo[m];
    }
    for (int m = 0; m < 4; ++m) frb[4 * (size_t)i + m] = frbv[m];
    nxb[i] += nxbv;
    nyb[i] += nybv;
}

// cal_flux_residual_b: same lane layout as the forward flux pass.
#ifndef FLUXB_MIN_BLOCKS
#define FLUXB_MIN_BLOCKS 3  // 168 registers; 4 blocks (128) spill (C3: 6.39 against 6.68 ms per reversed iteration)
#endif
__global__ void __launch_bounds__(BLK, FLUXB_MIN_BLOCKS)
k_flux_b(Geom g, Consts c, const R4 *__restrict__ q_in, const double *__restrict__ dq,
         const double *__restrict__ qm, const double *__restrict__ delta,
         const double *__restrict__ frb, double *__restrict__ qb, double *__restrict__ dqb,
         double *__restrict__ qmb, double *__restrict__ xb, double *__restrict__ yb,
         double *__restrict__ nxb, double *__restrict__ nyb, double *__restrict__ deltab,
         double *__restrict__ nbrec, const double *__restrict__ kst) {
    extern __shared__ double sm[];
    __shared__ double lb[GROUPS][4][11];  // fx_b[4] fy_b[4] sdx2_b sdy2_b sdxy_b per list
    const int grp = threadIdx.x / LPP, lane = threadIdx.x % LPP;
    const int i = blockIdx.x * GROUPS + grp;
    const bool valid = i < g.n;
    double *rec = sm + (size_t)grp * g.kp * BREC;
    int nb = 0, kind = KIND_INTERIOR;
    unsigned long long mx = 0, my = 0;
    double nx = 0.0, ny = 1.0;
    double2 pi_ = make_double2(0.0, 0.0);
    if (valid) {
        nb = g.nbhs[i];
        kind = i < g.nw ? KIND_WALL : (i < g.nw + g.no ? KIND_OUTER : KIND_INTERIOR);
        mx = g.mx[i];
        my = g.my[i];
        const double2 nn = g.nrm[i];
        nx = nn.x;
        ny = nn.y;
        pi_ = g.xy[i];
    }
    const double s2q = kind == KIND_WALL ? -1.0 : 1.0;
    // phase A: forward per slot
    if (valid) {
        for (int r = lane; r < nb; r += LPP) {
            const int k = g.conn[r * g.n + i];
            const double2 pk = g.xy[k];
            const double delx = pk.x - pi_.x, dely = pk.y - pi_.y;
            double e_[8];
            KState si, sk;
            if (kst) {
                // the forward re-run taped both reconstructions of this slot
                // (128 contiguous bytes, in four 256-bit loads)
                const double *tp = kst + ((size_t)i * g.kp + r) * KS_TAPE;
                double v[KS_TAPE];
#pragma unroll
                for (int hh = 0; hh < KS_TAPE / 4; ++hh) ld4nc(tp + 4 * hh, v + 4 * hh);
                si = kst_taped(v, nx, ny);
                sk = kst_taped(v + 8, nx, ny);
                e_[0] = v[6]; e_[1] = v[7]; e_[2] = si.rho; e_[3] = si.rho * si.pbr;
                e_[4] = v[14]; e_[5] = v[15]; e_[6] = sk.rho; e_[7] = sk.rho * sk.pbr;
            } else {
                const R4 qv = ld4(q_in + i), kv = ld4(q_in + k);
                const double qi[4] = {qv.a, qv.b, qv.c, qv.d}, qk[4] = {kv.a, kv.b, kv.c, kv.d};
                double dxi[4], dyi[4], qmaxi[4], qmini[4], dxk[4], dyk[4], qmaxk[4], qmink[4];
                ld8a(dq + 8 * (size_t)i, dxi, dyi);
                ld8a(qm + 8 * (size_t)i, qmaxi, qmini);
                ld8a(dq + 8 * (size_t)k, dxk, dyk);
                ld8a(qm + 8 * (size_t)k, qmaxk, qmink);
                reconstruct(qi, dxi, dyi, qmaxi, qmini, g.eps2[i], delx, dely, c.gm1, e_[0],
                            e_[1], e_[2], e_[3]);
                reconstruct(qk, dxk, dyk, qmaxk, qmink, g.eps2[k], delx, dely, c.gm1, e_[4],
                            e_[5], e_[6], e_[7]);
                si = kstate(e_[0], e_[1], e_[2], e_[3], nx, ny, c.pi);
                sk = kstate(e_[4], e_[5], e_[6], e_[7], nx, ny, c.pi);
            }
            double *e = rec + r * BREC;
            // one converged evaluation per direction and list holding the
            // neighbour (two only at a zero projection), lists in ascending
            // order, as in the forward kb_flux
            for (int d = 0; d < 2; ++d) {
                const unsigned long long bits = d == 0 ? mx : my;
                const bool in0 = (bits >> r) & 1ull, in1 = (bits >> (r + 32)) & 1ull;
                for (int pass = 0; pass < 2; ++pass) {
                    if (pass == 0 ? !(in0 || in1) : !(in0 && in1)) continue;
                    const int L = 2 * d + ((pass == 1 || !in0) ? 1 : 0);
                    const double sg = (L & 1) ? -1.0 : 1.0;
                    double Gi[4], Gk[4];
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
                    for (int m = 0; m < 4; ++m) e[4 * L + m] = Gk[m] - Gi[m];
                }
            }
            e[16] = delx * ny - dely * nx;
            e[17] = delx * nx + dely * ny;
            kst_store(e + 18, si);
            kst_store(e + 27, sk);
            for (int m = 0; m < 8; ++m) e[36 + m] = e_[m];
        }
    }
    __syncwarp();
    // phase B: list sums, forward G and the list-level adjoints
    double Gv0 = 0.0, Gv1 = 0.0;
    const int L = lane >> 1, c0 = (lane & 1) * 2;
    const bool used = valid && !((kind == KIND_WALL && L == 2) || (kind == KIND_OUTER && L == 3));
    const unsigned long long lbits = ((L < 2) ? mx : my) >> ((L & 1) ? 32 : 0);
    double sdx2 = 0.0, sdy2 = 0.0, sdxy = 0.0, fx[2] = {0.0, 0.0}, fy[2] = {0.0, 0.0};
    double obd = 0.0;
    if (used) {
        // the list's slots in slot order (lowest bit first): a lane loops
        // over its own members only (nb <= 20)
        unsigned rb = (unsigned)lbits & ((1u << nb) - 1u);
        while (rb) {
            const int r = __ffs(rb) - 1;
            rb &= rb - 1u;
            const double *e = rec + r * BREC;
            const double dels = e[16], deln = e[17];
            sdx2 = sdx2 + dels * dels;
            sdy2 = sdy2 + deln * deln;
            sdxy = sdxy + dels * deln;
            for (int h = 0; h < 2; ++h) {
                fx[h] = fx[h] + e[4 * L + c0 + h] * dels;
                fy[h] = fy[h] + e[4 * L + c0 + h] * deln;
            }
        }
        obd = 1.0 / (sdx2 * sdy2 - sdxy * sdxy);
        if (L < 2) {
            Gv0 = (fx[0] * sdy2 - fy[0] * sdxy) * obd;
            Gv1 = (fx[1] * sdy2 - fy[1] * sdxy) * obd;
        } else {
            Gv0 = (fy[0] * sdx2 - fx[0] * sdxy) * obd;
            Gv1 = (fy[1] * sdx2 - fx[1] * sdxy) * obd;
        }
    }
    double G[4][4];
    for (int LL = 0; LL < 4; ++LL)
        for (int h = 0; h < 2; ++h) {
            G[LL][2 * h] = __shfl_sync(0xffffffffu, Gv0, 2 * LL + h, LPP);
            G[LL][2 * h + 1] = __shfl_sync(0xffffffffu, Gv1, 2 * LL + h, LPP);
        }
    double frbv[4] = {0.0, 0.0, 0.0, 0.0}, dl = 0.0;
    if (valid) {
        for (int m = 0; m < 4; ++m) frbv[m] = frb[4 * (size_t)i + m];
        dl = delta[i];
    }
    const double coef = kind == KIND_WALL ? 2.0 * dl : dl;
    double sx2b = 0.0, sy2b = 0.0, sxyb = 0.0, obdb = 0.0, fxb[2] = {0.0, 0.0},
           fyb[2] = {0.0, 0.0};
    if (used) {
        for (int h = 0; h < 2; ++h) {
            const double Gb = coef * frbv[c0 + h];
            if (L < 2) {
                fxb[h] = Gb * sdy2 * obd;
                fyb[h] = -Gb * sdxy * obd;
                sy2b += Gb * fx[h] * obd;
                sxyb += -Gb * fy[h] * obd;
                obdb += Gb * (fx[h] * sdy2 - fy[h] * sdxy);
            } else {
                fyb[h] = Gb * sdx2 * obd;
                fxb[h] = -Gb * sdxy * obd;
                sx2b += Gb * fy[h] * obd;
                sxyb += -Gb * fx[h] * obd;
                obdb += Gb * (fy[h] * sdx2 - fx[h] * sdxy);
            }
        }
    }
    // combine the lane pair (components 0,1 and 2,3 of list L)
    sx2b += __shfl_xor_sync(0xffffffffu, sx2b, 1, LPP);
    sy2b += __shfl_xor_sync(0xffffffffu, sy2b, 1, LPP);
    sxyb += __shfl_xor_sync(0xffffffffu, sxyb, 1, LPP);
    obdb += __shfl_xor_sync(0xffffffffu, obdb, 1, LPP);
    if (used) {
        const double detb = -obdb * obd * obd;
        sx2b += detb * sdy2;
        sy2b += detb * sdx2;
        sxyb += -2.0 * detb * sdxy;
        for (int h = 0; h < 2; ++h) {
            lb[grp][L][c0 + h] = fxb[h];
            lb[grp][L][4 + c0 + h] = fyb[h];
        }
        if ((lane & 1) == 0) {
            lb[grp][L][8] = sx2b;
            lb[grp][L][9] = sy2b;
            lb[grp][L][10] = sxyb;
        }
    }
    if (valid && lane == 0) {
        double db = 0.0;
        for (int m = 0; m < 4; ++m) {
            double sg;
            if (kind == KIND_WALL) sg = 2.0 * (G[0][m] + G[1][m] + G[3][m]);
            else if (kind == KIND_OUTER) sg = G[0][m] + G[1][m] + G[2][m];
            else sg = G[0][m] + G[1][m] + G[2][m] + G[3][m];
            db += frbv[m] * sg;
        }
        deltab[i] += db;
    }
    __syncwarp();
    // phase C: per slot reverse of the fluxes, kinetic states and the
    // point's own reconstruction; the neighbour's reconstruction is left to
    // k_flux_b_nbr
    if (valid) {
        for (int r = lane; r < nb; r += LPP) {
            const int k = g.conn[r * g.n + i];
            const double2 pk = g.xy[k];
            const double delx = pk.x - pi_.x, dely = pk.y - pi_.y;
            double *e = rec + r * BREC;
            const double dels = e[16], deln = e[17];
            const KState si = kst_load(e + 18), sk = kst_load(e + 27);
            double pr_[8];
            for (int m = 0; m < 8; ++m) pr_[m] = e[36 + m];
            double delsb = 0.0, delnb = 0.0;
            KStateB sib, skb;
            kzero(sib);
            kzero(skb);
            for (int slot = 0; slot < 4; ++slot) {
                // (direction, pass) as in phase A: the lists holding the
                // neighbour in ascending order, one converged pass each
                const int d = slot >> 1, pass = slot & 1;
                const unsigned long long bits = d == 0 ? mx : my;
                const bool in0 = (bits >> r) & 1ull, in1 = (bits >> (r + 32)) & 1ull;
                if (pass == 0 ? !(in0 || in1) : !(in0 && in1)) continue;
                const int LL = 2 * d + ((pass == 1 || !in0) ? 1 : 0);
                if ((kind == KIND_WALL && LL == 2) || (kind == KIND_OUTER && LL == 3)) continue;
                const double sg = (LL & 1) ? -1.0 : 1.0;
                double dGb[4], mdGb[4];
                for (int m = 0; m < 4; ++m) {
                    const double fxbm = lb[grp][LL][m], fybm = lb[grp][LL][4 + m];
                    dGb[m] = fxbm * dels + fybm * deln;
                    mdGb[m] = -dGb[m];
                    delsb += fxbm * e[4 * LL + m];
                    delnb += fybm * e[4 * LL + m];
                }
                const double s2b = lb[grp][LL][8], n2b = lb[grp][LL][9], snb = lb[grp][LL][10];
                delsb += 2.0 * dels * s2b + deln * snb;
                delnb += 2.0 * deln * n2b + dels * snb;
                if (d == 0) {
                    if (kind == KIND_INTERIOR) {
                        flux_gx_b(sk, sg, dGb, skb);
                        flux_gx_b(si, sg, mdGb, sib);
                    } else {
                        flux_quad_b(sk, sg, s2q, dGb, skb);
                        flux_quad_b(si, sg, s2q, mdGb, sib);
                    }
                } else {
                    flux_gy_b(sk, sg, dGb, skb);
                    flux_gy_b(si, sg, mdGb, sib);
                }
            }
            double nxbv = 0.0, nybv = 0.0;
            double piu1b = 0.0, piu2b = 0.0, pirb = 0.0, pipb = 0.0;
            double pku1b = 0.0, pku2b = 0.0, pkrb = 0.0, pkpb = 0.0;
            kstate_b_s(si, pr_[0], pr_[1], nx, ny, sib, piu1b, piu2b, pirb, pipb, nxbv, nybv);
            kstate_b_s(sk, pr_[4], pr_[5], nx, ny, skb, pku1b, pku2b, pkrb, pkpb, nxbv, nybv);
            double delxb = delsb * ny + delnb * nx;
            double delyb = -delsb * nx + delnb * ny;
            nxbv += -delsb * dely + delnb * delx;
            nybv += delsb * delx + delnb * dely;
            const R4 qv = ld4(q_in + i);
            const double qi[4] = {qv.a, qv.b, qv.c, qv.d};
            double dxi[4], dyi[4], qmaxi[4], qmini[4];
            ld8a(dq + 8 * (size_t)i, dxi, dyi);
            ld8a(qm + 8 * (size_t)i, qmaxi, qmini);
            double qib[4] = {0, 0, 0, 0}, dxib[4] = {0, 0, 0, 0}, dyib[4] = {0, 0, 0, 0},
                   qmaxib[4] = {0, 0, 0, 0}, qminib[4] = {0, 0, 0, 0};
            reconstruct_b(qi, dxi, dyi, qmaxi, qmini, g.eps2[i], delx, dely, c.gm1, pr_[2], piu1b,
                          piu2b, pirb, pipb, qib, dxib, dyib, qmaxib, qminib, delxb, delyb);
            // the neighbour's side: its reconstruction is reversed by
            // k_flux_b_nbr from this record (the adjoint of its reconstructed
            // primitive state, its density, and delx/dely's adjoint so far)
            {
                const double v[NBREC] = {pku1b, pku2b, pkrb, pkpb, pr_[6], delxb, delyb, 0.0};
                st_pairs(nbrec + ((size_t)i * g.kp + r) * NBREC, v, NBREC);
            }
            // self contribution of this slot, summed in slot order below
            for (int m = 0; m < 4; ++m) {
                e[m] = qib[m];
                e[4 + m] = dxib[m];
                e[8 + m] = dyib[m];
                e[12 + m] = qmaxib[m];
                e[16 + m] = qminib[m];
            }
            e[20] = -delxb;
            e[21] = -delyb;
            e[22] = nxbv;
            e[23] = nybv;
        }
    }
    __syncwarp();
    if (!valid) return;
    for (int f = lane; f < 24; f += LPP) {
        double s = 0.0;
        for (int r = 0; r < nb; ++r) s = s + rec[r * BREC + f];
        if (f < 4) qb[4 * (size_t)i + f] += s;
        else if (f < 12) dqb[8 * (size_t)i + (f - 4)] += s;
        else if (f < 20) qmb[8 * (size_t)i + (f - 12)] += s;
        else if (f == 20) xb[i] += s;
        else if (f == 21) yb[i] += s;
        else if (f == 22) nxb[i] += s;
        else nyb[i] += s;
    }
}

// The neighbour side of cal_flux_residual_b, one thread per neighbour k:
// over the slots (i, r) that name k (the transposed stencil, in (i, r)
// order) it reverses k's reconstruction of that slot from k_flux_b's record
// and adds the results to k's own adjoints in registers: no scatter and no
// gather of contribution records.  The part of delx/dely's adjoint that this
// reconstruction adds belongs to point i as well (delx = x_k - x_i): it is
// left in back[(i, r)] for k_back_sum.
constexpr int NBR_BLK = 128;
#ifndef NBR_MIN_BLOCKS
#define NBR_MIN_BLOCKS 3  // 168 registers (4: 128 with spills, 1 % slower)
#endif
__global__ void __launch_bounds__(NBR_BLK, NBR_MIN_BLOCKS)
k_flux_b_nbr(Geom g, Consts c, const R4 *__restrict__ q_in, const double *__restrict__ dq,
             const double *__restrict__ qm, const int *__restrict__ tptr,
             const int *__restrict__ tlist, const double *__restrict__ nbrec,
             double *__restrict__ qb, double *__restrict__ dqb, double *__restrict__ qmb,
             double *__restrict__ xb, double *__restrict__ yb, double2 *__restrict__ back) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= g.n) return;
    const R4 kv = ld4(q_in + k);
    const double qk[4] = {kv.a, kv.b, kv.c, kv.d};
    double dxk[4], dyk[4], qmaxk[4], qmink[4];
    ld8a(dq + 8 * (size_t)k, dxk, dyk);
    ld8a(qm + 8 * (size_t)k, qmaxk, qmink);
    const double eps2 = g.eps2[k];
    const double2 pk = g.xy[k];
    double qkb[4] = {0, 0, 0, 0}, dxkb[4] = {0, 0, 0, 0}, dykb[4] = {0, 0, 0, 0},
           qmaxkb[4] = {0, 0, 0, 0}, qminkb[4] = {0, 0, 0, 0};
    double xkb = 0.0, ykb = 0.0;
    const int e1 = tptr[k + 1];
    for (int e = tptr[k]; e < e1; ++e) {
        const int slot = tlist[e];
        const int i = slot / g.kp;
        const double2 pi_ = g.xy[i];
        const double delx = pk.x - pi_.x, dely = pk.y - pi_.y;
        // the record: (u1b, u2b), (rhob, prb), (rho, delxb), (delyb, 0)
        const double2 *rv = reinterpret_cast<const double2 *>(nbrec + (size_t)slot * NBREC);
        const double2 ub = __ldg(rv), pb = __ldg(rv + 1), rd = __ldg(rv + 2), dy = __ldg(rv + 3);
        double dxr = 0.0, dyr = 0.0;
        reconstruct_b(qk, dxk, dyk, qmaxk, qmink, eps2, delx, dely, c.gm1, rd.x, ub.x, ub.y, pb.x,
                      pb.y, qkb, dxkb, dykb, qmaxkb, qminkb, dxr, dyr);
        xkb += rd.y + dxr;
        ykb += dy.x + dyr;
        back[slot] = make_double2(dxr, dyr);
    }
    add_pairs(qb + 4 * (size_t)k, qkb, 4);
    double v8[8];
    for (int m = 0; m < 4; ++m) {
        v8[m] = dxkb[m];
        v8[4 + m] = dykb[m];
    }
    add_pairs(dqb + 8 * (size_t)k, v8, 8);
    for (int m = 0; m < 4; ++m) {
        v8[m] = qmaxkb[m];
        v8[4 + m] = qminkb[m];
    }
    add_pairs(qmb + 8 * (size_t)k, v8, 8);
    xb[k] += xkb;
    yb[k] += ykb;
}

// x_i, y_i receive minus the delx/dely adjoint parts of their slots'
// neighbour reconstructions, in slot order.
__global__ void __launch_bounds__(256)
k_back_sum(Geom g, const double2 *__restrict__ back, double *__restrict__ xb,
           double *__restrict__ yb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.n) return;
    const int nb = g.nbhs[i];
    double sx = 0.0, sy = 0.0;
    for (int r = 0; r < nb; ++r) {
        const double2 v = __ldg(back + (size_t)i * g.kp + r);
        sx = sx + v.x;
        sy = sy + v.y;
    }
    xb[i] -= sx;
    yb[i] -= sy;
}

// eval_q_inner_loop_b: one inner iteration; dqb_out is the adjoint of its
// output, dqb_in receives the point's own share of the input adjoint.
__global__ void __launch_bounds__(BLK, ADJ_MIN_BLOCKS)
k_inner_b(Geom g, const R4 *__restrict__ q, const double *__restrict__ dq_in,
          const double *__restrict__ dqb_out, double *__restrict__ dqb_in, double *__restrict__ qb,
          double *__restrict__ xb, double *__restrict__ yb, double *__restrict__ contrib) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.n) return;
    const double2 pi_ = g.xy[i];
    const R4 qv = ld4(q + i);
    const double qi[4] = {qv.a, qv.b, qv.c, qv.d};
    double dxi[4], dyi[4];
    ld8a(dq_in + 8 * (size_t)i, dxi, dyi);
    const int nb = g.nbhs[i];
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, sx[4] = {0, 0, 0, 0}, sy[4] = {0, 0, 0, 0};
    for (int r = 0; r < nb; ++r) {
        const int k = g.conn[r * g.n + i];
        const R4 kv = ld4(q + k);
        const double qk[4] = {kv.a, kv.b, kv.c, kv.d};
        double dxk[4], dyk[4];
        ld8a(dq_in + 8 * (size_t)k, dxk, dyk);
        const double2 pk = g.xy[k];
        const double delx = pk.x - pi_.x, dely = pk.y - pi_.y;
        s0 = s0 + delx * delx;
        s1 = s1 + dely * dely;
        s2 = s2 + delx * dely;
        for (int m = 0; m < 4; ++m) {
            const double t1 = qi[m] - 0.5 * (delx * dxi[m] + dely * dyi[m]);
            const double t2 = qk[m] - 0.5 * (delx * dxk[m] + dely * dyk[m]);
            sx[m] = sx[m] + delx * (t2 - t1);
            sy[m] = sy[m] + dely * (t2 - t1);
        }
    }
    const double obd = 1.0 / (s0 * s1 - s2 * s2);
    double dxb[4], dyb[4];
    ld8a(dqb_out + 8 * (size_t)i, dxb, dyb);
    double sxb[4], syb[4], s0b = 0.0, s1b = 0.0, s2b = 0.0, obdb = 0.0;
    for (int m = 0; m < 4; ++m) {
        sxb[m] = (dxb[m] * s1 - dyb[m] * s2) * obd;
        syb[m] = (-dxb[m] * s2 + dyb[m] * s0) * obd;
        s1b += dxb[m] * sx[m] * obd;
        s0b += dyb[m] * sy[m] * obd;
        s2b += (-dxb[m] * sy[m] - dyb[m] * sx[m]) * obd;
        obdb += dxb[m] * (sx[m] * s1 - sy[m] * s2) + dyb[m] * (sy[m] * s0 - sx[m] * s2);
    }
    const double detb = -obdb * obd * obd;
    s0b += detb * s1;
    s1b += detb * s0;
    s2b += -2.0 * detb * s2;
    double qib[4] = {0, 0, 0, 0}, dxib[4] = {0, 0, 0, 0}, dyib[4] = {0, 0, 0, 0};
    double xib = 0.0, yib = 0.0;
    for (int r = 0; r < nb; ++r) {
        const int k = g.conn[r * g.n + i];
        const R4 kv = ld4(q + k);
        const double qk[4] = {kv.a, kv.b, kv.c, kv.d};
        double dxk[4], dyk[4];
        ld8a(dq_in + 8 * (size_t)k, dxk, dyk);
        const double2 pk = g.xy[k];
        const double delx = pk.x - pi_.x, dely = pk.y - pi_.y;
        double delxb = 2.0 * delx * s0b + dely * s2b;
        double delyb = 2.0 * dely * s1b + delx * s2b;
        double *cb = contrib + ((size_t)i * g.kp + r) * ADJ_CW;
        double v[14];  // the record, stored as 16-byte pairs at the end
        for (int m = 0; m < 4; ++m) {
            const double t1 = qi[m] - 0.5 * (delx * dxi[m] + dely * dyi[m]);
            const double t2 = qk[m] - 0.5 * (delx * dxk[m] + dely * dyk[m]);
            const double d = t2 - t1;
            const double db = sxb[m] * delx + syb[m] * dely;
            delxb += sxb[m] * d;
            delyb += syb[m] * d;
            v[m] = db;
            v[4 + m] = -0.5 * delx * db;
            v[8 + m] = -0.5 * dely * db;
            delxb += -0.5 * dxk[m] * db + 0.5 * dxi[m] * db;
            delyb += -0.5 * dyk[m] * db + 0.5 * dyi[m] * db;
            qib[m] -= db;
            dxib[m] += 0.5 * delx * db;
            dyib[m] += 0.5 * dely * db;
        }
        v[12] = delxb;
        v[13] = delyb;
        st_pairs(cb, v, 14);
        xib -= delxb;
        yib -= delyb;
    }
    add_pairs(qb + 4 * (size_t)i, qib, 4);
    st_pairs(dqb_in + 8 * (size_t)i, dxib, 4);
    st_pairs(dqb_in + 8 * (size_t)i + 4, dyib, 4);
    xb[i] += xib;
    yb[i] += yib;
}

// eval_q_derivatives_b (+ func_delta_b on the first stage)
// eval_q_derivatives_b + func_delta_b, the point's own side.  The
// neighbours' side reads the point's record grec[i] (GREC doubles: sxb[4],
// syb[4], s0b, s1b, s2b, deltab, qmaxb[4], qminb[4], the packed arg-max /
// arg-min slots, the time-step minimum's slot) in k_grad_b_nbr.
__global__ void __launch_bounds__(BLK, ADJ_MIN_BLOCKS)
k_grad_b(Geom g, Consts c, const R4 *__restrict__ q, const R4 *__restrict__ primA,
         const double *__restrict__ spdA, const double *__restrict__ dqb,
         const double *__restrict__ qmb,
         const double *__restrict__ deltab, int with_delta, double *__restrict__ qb,
         double *__restrict__ xb, double *__restrict__ yb, double *__restrict__ grec) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.n) return;
    const double2 pi_ = g.xy[i];
    const R4 qv = ld4(q + i);
    const double qi[4] = {qv.a, qv.b, qv.c, qv.d};
    const int nb = g.nbhs[i];
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, sx[4] = {0, 0, 0, 0}, sy[4] = {0, 0, 0, 0};
    double qmax[4] = {qi[0], qi[1], qi[2], qi[3]}, qmin[4] = {qi[0], qi[1], qi[2], qi[3]};
    int amax[4] = {-1, -1, -1, -1}, amin[4] = {-1, -1, -1, -1};
    double min_delt = 1.0;
    int amd = -1;
    for (int r = 0; r < nb; ++r) {
        const int k = g.conn[r * g.n + i];
        const R4 kv = ld4(q + k);
        const double qk[4] = {kv.a, kv.b, kv.c, kv.d};
        for (int m = 0; m < 4; ++m) {
            if (qk[m] > qmax[m]) { qmax[m] = qk[m]; amax[m] = r; }
            if (qk[m] < qmin[m]) { qmin[m] = qk[m]; amin[m] = r; }
        }
        const double2 pk = g.xy[k];
        const double delx = pk.x - pi_.x, dely = pk.y - pi_.y;
        s0 = s0 + delx * delx;
        s1 = s1 + dely * dely;
        s2 = s2 + delx * dely;
        for (int m = 0; m < 4; ++m) {
            sx[m] = sx[m] + delx * (qk[m] - qi[m]);
            sy[m] = sy[m] + dely * (qk[m] - qi[m]);
        }
        if (with_delta) {
            // the taped spd of the stage's input state: the forward's own values
            const double dist = sqrt(delx * delx + dely * dely);
            double delta_t = dist / spdA[k];
            delta_t = c.cfl * delta_t;
            if (min_delt > delta_t) { min_delt = delta_t; amd = r; }
        }
    }
    const double obd = 1.0 / (s0 * s1 - s2 * s2);
    double dxb[4], dyb[4], qmxb[4], qmnb[4];
    ld8a(dqb + 8 * (size_t)i, dxb, dyb);
    ld8a(qmb + 8 * (size_t)i, qmxb, qmnb);
    double sxb[4], syb[4], s0b = 0.0, s1b = 0.0, s2b = 0.0, obdb = 0.0;
    for (int m = 0; m < 4; ++m) {
        sxb[m] = (dxb[m] * s1 - dyb[m] * s2) * obd;
        syb[m] = (-dxb[m] * s2 + dyb[m] * s0) * obd;
        s1b += dxb[m] * sx[m] * obd;
        s0b += dyb[m] * sy[m] * obd;
        s2b += (-dxb[m] * sy[m] - dyb[m] * sx[m]) * obd;
        obdb += dxb[m] * (sx[m] * s1 - sy[m] * s2) + dyb[m] * (sy[m] * s0 - sx[m] * s2);
    }
    const double detb = -obdb * obd * obd;
    s0b += detb * s1;
    s1b += detb * s0;
    s2b += -2.0 * detb * s2;
    const double dlb = with_delta ? deltab[i] : 0.0;
    const int amd_used = (with_delta && dlb != 0.0) ? amd : -1;
    {
        // the record: slots packed 5 bits each (+1, so -1 -> 0), arg-max in
        // bits 0-19, arg-min in bits 20-39
        long long code = 0;
        for (int m = 0; m < 4; ++m) {
            code |= (long long)(amax[m] + 1) << (5 * m);
            code |= (long long)(amin[m] + 1) << (20 + 5 * m);
        }
        double v[GREC];
        for (int m = 0; m < 4; ++m) {
            v[m] = sxb[m];
            v[4 + m] = syb[m];
            v[12 + m] = qmxb[m];
            v[16 + m] = qmnb[m];
        }
        v[8] = s0b;
        v[9] = s1b;
        v[10] = s2b;
        v[11] = dlb;
        v[20] = __longlong_as_double(code);
        v[21] = (double)amd_used;
        v[22] = 0.0;
        v[23] = 0.0;
        st_pairs(grec + (size_t)i * GREC, v, GREC);
    }
    double qib[4] = {0, 0, 0, 0}, xib = 0.0, yib = 0.0;
    for (int m = 0; m < 4; ++m) {
        if (amax[m] < 0) qib[m] += qmxb[m];
        if (amin[m] < 0) qib[m] += qmnb[m];
    }
    for (int r = 0; r < nb; ++r) {
        const int k = g.conn[r * g.n + i];
        const R4 kv = ld4(q + k);
        const double qk[4] = {kv.a, kv.b, kv.c, kv.d};
        const double2 pk = g.xy[k];
        const double delx = pk.x - pi_.x, dely = pk.y - pi_.y;
        double delxb = 2.0 * delx * s0b + dely * s2b;
        double delyb = 2.0 * dely * s1b + delx * s2b;
        for (int m = 0; m < 4; ++m) {
            const double t = sxb[m] * delx + syb[m] * dely;
            qib[m] -= t;
            delxb += sxb[m] * (qk[m] - qi[m]);
            delyb += syb[m] * (qk[m] - qi[m]);
        }
        if (r == amd_used) {
            const R4 P = ld4(primA + k);
            const double modu = sqrt(P.b * P.b + P.c * P.c);
            const double cs = sqrt(P.d / P.a);
            const double spd = modu + 3.0 * cs;
            const double dist = sqrt(delx * delx + dely * dely);
            const double distb = dlb * c.cfl / spd;
            delxb += distb * delx / dist;
            delyb += distb * dely / dist;
        }
        xib -= delxb;
        yib -= delyb;
    }
    for (int m = 0; m < 4; ++m) qb[4 * (size_t)i + m] += qib[m];
    xb[i] += xib;
    yb[i] += yib;
}

// The neighbours' side of eval_q_derivatives_b + func_delta_b, one thread
// per neighbour k over the slots (i, r) naming it, in the transposed
// stencil's (i, r) order: q_k's adjoint from the point's least-squares sums
// and max/min, the time-step minimum's adjoint through k's taped state, and
// delx/dely's (the point's side takes the same value with the other sign).
__global__ void __launch_bounds__(BLK)
k_grad_b_nbr(Geom g, Consts c, const R4 *__restrict__ q, const R4 *__restrict__ primA,
             const int *__restrict__ tptr, const int *__restrict__ tlist,
             const double *__restrict__ grec, double *__restrict__ qb, double *__restrict__ pb,
             double *__restrict__ xb, double *__restrict__ yb) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= g.n) return;
    const R4 kv = ld4(q + k);
    const double qk[4] = {kv.a, kv.b, kv.c, kv.d};
    const double2 pk = g.xy[k];
    double qkb[4] = {0, 0, 0, 0}, pkb[4] = {0, 0, 0, 0}, xkb = 0.0, ykb = 0.0;
    const int e1 = tptr[k + 1];
    for (int e = tptr[k]; e < e1; ++e) {
        const int slot = tlist[e];
        const int i = slot / g.kp, r = slot - i * g.kp;
        const double2 *rv = reinterpret_cast<const double2 *>(grec + (size_t)i * GREC);
        double v[GREC];
#pragma unroll
        for (int h = 0; h < 6; ++h) {  // sxb, syb, s0b..s2b, deltab
            const double2 t2 = __ldg(rv + h);
            v[2 * h] = t2.x;
            v[2 * h + 1] = t2.y;
        }
        const double2 cd = __ldg(rv + 10);
        const long long code = __double_as_longlong(cd.x);
        const int amd = (int)cd.y;
        const R4 qv = ld4(q + i);
        const double qi[4] = {qv.a, qv.b, qv.c, qv.d};
        const double2 pi_ = g.xy[i];
        const double delx = pk.x - pi_.x, dely = pk.y - pi_.y;
        double delxb = 2.0 * delx * v[8] + dely * v[10];
        double delyb = 2.0 * dely * v[9] + delx * v[10];
        for (int m = 0; m < 4; ++m) {
            qkb[m] += v[m] * delx + v[4 + m] * dely;
            if ((int)((code >> (5 * m)) & 31) == r + 1) qkb[m] += grec[(size_t)i * GREC + 12 + m];
            if ((int)((code >> (20 + 5 * m)) & 31) == r + 1)
                qkb[m] += grec[(size_t)i * GREC + 16 + m];
            delxb += v[m] * (qk[m] - qi[m]);
            delyb += v[4 + m] * (qk[m] - qi[m]);
        }
        if (r == amd) {
            const double dlb = v[11];
            const R4 P = ld4(primA + k);
            const double modu = sqrt(P.b * P.b + P.c * P.c);
            const double cs = sqrt(P.d / P.a);
            const double spd = modu + 3.0 * cs;
            const double dist = sqrt(delx * delx + dely * dely);
            const double distb = dlb * c.cfl / spd;
            const double spdb = -dlb * c.cfl * dist / (spd * spd);
            delxb += distb * delx / dist;
            delyb += distb * dely / dist;
            if (modu > 0.0) {
                pkb[1] += spdb * P.b / modu;
                pkb[2] += spdb * P.c / modu;
            }
            const double csb = 3.0 * spdb;
            pkb[3] += csb * 0.5 / (cs * P.a);
            pkb[0] += -csb * 0.5 * P.d / (cs * P.a * P.a);
        }
        xkb += delxb;
        ykb += delyb;
    }
    add_pairs(qb + 4 * (size_t)k, qkb, 4);
    add_pairs(pb + 4 * (size_t)k, pkb, 4);
    xb[k] += xkb;
    yb[k] += ykb;
}

// Adds the neighbour contributions per point in the fixed transposed order.
// MODE fixes the record width (14 inner, 10 grad fields) so the
// accumulators stay in registers; records are read as 16-byte pairs.
template <int MODE>
__global__ void __launch_bounds__(256)
k_gather(int n, const int *__restrict__ tptr, const int *__restrict__ tlist,
         const double *__restrict__ contrib, double *__restrict__ a4, double *__restrict__ a8,
         double *__restrict__ b8, double *__restrict__ xb, double *__restrict__ yb) {
    constexpr int NF = MODE == ADJ_GATHER_INNER ? 14 : 10;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double acc[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) acc[f] = 0.0;
    const int e1 = tptr[k + 1];
    for (int e = tptr[k]; e < e1; ++e) {
        const double2 *cb = reinterpret_cast<const double2 *>(contrib + (size_t)tlist[e] * ADJ_CW);
#pragma unroll
        for (int f = 0; f < NF / 2; ++f) {
            const double2 v = __ldg(cb + f);
            acc[2 * f] = acc[2 * f] + v.x;
            acc[2 * f + 1] = acc[2 * f + 1] + v.y;
        }
    }
    add_pairs(a4 + 4 * (size_t)k, acc, 4);
    if constexpr (MODE == ADJ_GATHER_INNER) {
        add_pairs(a8 + 8 * (size_t)k, acc + 4, 8);
    } else {
        add_pairs(b8 + 4 * (size_t)k, acc + 4, 4);
    }
    xb[k] += acc[NF - 2];
    yb[k] += acc[NF - 1];
}

// eval_q_variables_b: pb += (dq/dprim)^T qb
__global__ void __launch_bounds__(256)
k_qvar_b(int n, const R4 *__restrict__ prim, const double *__restrict__ qb,
         double *__restrict__ pb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const R4 P = ld4(prim + i);
    double p[4] = {0.0, 0.0, 0.0, 0.0};
    q_from_prim_b(P.a, P.b, P.c, P.d, qb + 4 * (size_t)i, p);
    for (int m = 0; m < 4; ++m) pb[4 * (size_t)i + m] += p[m];
}

// compute_force_coeffs_b: J = sum over shapes of Cl (objective 0) or Cd (1).
__global__ void k_forces_b(AdjShape t, const R4 *__restrict__ prim, const double2 *__restrict__ xy,
                           double mach, double cos_t, double sin_t, int objective,
                           double *__restrict__ pb, double *__restrict__ xb,
                           double *__restrict__ yb, double *__restrict__ nxb,
                           double *__restrict__ nyb) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double pr_inf = 1.0 / 1.4;
    const double temp = 0.5 * 1.0 * mach * mach;
    const double Hb = objective == 1 ? cos_t : -sin_t;
    const double Vb = objective == 1 ? sin_t : cos_t;
    for (int j = 0; j < t.npts; ++j) {
        const int m = t.idx[j], l = t.left[j], r = t.right[j];
        const double nx = t.nx[j], ny = t.ny[j];
        const double2 L = xy[l], M = xy[m], R = xy[r];
        const double ds1 = sqrt((M.x - L.x) * (M.x - L.x) + (M.y - L.y) * (M.y - L.y));
        const double ds2 = sqrt((R.x - M.x) * (R.x - M.x) + (R.y - M.y) * (R.y - M.y));
        const double ds = 0.5 * (ds1 + ds2);
        double cp = prim[m].d - pr_inf;
        cp = -cp / temp;
        const double cpb = Hb * nx * ds + Vb * ny * ds;
        nxb[m] += Hb * cp * ds;
        nyb[m] += Vb * cp * ds;
        const double dsb = Hb * cp * nx + Vb * cp * ny;
        pb[4 * (size_t)m + 3] += -cpb / temp;
        const double d1 = 0.5 * dsb / ds1, d2 = 0.5 * dsb / ds2;
        xb[m] += d1 * (M.x - L.x) - d2 * (R.x - M.x);
        yb[m] += d1 * (M.y - L.y) - d2 * (R.y - M.y);
        xb[l] -= d1 * (M.x - L.x);
        yb[l] -= d1 * (M.y - L.y);
        xb[r] += d2 * (R.x - M.x);
        yb[r] += d2 * (R.y - M.y);
    }
}

// compute_normals_b for wall and outer points (point_normals.F90:19-89).
__global__ void k_normals_b(int nbnd, const int *__restrict__ left, const int *__restrict__ right,
                            const double2 *__restrict__ xy, const double *__restrict__ nxb,
                            const double *__restrict__ nyb, double *__restrict__ xb,
                            double *__restrict__ yb) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int m = 0; m < nbnd; ++m) {
        const int l = left[m], r = right[m];
        const double2 L = xy[l], M = xy[m], R = xy[r];
        const double vx = 0.5 * ((M.y - L.y) + (R.y - M.y));
        const double vy = 0.5 * ((M.x - L.x) + (R.x - M.x));
        const double det = sqrt(vx * vx + vy * vy);
        double vxb = -nxb[m] / det;
        double vyb = nyb[m] / det;
        const double detb = nxb[m] * vx / (det * det) - nyb[m] * vy / (det * det);
        vxb += detb * vx / det;
        vyb += detb * vy / det;
        yb[r] += 0.5 * vxb;
        yb[l] -= 0.5 * vxb;
        xb[r] += 0.5 * vyb;
        xb[l] -= 0.5 * vyb;
    }
}

// The same two reverses with a thread per boundary point q.  src[ptr[q] ..
// ptr[q+1]) lists the entries j whose loop body above adds to xb[q] / yb[q],
// in the loop's order (ascending j; within one j the order of its
// statements), so that each sum is formed in the serial kernel's order and
// the results are the same bit for bit.  Normals: src = 2j + (0: q is
// right[j], 1: q is left[j]).  Forces: src = 3j + (0: q is idx[j], 1: q is
// left[j], 2: q is right[j]).
__global__ void k_normals_b_gather(int nbnd, const int *__restrict__ left,
                                   const int *__restrict__ right, const double2 *__restrict__ xy,
                                   const double *__restrict__ nxb, const double *__restrict__ nyb,
                                   const int *__restrict__ ptr, const int *__restrict__ src,
                                   double *__restrict__ xb, double *__restrict__ yb) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nbnd) return;
    double xq = xb[q], yq = yb[q];
    for (int e = ptr[q]; e < ptr[q + 1]; ++e) {
        const int m = src[e] >> 1, role = src[e] & 1;
        const int l = left[m], r = right[m];
        const double2 L = xy[l], M = xy[m], R = xy[r];
        const double vx = 0.5 * ((M.y - L.y) + (R.y - M.y));
        const double vy = 0.5 * ((M.x - L.x) + (R.x - M.x));
        const double det = sqrt(vx * vx + vy * vy);
        double vxb = -nxb[m] / det;
        double vyb = nyb[m] / det;
        const double detb = nxb[m] * vx / (det * det) - nyb[m] * vy / (det * det);
        vxb += detb * vx / det;
        vyb += detb * vy / det;
        if (role == 0) {
            yq += 0.5 * vxb;
            xq += 0.5 * vyb;
        } else {
            yq -= 0.5 * vxb;
            xq -= 0.5 * vyb;
        }
    }
    xb[q] = xq;
    yb[q] = yq;
}

__global__ void k_forces_b_gather(AdjShape t, int nbnd, const R4 *__restrict__ prim,
                                  const double2 *__restrict__ xy, double mach, double cos_t,
                                  double sin_t, int objective, const int *__restrict__ ptr,
                                  const int *__restrict__ src, double *__restrict__ pb,
                                  double *__restrict__ xb, double *__restrict__ yb,
                                  double *__restrict__ nxb, double *__restrict__ nyb) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nbnd) return;
    const double pr_inf = 1.0 / 1.4;
    const double temp = 0.5 * 1.0 * mach * mach;
    const double Hb = objective == 1 ? cos_t : -sin_t;
    const double Vb = objective == 1 ? sin_t : cos_t;
    double xq = xb[q], yq = yb[q];
    for (int e = ptr[q]; e < ptr[q + 1]; ++e) {
        const int j = src[e] / 3, role = src[e] % 3;
        const int m = t.idx[j], l = t.left[j], r = t.right[j];
        const double nx = t.nx[j], ny = t.ny[j];
        const double2 L = xy[l], M = xy[m], R = xy[r];
        const double ds1 = sqrt((M.x - L.x) * (M.x - L.x) + (M.y - L.y) * (M.y - L.y));
        const double ds2 = sqrt((R.x - M.x) * (R.x - M.x) + (R.y - M.y) * (R.y - M.y));
        const double ds = 0.5 * (ds1 + ds2);
        double cp = prim[m].d - pr_inf;
        cp = -cp / temp;
        const double dsb = Hb * cp * nx + Vb * cp * ny;
        const double d1 = 0.5 * dsb / ds1, d2 = 0.5 * dsb / ds2;
        if (role == 0) {
            const double cpb = Hb * nx * ds + Vb * ny * ds;
            nxb[m] += Hb * cp * ds;
            nyb[m] += Vb * cp * ds;
            pb[4 * (size_t)m + 3] += -cpb / temp;
            xq += d1 * (M.x - L.x) - d2 * (R.x - M.x);
            yq += d1 * (M.y - L.y) - d2 * (R.y - M.y);
        } else if (role == 1) {
            xq -= d1 * (M.x - L.x);
            yq -= d1 * (M.y - L.y);
        } else {
            xq += d2 * (R.x - M.x);
            yq += d2 * (R.y - M.y);
        }
    }
    xb[q] = xq;
    yb[q] = yq;
}

inline int nblk(int n, int b) { return (n + b - 1) / b; }

}  // namespace

cudaError_t init_adjoint_kernels() {
    return cudaFuncSetAttribute(k_flux_b, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                GROUPS * 20 * BREC * (int)sizeof(double));
}

void launch_update_b(const Geom &g, const Consts &c, const AdjConsts &a, const R4 *prim_in,
                     const R4 *prim_old, const R4 *fr, const double *pb_out, double *pb_in,
                     double *pb_old, double *frb, double *nxb, double *nyb, int rk,
                     cudaStream_t s) {
    k_update_b<<<nblk(g.n, BLK), BLK, 0, s>>>(g, c, a, prim_in, prim_old, fr, pb_out, pb_in,
                                             pb_old, frb, nxb, nyb, rk);
}

void launch_flux_b(const Geom &g, const Consts &c, const R4 *q_in, const double *dq,
                   const double *qm, const double *delta, const double *frb, double *qb,
                   double *dqb, double *qmb, double *xb, double *yb, double *nxb, double *nyb,
                   double *deltab, double *nbrec, double *back, const int *tptr,
                   const int *tlist, const double *kst, cudaStream_t s) {
    size_t smem = (size_t)GROUPS * g.kp * BREC * sizeof(double);
    k_flux_b<<<nblk(g.n, GROUPS), BLK, smem, s>>>(g, c, q_in, dq, qm, delta, frb, qb, dqb, qmb,
                                                  xb, yb, nxb, nyb, deltab, nbrec, kst);
    double2 *bk = reinterpret_cast<double2 *>(back);
    k_flux_b_nbr<<<nblk(g.n, NBR_BLK), NBR_BLK, 0, s>>>(g, c, q_in, dq, qm, tptr, tlist, nbrec,
                                                       qb, dqb, qmb, xb, yb, bk);
    k_back_sum<<<nblk(g.n, 256), 256, 0, s>>>(g, bk, xb, yb);
}

void launch_inner_b(const Geom &g, const R4 *q, const double *dq_in, const double *dqb_out,
                    double *dqb_in, double *qb, double *xb, double *yb, double *contrib,
                    cudaStream_t s) {
    k_inner_b<<<nblk(g.n, BLK), BLK, 0, s>>>(g, q, dq_in, dqb_out, dqb_in, qb, xb, yb, contrib);
}

void launch_grad_b(const Geom &g, const Consts &c, const R4 *q, const R4 *primA,
                   const double *spdA, const double *dqb, const double *qmb,
                   const double *deltab, bool with_delta, double *qb, double *pb, double *xb,
                   double *yb, double *grec, const int *tptr, const int *tlist,
                   cudaStream_t s) {
    k_grad_b<<<nblk(g.n, BLK), BLK, 0, s>>>(g, c, q, primA, spdA, dqb, qmb, deltab,
                                           with_delta ? 1 : 0, qb, xb, yb, grec);
    k_grad_b_nbr<<<nblk(g.n, BLK), BLK, 0, s>>>(g, c, q, primA, tptr, tlist, grec, qb, pb, xb,
                                               yb);
}

void launch_gather(int n, int kp, const int *tptr, const int *tlist, const double *contrib,
                   int mode, double *a4, double *a8, double *b8, double *xb, double *yb,
                   cudaStream_t s) {
    (void)kp;
    if (mode == ADJ_GATHER_INNER)
        k_gather<ADJ_GATHER_INNER><<<nblk(n, 256), 256, 0, s>>>(n, tptr, tlist, contrib, a4, a8,
                                                               b8, xb, yb);
    else
        k_gather<ADJ_GATHER_GRAD><<<nblk(n, 256), 256, 0, s>>>(n, tptr, tlist, contrib, a4, a8, b8,
                                                              xb, yb);
}

void launch_qvar_b(int n, const R4 *prim, const double *qb, double *pb, cudaStream_t s) {
    k_qvar_b<<<nblk(n, 256), 256, 0, s>>>(n, prim, qb, pb);
}

void launch_forces_b(const AdjShape &t, const AdjGather &gth, const R4 *prim, const double2 *xy,
                     double mach, double cos_t, double sin_t, int objective, double *pb,
                     double *xb, double *yb, double *nxb, double *nyb, cudaStream_t s) {
    if (gth.fptr)
        k_forces_b_gather<<<nblk(std::max(gth.nbnd, 1), 128), 128, 0, s>>>(
            t, gth.nbnd, prim, xy, mach, cos_t, sin_t, objective, gth.fptr, gth.fsrc, pb, xb, yb,
            nxb, nyb);
    else
        k_forces_b<<<1, 32, 0, s>>>(t, prim, xy, mach, cos_t, sin_t, objective, pb, xb, yb, nxb,
                                    nyb);
}

void launch_normals_b(int nbnd, const AdjGather &gth, const int *left, const int *right,
                      const double2 *xy, const double *nxb, const double *nyb, double *xb,
                      double *yb, cudaStream_t s) {
    if (gth.nptr)
        k_normals_b_gather<<<nblk(std::max(nbnd, 1), 128), 128, 0, s>>>(
            nbnd, left, right, xy, nxb, nyb, gth.nptr, gth.nsrc, xb, yb);
    else
        k_normals_b<<<1, 32, 0, s>>>(nbnd, left, right, xy, nxb, nyb, xb, yb);
}

}  // namespace lskum
