// C ABI of mfcfd_b200: handle, host-side set-up and the pseudo-time driver.
//
// Set-up restates the reference's once-per-run work on the host, in the
// reference's arithmetic (this file is compiled without FMA contraction):
//   point_normals.F90:8-105        wall/outer normals, interior (0,1)/(1,0)
//   generate_connectivity.F90      xpos/xneg/ypos/yneg membership, kept as
//                                  per-point bit masks over the stencil slots
//   point_preprocessor.F90:374-435 wall/interior/outer/shape classification
//   parameter.F90:16-34            theta and the freestream state
// then renumbers the points (wall | outer | interior, optionally after RCM)
// and uploads everything once.  mfcfd_run enqueues the iterations as CUDA
// graphs (two iterations per graph, because the prim buffers alternate) with
// no host synchronisation until the residue history is read back.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <deque>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "handle.h"
#include "mfcfd_b200.h"
#include "primal.h"

using namespace lskum;

namespace {

constexpr int MAXNB = 20;
thread_local std::string g_create_error;

}  // namespace

using lskum_host::dmalloc;

namespace lskum_host {

int fail(mfcfd_t *h, int code, const std::string &msg) {
    if (h) h->err = msg;
    else g_create_error = msg;
    return code;
}

int cuda_fail(mfcfd_t *h, cudaError_t e, const char *where) {
    std::string m = std::string(where) + ": " + cudaGetErrorString(e);
    return fail(h, e == cudaErrorMemoryAllocation ? MFCFD_ERR_OOM : MFCFD_ERR_CUDA, m);
}

}  // namespace lskum_host

using lskum_host::cuda_fail;
using lskum_host::fail;

namespace {

void free_all(mfcfd_t *h) {
    lskum_host::free_adjoint(h);
    for (auto &row : h->pair_exec)
        for (auto &g : row)
            if (g) cudaGraphExecDestroy(g);
    for (auto &row : h->one_exec)
        for (auto &g : row)
            if (g) cudaGraphExecDestroy(g);
    void *bufs[] = {h->d_xy, h->d_nrm, h->d_eps2, h->d_obc, h->d_conn, h->d_nbhs, h->d_mx,
                    h->d_my, h->d_hoff, h->d_hrow, h->d_hloc, h->d_prim[0], h->d_prim[1], h->d_q[0], h->d_q[1], h->d_dq[0],
                    h->d_dq[1], h->d_dq[2], h->d_qm, h->d_delta, h->d_spd, h->d_res_part, h->d_flux_dbg,
                    h->d_hist, h->d_forces, h->d_ctl, h->d_sh_idx, h->d_sh_shape, h->d_sh_geo,
                    h->d_sh_my, h->f_prim[0], h->f_prim[1], h->f_q[0], h->f_q[1],
                    h->f_dq[0], h->f_dq[1], h->f_dq[2], h->f_qm, h->f_eps2, h->f_dxy, h->f_w, h->f_lsq,
                    h->f_flsq, h->d_inst, h->d_sched,
                    h->d_run, h->d_part_sum};
    for (void *b : bufs)
        if (b) cudaFree(b);
    if (h->h_ctl) cudaFreeHost(h->h_ctl);
    if (h->h_stage) cudaFreeHost(h->h_stage);
    if (h->h_sched) cudaFreeHost(h->h_sched);
    if (h->own) cudaStreamDestroy(h->own);
}

// Reverse Cuthill-McKee over the symmetrised stencil graph.
std::vector<int> rcm_order(int n, const std::vector<std::vector<int>> &adj) {
    std::vector<int> order;
    order.reserve(n);
    std::vector<char> seen(n, 0);
    std::vector<int> byDeg(n);
    for (int i = 0; i < n; ++i) byDeg[i] = i;
    std::stable_sort(byDeg.begin(), byDeg.end(),
                     [&](int a, int b) { return adj[a].size() < adj[b].size(); });
    for (int root : byDeg) {
        if (seen[root]) continue;
        std::deque<int> qq{root};
        seen[root] = 1;
        while (!qq.empty()) {
            int v = qq.front();
            qq.pop_front();
            order.push_back(v);
            std::vector<int> nb;
            for (int w : adj[v])
                if (!seen[w]) {
                    seen[w] = 1;
                    nb.push_back(w);
                }
            std::stable_sort(nb.begin(), nb.end(),
                             [&](int a, int b) { return adj[a].size() < adj[b].size(); });
            for (int w : nb) qq.push_back(w);
        }
    }
    std::reverse(order.begin(), order.end());
    return order;
}

// Launches the kernels of pseudo-time stage rk (prim buffers A -> B) and
// calls `after` once after each launch.
template <class F>
void launch_stage(mfcfd_t *h, cudaStream_t s, int rk, int A, int B, F after) {
    const int m = h->p.inner_iterations;
    const bool last = rk == h->p.rks;
    if (!h->fp32) {
        const R4 *q_in = h->d_q[h->qcur];
        launch_grad(h->geom, h->consts, h->sched, q_in, h->d_spd, h->d_dq[0], h->d_qm,
                    h->d_delta, rk == 1, h->point_block, h->point_grid, s);
        after();
        for (int t = 1; t <= m; ++t) {
            launch_inner(h->geom, h->consts, h->sched, h->d_dq[0], h->d_dq[dq_src(t)],
                         h->d_dq[dq_dst(t)], h->point_block, h->inner_grid, s);
            after();
        }
        StageBufs b;
        b.prim_in = rk == 1 ? h->d_prim[A] : h->d_prim[B];
        b.prim_out = h->d_prim[B];
        b.prim_old = h->d_prim[A];
        b.q_in = q_in;
        b.q_out = h->d_q[h->qcur ^ 1];
        b.dq = h->d_dq[dq_final(m)];
        b.qm = h->d_qm;
        b.delta = h->d_delta;
        b.spd = h->d_spd;
        b.res_part = h->d_res_part;
        b.flux_dbg = h->keep_diag ? h->d_flux_dbg : nullptr;
        launch_flux(h->geom, h->consts, h->sched, b, rk, last, h->flux_grid, s);
        after();
    } else {
        const float4 *q_in = h->f_q[h->qcur];
        launch_grad32(h->geom, h->consts, h->geom32, h->sched, q_in, h->d_spd, h->f_dq[0],
                      h->f_qm, h->d_delta, rk == 1, h->point_block, h->point_grid, s);
        after();
        for (int t = 1; t <= m; ++t) {
            launch_inner32(h->geom, h->consts, h->geom32, h->sched, h->f_dq[0],
                           h->f_dq[dq32_src(t)], h->f_dq[dq32_dst(t)], h->point_block,
                           h->inner_grid, s);
            after();
        }
        StageBufs32 b;
        b.prim_in = rk == 1 ? h->f_prim[A] : h->f_prim[B];
        b.prim_out = h->f_prim[B];
        b.prim_old = h->f_prim[A];
        b.q_in = q_in;
        b.q_out = h->f_q[h->qcur ^ 1];
        b.dq = h->f_dq[dq32_final(m)];
        b.qm = h->f_qm;
        b.eps2f = h->f_eps2;
        b.delta = h->d_delta;
        b.spd = h->d_spd;
        b.res_part = h->d_res_part;
        b.flux_dbg = h->keep_diag ? h->d_flux_dbg : nullptr;
        b.f = h->geom32;
        launch_flux32(h->geom, h->consts, h->sched, b, rk, last, h->flux_grid, s);
        after();
    }
    h->qcur ^= 1;
    h->launches += 2 + m;
}

}  // namespace

// One iteration (fpi_solver): the stages, then the residual into hist.
int lskum_host::enqueue_iteration_to(mfcfd_t *h, cudaStream_t s, double *hist) {
    const int A = h->cur, B = h->cur ^ 1;
    for (int rk = 1; rk <= h->p.rks; ++rk) launch_stage(h, s, rk, A, B, [] {});
    launch_residual(h->d_inst, 1, h->d_res_part, h->d_ctl, hist, 0, h->d_run, h->d_sched, s);
    h->launches += 1;
    h->cur = B;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(h, e, "kernel launch");
    return MFCFD_OK;
}

namespace {
using lskum_host::enqueue_iteration_to;

int enqueue_iteration(mfcfd_t *h, cudaStream_t s) { return enqueue_iteration_to(h, s, h->d_hist); }

// Captures two consecutive iterations into one graph.  After two iterations
// both the prim and the q buffer parity are back where they started.
void drop_graphs(mfcfd_t *h) {
    for (auto *tab : {&h->pair_exec, &h->one_exec})
        for (auto &row : *tab)
            for (auto &g : row)
                if (g) {
                    cudaGraphExecDestroy(g);
                    g = nullptr;
                }
}

// Captures one iteration (the odd one of an odd count) into a graph and
// records the (cur, qcur) it leaves current.
int build_one_graph(mfcfd_t *h) {
    const int cur0 = h->cur, q0 = h->qcur;
    cudaGraphExec_t &slot = h->one_exec[cur0][q0];
    if (slot) {
        cudaGraphExecDestroy(slot);
        slot = nullptr;
    }
    const long long l0 = h->launches;
    cudaGraph_t graph;
    CK(cudaStreamBeginCapture(h->own, cudaStreamCaptureModeThreadLocal));
    const int st = enqueue_iteration(h, h->own);
    cudaError_t e = cudaStreamEndCapture(h->own, &graph);
    h->one_next[cur0][q0][0] = h->cur;
    h->one_next[cur0][q0][1] = h->qcur;
    h->cur = cur0;
    h->qcur = q0;
    h->launches = l0;
    if (st != MFCFD_OK) return st;
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&slot, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaGraphInstantiate");
    return MFCFD_OK;
}

int build_pair_graph(mfcfd_t *h) {
    int cur0 = h->cur, q0 = h->qcur;
    cudaGraphExec_t &slot = h->pair_exec[cur0][q0];
    if (slot) {
        cudaGraphExecDestroy(slot);
        slot = nullptr;
    }
    long long l0 = h->launches;
    cudaGraph_t graph;
    CK(cudaStreamBeginCapture(h->own, cudaStreamCaptureModeThreadLocal));
    int st = enqueue_iteration(h, h->own);
    if (st == MFCFD_OK) st = enqueue_iteration(h, h->own);
    cudaError_t e = cudaStreamEndCapture(h->own, &graph);
    h->cur = cur0;
    h->qcur = q0;
    h->launches = l0;
    if (st != MFCFD_OK) return st;
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&slot, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaGraphInstantiate");
    return MFCFD_OK;
}

}  // namespace

int lskum_host::upload_state_aux(mfcfd_t *h) {
    if (h->fp32)
        launch_init_state32(h->geom, h->f_prim[h->cur], h->f_q[h->qcur], h->d_spd, h->stream);
    else
        launch_init_state(h->geom, h->d_prim[h->cur], h->d_q[h->qcur], h->d_spd, h->stream);
    h->launches += 1;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(h, e, "init_state launch");
    return MFCFD_OK;
}

using lskum_host::upload_state_aux;

// A tile's halo lists its rows in ascending order, so that the rows of
// neighbouring rings come in contiguous runs and the staging copies
// coalesce; the local indices are positions in that list.
void lskum_host::build_halo(int n, int kp, const int *conn, const int *nbhs,
                            const std::vector<std::pair<int, int>> &ranges, HostHalo &out) {
    const int ntile = (n + TILE - 1) / TILE;
    out.hkp = ((kp + 1 + 7) / 8) * 8;
    out.hc = 0;
    out.off.assign((size_t)ntile + 1, 0);
    out.rows.clear();
    out.loc.assign((size_t)n * out.hkp, 0);
    if (out.hkp > 24) {  // local row bytes beyond three words: no halos
        out.off.assign((size_t)ntile + 1, 0);
        out.loc.clear();
        return;
    }
    std::vector<int> tend(ntile, -1);  // end of the tile's owned points (-1: not scheduled)
    for (const auto &rg : ranges)
        for (int p0 = rg.first; p0 < rg.first + rg.second; p0 += TILE)
            tend[p0 / TILE] = std::min(p0 + TILE, rg.first + rg.second);
    std::vector<int> rows;
    rows.reserve((size_t)TILE * (kp + 1));
    for (int t = 0; t < ntile; ++t) {
        out.off[t] = (int)out.rows.size();
        if (tend[t] < 0) continue;
        rows.clear();
        for (int p = t * TILE; p < tend[t]; ++p) {
            rows.push_back(p);
            for (int r = 0; r < nbhs[p]; ++r) rows.push_back(conn[(size_t)r * n + p]);
        }
        std::sort(rows.begin(), rows.end());
        rows.erase(std::unique(rows.begin(), rows.end()), rows.end());
        if ((int)rows.size() > HALO_CAP) continue;  // gathered directly
        auto pos = [&](int k) {
            return (unsigned char)(std::lower_bound(rows.begin(), rows.end(), k) - rows.begin());
        };
        for (int p = t * TILE; p < tend[t]; ++p) {
            unsigned char *l = out.loc.data() + (size_t)p * out.hkp;
            for (int r = 0; r < nbhs[p]; ++r) l[r] = pos(conn[(size_t)r * n + p]);
            l[out.hkp - 1] = pos(p);
        }
        out.hc = std::max(out.hc, (int)rows.size());
        out.rows.insert(out.rows.end(), rows.begin(), rows.end());
    }
    out.off[ntile] = (int)out.rows.size();
    // the staging stride: one more than a multiple of eight rows, so that a
    // row's 16-byte pieces in consecutive arrays fall on different banks
    // (C2 I pass: 0.091 ms; 0.109 with no padding, 0.097 - 0.101 at two to
    // seven more than a multiple of eight)
    if (out.hc > 0) out.hc += (9 - out.hc % 8) % 8;
}

int lskum_host::reset_run(mfcfd_t *h, int it_first) {
    h->h_ctl->it = it_first;
    h->h_ctl->it_first = it_first;
    h->h_ctl->halted = 0;
    h->h_ctl->done = 0;
    h->h_ctl->active = 1;
    h->h_ctl->state = BATCH_RUNNING;
    const int one = 1;
    sched_fill(h->h_sched, &h->inst_h, &one, 1);
    CK(cudaMemcpyAsync(h->d_ctl, h->h_ctl, CTL_RESET_BYTES, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_sched, h->h_sched, sizeof(int) * SCHED_INTS, cudaMemcpyHostToDevice,
                       h->stream));
    return MFCFD_OK;
}

extern "C" {

int mfcfd_default_params(mfcfd_params *p) {
    if (!p) return MFCFD_ERR_ARG;
    memset(p, 0, sizeof(*p));
    p->cfl = 0.0;
    p->power = 0.0;
    p->vl_const = 150.0;
    p->mach = 0.63;
    p->aoa = 2.0;
    p->rks = 4;
    p->euler = 1.0;
    p->inner_iterations = 0;
    p->interior_points_normal_flag = 0;
    p->format = 1;
    p->restart = 0;
    p->res_old = 0.0;
    p->precision = MFCFD_FP64;
    p->ordering = MFCFD_ORDER_KIND;
    return MFCFD_OK;
}

}  // extern "C"

namespace {

// Geometry of the FP32-mixed passes, formed once in FP64 with the
// reference's sums and rounded to FP32: per stencil slot the offset (and
// weight); per point the inverse of the normal matrix of eval_q_derivatives
// (q_variables.F90:84-110: dx = a Sx + b Sy, dy = b Sx + c Sy); per point and
// split list the two coefficients of the flux least-squares solve
// (interior_fluxes.F90: x lists G = a Sx + b Sy, y lists G = a Sy + b Sx,
// with Sx, Sy the sums of dG dels_w, dG deln_w).
void build_geom32(HostGrid &hg, int nw, int no, double power) {
    const int n = hg.n, kp = hg.kp;
    hg.dxy.assign((size_t)kp * n, make_float2(0.f, 0.f));
    hg.wslot.assign(power != 0.0 ? (size_t)kp * n : 0, 0.f);
    hg.lsq.assign(n, make_float4(0.f, 0.f, 0.f, 0.f));
    hg.flsq.assign(2 * (size_t)n, make_float4(0.f, 0.f, 0.f, 0.f));
    for (int p = 0; p < n; ++p) {
        const double xi = hg.xy[p].x, yi = hg.xy[p].y, nx = hg.nrm[p].x, ny = hg.nrm[p].y;
        const int kind = p < nw ? 0 : (p < nw + no ? 2 : 1);
        double sdx2 = 0.0, sdy2 = 0.0, sdxy = 0.0;
        double ls[4][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int r = 0; r < hg.nbhs[p]; ++r) {
            const int k = hg.conn[(size_t)r * n + p];
            const double delx = hg.xy[k].x - xi, dely = hg.xy[k].y - yi;
            double w = 1.0;
            if (power != 0.0) w = pow(sqrt(delx * delx + dely * dely), power);
            hg.dxy[(size_t)r * n + p] = make_float2((float)delx, (float)dely);
            if (power != 0.0) hg.wslot[(size_t)r * n + p] = (float)w;
            sdx2 = sdx2 + delx * delx * w;
            sdy2 = sdy2 + dely * dely * w;
            sdxy = sdxy + delx * dely * w;
            const double tx = ny, ty = -nx;
            const double dels = delx * tx + dely * ty, deln = delx * nx + dely * ny;
            double wl = 1.0;
            if (power != 0.0) wl = pow(sqrt(dels * dels + deln * deln), power);
            const double dels_w = dels * wl, deln_w = deln * wl;
            for (int L = 0; L < 4; ++L) {
                const unsigned long long bits = L < 2 ? hg.mx[p] : hg.my[p];
                if (!((bits >> (r + ((L & 1) ? 32 : 0))) & 1ull)) continue;
                ls[L][0] = ls[L][0] + dels * dels_w;
                ls[L][1] = ls[L][1] + deln * deln_w;
                ls[L][2] = ls[L][2] + dels * deln_w;
            }
        }
        const double obd = 1.0 / (sdx2 * sdy2 - sdxy * sdxy);
        hg.lsq[p] = make_float4((float)(sdy2 * obd), (float)(-sdxy * obd), (float)(sdx2 * obd), 0.f);
        float co[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        for (int L = 0; L < 4; ++L) {
            if ((kind == 0 && L == 2) || (kind == 2 && L == 3)) continue;
            const double ob = 1.0 / (ls[L][0] * ls[L][1] - ls[L][2] * ls[L][2]);
            co[2 * L] = (float)((L < 2 ? ls[L][1] : ls[L][0]) * ob);
            co[2 * L + 1] = (float)(-ls[L][2] * ob);
        }
        hg.flsq[2 * (size_t)p] = make_float4(co[0], co[1], co[2], co[3]);
        hg.flsq[2 * (size_t)p + 1] = make_float4(co[4], co[5], co[6], co[7]);
    }
}

}  // namespace

// Host half of mfcfd_create: checks of the grid and parameters, normals,
// split membership, renumbering and the renumbered arrays, all in caller
// arithmetic; no device call.  Errors are reported as by mfcfd_create.
int lskum_host::prepare_grid(const mfcfd_grid &G, const mfcfd_params &P, HostGrid &hg,
                             int n_local) {
    const int n = G.n;
    if (n <= 0) return fail(nullptr, MFCFD_ERR_ARG, "grid.n must be positive");
    // points [n_local, n) are ghosts of a partitioned grid: only their x, y
    // and min_dist are used (the reference's ghost rows,
    // point_preprocessor.F90:489-501)
    const int nl = n_local < 0 ? n : n_local;
    if (nl < 1 || nl > n) return fail(nullptr, MFCFD_ERR_ARG, "n_local out of range [1, n]");
    if (!G.x || !G.y || !G.nx || !G.ny || !G.min_dist || !G.flag_1 || !G.flag_2 || !G.left ||
        !G.right || !G.nbhs || !G.conn)
        return fail(nullptr, MFCFD_ERR_ARG, "a grid array is NULL");
    if (G.ld_conn < n) return fail(nullptr, MFCFD_ERR_ARG, "grid.ld_conn < grid.n");
    if (G.shapes < 1) return fail(nullptr, MFCFD_ERR_ARG, "grid.shapes must be >= 1");
    if (!(P.rks == 1 || P.rks == 4))
        return fail(nullptr, MFCFD_ERR_ARG, "params.rks must be 4 (ssprk43) or 1 (first)");
    if (P.inner_iterations < 0 || P.inner_iterations > 64)
        return fail(nullptr, MFCFD_ERR_ARG, "params.inner_iterations out of range");
    if (!(P.cfl > 0.0) || !isfinite(P.mach) || !isfinite(P.aoa) || !isfinite(P.vl_const) ||
        !isfinite(P.power) || !isfinite(P.euler))
        return fail(nullptr, MFCFD_ERR_ARG, "params: cfl must be > 0 and all finite");
    if (P.precision != MFCFD_FP64 && P.precision != MFCFD_FP32_MIXED)
        return fail(nullptr, MFCFD_ERR_ARG, "params.precision unknown");
    if (P.ordering != MFCFD_ORDER_KIND && P.ordering != MFCFD_ORDER_RCM)
        return fail(nullptr, MFCFD_ERR_ARG, "params.ordering unknown");

    // grid checks (point_preprocessor.F90:32,73 reject bad partitions and shapes)
    int nw = 0, no = 0, kp = 1;
    for (int i = 0; i < nl; ++i) {
        int f = G.flag_1[i], nb = G.nbhs[i];
        if (f < 0 || f > 2) return fail(nullptr, MFCFD_ERR_GRID, "flag_1 must be 0, 1 or 2");
        if (G.flag_2[i] < 0 || G.flag_2[i] > G.shapes)
            return fail(nullptr, MFCFD_ERR_GRID, "shapes value wrong, check again (flag_2)");
        if (nb < 1 || nb > MAXNB)
            return fail(nullptr, MFCFD_ERR_GRID, "nbhs out of range [1, 20]");
        kp = std::max(kp, nb);
        for (int r = 0; r < nb; ++r) {
            int k = G.conn[(size_t)r * G.ld_conn + i];
            if (k < 1 || k > n) return fail(nullptr, MFCFD_ERR_GRID, "conn index out of range");
        }
        if (f != 1) {
            if (G.left[i] < 1 || G.left[i] > n || G.right[i] < 1 || G.right[i] > n)
                return fail(nullptr, MFCFD_ERR_GRID, "left/right out of range on a boundary point");
            (f == 0 ? nw : no) += 1;
        }
    }

    // parameter.F90:16-34
    const double pi = 4.0 * atan(1.0);
    const double theta = P.aoa * pi / 180.0;
    const double q_inf[4] = {1.0, P.mach * cos(theta), P.mach * sin(theta), 1.0 / 1.4};

    // point_normals.F90:8-105 (caller order)
    std::vector<double> nx(n, 0.0), ny(n, 1.0);
    for (int i = 0; i < nl; ++i) {
        int f = G.flag_1[i];
        if (f == 1) {
            if (P.interior_points_normal_flag == 0 && P.format != 2) {
                nx[i] = 0.0;
                ny[i] = 1.0;
            } else if (P.interior_points_normal_flag == 1 && P.format != 2) {
                nx[i] = 1.0;
                ny[i] = 0.0;
            } else {
                nx[i] = G.nx[i];
                ny[i] = G.ny[i];
            }
            continue;
        }
        int l = G.left[i] - 1, r = G.right[i] - 1;
        double lx = G.x[l], ly = G.y[l], mx = G.x[i], my = G.y[i], rx = G.x[r], ry = G.y[r];
        double nx1 = my - ly, nx2 = ry - my, ny1 = mx - lx, ny2 = rx - mx;
        double vx = 0.5 * (nx1 + nx2), vy = 0.5 * (ny1 + ny2);
        double det = sqrt(vx * vx + vy * vy);
        nx[i] = -vx / det;
        ny[i] = vy / det;
    }

    // generate_connectivity.F90:39-256 as bit masks (caller order, caller slots)
    std::vector<unsigned long long> mx(n, 0), my(n, 0);
    for (int i = 0; i < nl; ++i) {
        int f = G.flag_1[i];
        double xi = G.x[i], yi = G.y[i], tx = ny[i], ty = -nx[i];
        unsigned cnt[4] = {0, 0, 0, 0};
        for (int r = 0; r < G.nbhs[i]; ++r) {
            int k = G.conn[(size_t)r * G.ld_conn + i] - 1;
            double delx = G.x[k] - xi, dely = G.y[k] - yi;
            double dels = delx * tx + dely * ty;
            double deln = delx * nx[i] + dely * ny[i];
            if (dels <= 0.0) { mx[i] |= 1ull << r; ++cnt[0]; }
            if (dels >= 0.0) { mx[i] |= 1ull << (32 + r); ++cnt[1]; }
            if (f == 1) {
                if (deln <= 0.0) { my[i] |= 1ull << r; ++cnt[2]; }
                if (deln >= 0.0) { my[i] |= 1ull << (32 + r); ++cnt[3]; }
            } else if (f == 0) {
                my[i] |= 1ull << (32 + r);
                ++cnt[3];
            } else {
                my[i] |= 1ull << r;
                ++cnt[2];
            }
        }
        bool bad = cnt[0] == 0 || cnt[1] == 0 || (f != 0 && cnt[2] == 0) || (f != 2 && cnt[3] == 0);
        if (bad) {
            char msg[160];
            snprintf(msg, sizeof msg,
                     "point %d (flag_1 %d) has an empty split list (xpos %u xneg %u ypos %u yneg %u)",
                     i + 1, f, cnt[0], cnt[1], cnt[2], cnt[3]);
            return fail(nullptr, MFCFD_ERR_GRID, msg);
        }
    }
    // shape points need ring neighbours for ds (compute_force_coeffs.F90:43-62)
    for (int i = 0; i < nl; ++i)
        if (G.flag_2[i] > 0 && (G.left[i] < 1 || G.left[i] > n || G.right[i] < 1 || G.right[i] > n))
            return fail(nullptr, MFCFD_ERR_GRID, "shape point without valid left/right");

    hg.n = n;
    hg.n_local = nl;
    hg.kp = kp;
    hg.nw = nw;
    hg.no = no;
    hg.shapes = G.shapes;
    hg.pi = pi;
    hg.theta = theta;
    hg.cos_t = cos(theta);
    hg.sin_t = sin(theta);
    for (int c = 0; c < 4; ++c) hg.q_inf[c] = q_inf[c];
    // renumbering: new -> caller index
    std::vector<int> base(n);
    if (P.ordering == MFCFD_ORDER_RCM) {
        std::vector<std::vector<int>> adj(n);
        for (int i = 0; i < nl; ++i)
            for (int r = 0; r < G.nbhs[i]; ++r) {
                int k = G.conn[(size_t)r * G.ld_conn + i] - 1;
                if (k == i) continue;
                adj[i].push_back(k);
                adj[k].push_back(i);
            }
        for (auto &a : adj) {
            std::sort(a.begin(), a.end());
            a.erase(std::unique(a.begin(), a.end()), a.end());
        }
        base = rcm_order(n, adj);
    } else {
        for (int i = 0; i < n; ++i) base[i] = i;
    }
    hg.perm.reserve(n);
    for (int want : {0, 2, 1})
        for (int i : base)
            if (i < nl && G.flag_1[i] == want) hg.perm.push_back(i);
    for (int i = nl; i < n; ++i) hg.perm.push_back(i);  // ghosts last, in caller order
    std::vector<int> inv(n);
    for (int p = 0; p < n; ++p) inv[hg.perm[p]] = p;

    // renumbered host arrays
    auto &hxy = hg.xy, &hnrm = hg.nrm;
    auto &heps = hg.eps2, &hobc = hg.obc;
    auto &hconn = hg.conn, &hnb = hg.nbhs;
    auto &hmx = hg.mx, &hmy = hg.my;
    hxy.resize(n); hnrm.resize(n); heps.resize(n); hobc.assign((size_t)8 * std::max(no, 1), 0.0);
    hconn.resize((size_t)kp * n); hnb.resize(n); hmx.resize(n); hmy.resize(n);
    for (int p = 0; p < n; ++p) {
        int i = hg.perm[p];
        hxy[p] = make_double2(G.x[i], G.y[i]);
        hnrm[p] = make_double2(nx[i], ny[i]);
        double epsi = P.vl_const * G.min_dist[i];
        epsi = pow(epsi, 3.0);  // limiters.F90:88-89
        heps[p] = epsi * epsi;
        const int nbi = i < nl ? G.nbhs[i] : 0;  // a ghost has no stencil
        hnb[p] = nbi;
        for (int r = 0; r < kp; ++r) {
            int k = r < nbi ? inv[G.conn[(size_t)r * G.ld_conn + i] - 1] : p;
            hconn[(size_t)r * n + p] = k;
        }
        hmx[p] = mx[i];
        hmy[p] = my[i];
        if (p >= nw && p < nw + no) {
            // state_update.F90:248-263: the freestream half of Ubar
            const double pr_inf = 1.0 / 1.4, rho_inf = 1.0, gamma = 1.4;
            double u1_inf = hg.q_inf[1], u2_inf = hg.q_inf[2];
            double tx = ny[i], ty = -nx[i];
            double u1r = u1_inf * tx + u2_inf * ty;
            double u2r = u1_inf * nx[i] + u2_inf * ny[i];
            double temp1 = (u1r * u1r + u2r * u2r);
            double e_inf = pr_inf / (rho_inf * (gamma - 1.0)) + 0.5 * (temp1);
            double beta = (0.5 * rho_inf) / pr_inf;
            double S2 = u2r * sqrt(beta);
            double B2_inf = exp(-S2 * S2) / (2.0 * sqrt(hg.pi * beta));
            double A2n_inf = 0.5 * (1.0 - erf(S2));
            double *o = &hobc[(size_t)8 * (p - nw)];
            o[0] = u1r; o[1] = u2r; o[2] = e_inf; o[3] = A2n_inf; o[4] = B2_inf;
        }
    }
    // shape points in grid order (compute_force_coeffs.F90:40-78)
    auto &sidx = hg.sidx, &sshape = hg.sshape;
    auto &sgeo = hg.sgeo, &smy = hg.smy;
    for (int i = 0; i < nl; ++i) {
        if (G.flag_2[i] <= 0) continue;
        int l = G.left[i] - 1, r = G.right[i] - 1;
        double lx = G.x[l], ly = G.y[l], mxx = G.x[i], myy = G.y[i], rx = G.x[r], ry = G.y[r];
        double ds1 = (mxx - lx) * (mxx - lx) + (myy - ly) * (myy - ly);
        ds1 = sqrt(ds1);
        double ds2 = (rx - mxx) * (rx - mxx) + (ry - myy) * (ry - myy);
        ds2 = sqrt(ds2);
        double ds = 0.5 * (ds1 + ds2);
        sidx.push_back(inv[i]);
        sshape.push_back(G.flag_2[i] - 1);
        sgeo.insert(sgeo.end(), {nx[i], ny[i], ds, mxx});
        smy.push_back(myy);
    }
    hg.nshape = (int)sidx.size();
    if (P.precision == MFCFD_FP32_MIXED) build_geom32(hg, nw, no, P.power);
    return MFCFD_OK;
}

// ---------------------------------------------------------------------------
// The fixed residue-history array of mfcfd_run_noalloc.
//
// mfcfd_run keeps each call's residue history in a device buffer that it
// grows with cudaMalloc when a call asks for more iterations than any call
// before, and it instantiates CUDA graphs.  Callers that must not allocate
// device memory once they are running -- a Fortran/OpenACC host whose device
// memory belongs to its own pool, a time-critical service that allocates
// only at start-up -- use mfcfd_run_noalloc instead, which keeps the history
// in this array.
//
// In host code the array's name is a host-side stand-in, not a device
// address.  Its address on a device is taken with cudaGetSymbolAddress, with
// that device current, once per device: by the first mfcfd_create on the
// device (set-up time, when the caller allows allocation; the lookup also
// loads this file's module on the device, which places the array).  The
// address is kept in every handle made on the device.
namespace {

constexpr int NOALLOC_MAX_DEVICES = 64;
__device__ __align__(256) double g_noalloc_hist[MFCFD_NOALLOC_MAX_ITERS];

std::mutex g_noalloc_mu;
double *g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {nullptr};

// Called by mfcfd_create with h->dev current.  A failed lookup does not fail
// the create (mfcfd_run does not need the array); mfcfd_run_noalloc reports
// it instead.
void noalloc_resolve(mfcfd_t *h) {
    h->noalloc_hist = nullptr;
    if (h->dev < 0 || h->dev >= NOALLOC_MAX_DEVICES) {
        h->noalloc_err = "mfcfd_run_noalloc: device index out of range";
        return;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[h->dev]) {
        double *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&p), g_noalloc_hist);
        if (e != cudaSuccess) {
            h->noalloc_err = std::string("cudaGetSymbolAddress(g_noalloc_hist): ") +
                             cudaGetErrorString(e);
            return;
        }
        g_noalloc_ptr[h->dev] = p;
    }
    h->noalloc_hist = g_noalloc_ptr[h->dev];
}

}  // namespace

static int create_handle(const mfcfd_grid *grid, const mfcfd_params *params, int n_local,
                         int plen, mfcfd_t **out);

extern "C" {

int mfcfd_create(const mfcfd_grid *grid, const mfcfd_params *params, mfcfd_t **out) {
    return create_handle(grid, params, -1, -1, out);
}

int mfcfd_create_part(const mfcfd_grid *grid, const mfcfd_params *params, int n_local,
                      int plen, mfcfd_t **out) {
    if (out) *out = nullptr;
    if (!grid || !params || !out) return fail(nullptr, MFCFD_ERR_ARG, "NULL argument");
    if (n_local < 1 || n_local > grid->n || plen < n_local)
        return fail(nullptr, MFCFD_ERR_ARG, "need 1 <= n_local <= grid.n and plen >= n_local");
    if (params->precision != MFCFD_FP64)
        return fail(nullptr, MFCFD_ERR_ARG, "a partitioned grid runs the FP64 loop only");
    return create_handle(grid, params, n_local, plen, out);
}

}  // extern "C"

// The body of mfcfd_create; n_local / plen >= 0 make a partitioned handle
// (points [n_local, n) are ghosts; the residual norm divides by plen).
static int create_handle(const mfcfd_grid *grid, const mfcfd_params *params, int n_local,
                         int plen, mfcfd_t **out) {
    mfcfd_t *h = nullptr;
    if (!out) return fail(nullptr, MFCFD_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (!grid || !params) return fail(nullptr, MFCFD_ERR_ARG, "grid or params is NULL");
    const mfcfd_grid &G = *grid;
    const mfcfd_params &P = *params;
    HostGrid hg;
    {
        int st0 = lskum_host::prepare_grid(G, P, hg, n_local);
        if (st0) return st0;
    }
    const int n = hg.n, kp = hg.kp, nw = hg.nw, no = hg.no;
    const int nl = hg.n_local;
    const auto &hxy = hg.xy, &hnrm = hg.nrm;
    const auto &heps = hg.eps2, &hobc = hg.obc;
    const auto &hconn = hg.conn, &hnb = hg.nbhs;
    const auto &hmx = hg.mx, &hmy = hg.my;
    const auto &sidx = hg.sidx, &sshape = hg.sshape;
    const auto &sgeo = hg.sgeo, &smy = hg.smy;
    // host checks done: now the device
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0)
        return fail(nullptr, MFCFD_ERR_NODEV, "no CUDA device");
    {
        cudaError_t e = init_kernels();
        if (e == cudaSuccess) e = init_kernels32();
        if (e != cudaSuccess) return fail(nullptr, MFCFD_ERR_CUDA, cudaGetErrorString(e));
    }
    h = new (std::nothrow) mfcfd();
    if (!h) return fail(nullptr, MFCFD_ERR_OOM, "host allocation failed");
    h->n = n;
    h->n_local = nl;
    h->kp = kp;
    h->nw = nw;
    h->no = no;
    h->nint = nl - nw - no;
    h->shapes = hg.shapes;
    h->nshape = hg.nshape;
    h->perm = std::move(hg.perm);
    h->p = P;
    h->fp32 = P.precision == MFCFD_FP32_MIXED;
    h->left0.assign(G.left, G.left + n);
    h->right0.assign(G.right, G.right + n);
    h->flag2_0.assign(G.flag_2, G.flag_2 + n);
    cudaGetDevice(&h->dev);
    noalloc_resolve(h);
    h->pi = hg.pi;
    h->theta = hg.theta;
    h->cos_t = hg.cos_t;
    h->sin_t = hg.sin_t;
    for (int c = 0; c < 4; ++c) h->q_inf[c] = hg.q_inf[c];

    // device arrays
    HostHalo halo;  // tile halos of the D and I passes
    int st = MFCFD_OK;
    auto up = [&](auto *d, const auto &v) -> int {
        cudaError_t e = cudaMemcpy(d, v.data(), v.size() * sizeof(v[0]), cudaMemcpyHostToDevice);
        return e == cudaSuccess ? MFCFD_OK : cuda_fail(h, e, "cudaMemcpy");
    };
#define ALLOC(ptr, cnt)                                                     \
    do {                                                                    \
        cudaError_t e_ = dmalloc(&(ptr), (size_t)(cnt));                    \
        if (e_ != cudaSuccess) {                                            \
            st = cuda_fail(h, e_, "cudaMalloc " #ptr);                      \
            goto fail_create;                                               \
        }                                                                   \
    } while (0)
    {
        cudaError_t e = cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            st = cuda_fail(h, e, "cudaStreamCreate");
            goto fail_create;
        }
        h->stream = h->own;
    }
    ALLOC(h->d_xy, n);
    ALLOC(h->d_nrm, n);
    ALLOC(h->d_eps2, n);
    ALLOC(h->d_obc, hobc.size());
    ALLOC(h->d_conn, (size_t)kp * n);
    ALLOC(h->d_nbhs, n);
    ALLOC(h->d_mx, n);
    ALLOC(h->d_my, n);
    {
        lskum_host::build_halo(n, kp, hconn.data(), hnb.data(), {{0, nl}}, halo);
        ALLOC(h->d_hoff, halo.off.size());
        ALLOC(h->d_hrow, halo.rows.size());
        ALLOC(h->d_hloc, halo.loc.size());
    }
    if (!h->fp32) {
        for (int b = 0; b < 2; ++b) {
            ALLOC(h->d_prim[b], n);
            ALLOC(h->d_q[b], n);
        }
        for (int b = 0; b < 3; ++b) ALLOC(h->d_dq[b], (size_t)8 * n);
        ALLOC(h->d_qm, (size_t)8 * n);
    } else {
        ALLOC(h->d_prim[0], n);  // FP64 copy of the state for forces/diagnostics
        for (int b = 0; b < 2; ++b) {
            ALLOC(h->f_prim[b], n);
            ALLOC(h->f_q[b], n);
        }
        for (int b = 0; b < 3; ++b) ALLOC(h->f_dq[b], (size_t)8 * n);
        ALLOC(h->f_qm, (size_t)8 * n);
        ALLOC(h->f_eps2, n);
        ALLOC(h->f_dxy, (size_t)kp * n);
        if (!hg.wslot.empty()) ALLOC(h->f_w, (size_t)kp * n);
        ALLOC(h->f_lsq, n);
        ALLOC(h->f_flsq, 2 * (size_t)n);
    }
    ALLOC(h->d_delta, n);
    ALLOC(h->d_spd, n);
    ALLOC(h->d_res_part, flux_blocks(n));
    ALLOC(h->d_forces, 3 * h->shapes + std::max(h->nshape, 1));
    ALLOC(h->d_ctl, 1);
    ALLOC(h->d_inst, 1);
    ALLOC(h->d_sched, SCHED_INTS);
    ALLOC(h->d_run, 1);
    ALLOC(h->d_sh_idx, std::max(h->nshape, 1));
    ALLOC(h->d_sh_shape, std::max(h->nshape, 1));
    ALLOC(h->d_sh_geo, 4 * std::max(h->nshape, 1));
    ALLOC(h->d_sh_my, std::max(h->nshape, 1));
    {
        cudaError_t e = cudaMallocHost(reinterpret_cast<void **>(&h->h_ctl), sizeof(Ctl));
        if (e == cudaSuccess)
            e = cudaMallocHost(reinterpret_cast<void **>(&h->h_sched), sizeof(int) * SCHED_INTS);
        if (e == cudaSuccess)
            e = cudaMallocHost(reinterpret_cast<void **>(&h->h_stage), sizeof(double) * 4 * (size_t)n);
        if (e != cudaSuccess) {
            st = cuda_fail(h, e, "cudaMallocHost");
            goto fail_create;
        }
    }
    if ((st = up(h->d_xy, hxy)) || (st = up(h->d_nrm, hnrm)) || (st = up(h->d_eps2, heps)) ||
        (st = up(h->d_obc, hobc)) || (st = up(h->d_conn, hconn)) || (st = up(h->d_nbhs, hnb)) ||
        (st = up(h->d_mx, hmx)) || (st = up(h->d_my, hmy)))
        goto fail_create;
    if (h->d_hoff && ((st = up(h->d_hoff, halo.off)) || (st = up(h->d_hrow, halo.rows)) ||
                      (st = up(h->d_hloc, halo.loc))))
        goto fail_create;
    if (h->fp32) {
        std::vector<float> feps(heps.begin(), heps.end());
        if ((st = up(h->f_eps2, feps)) || (st = up(h->f_dxy, hg.dxy)) ||
            (st = up(h->f_lsq, hg.lsq)) || (st = up(h->f_flsq, hg.flsq)))
            goto fail_create;
        if (h->f_w && (st = up(h->f_w, hg.wslot))) goto fail_create;
        h->geom32 = Geom32{h->f_dxy, h->f_w, h->f_lsq, h->f_flsq};
    }
    if (h->nshape > 0) {
        if ((st = up(h->d_sh_idx, sidx)) || (st = up(h->d_sh_shape, sshape)) ||
            (st = up(h->d_sh_geo, sgeo)) || (st = up(h->d_sh_my, smy)))
            goto fail_create;
    }
    h->geom = Geom{n, kp, nw, no, h->d_xy, h->d_nrm, h->d_eps2, h->d_conn, h->d_nbhs,
                   h->d_mx, h->d_my, h->d_obc};
    if (h->d_hoff) {
        h->geom.hoff = h->d_hoff;
        h->geom.hrow = h->d_hrow;
        h->geom.hloc = h->d_hloc;
        h->geom.hkp = halo.hkp;
        h->geom.hc = halo.hc;
    }
    h->consts.cfl = P.cfl;
    h->consts.power = P.power;
    h->consts.euler = P.euler;
    h->consts.pi = h->pi;
    h->consts.gm1 = 1.4 - 1;
    h->consts.power_zero = P.power == 0.0 ? 1 : 0;
    h->consts.rks = P.rks;
    h->shape = ShapeTab{h->nshape, h->shapes, h->d_sh_idx, h->d_sh_shape, h->d_sh_geo, h->d_sh_my};
    // the grid as a schedule of one instance; launch shape: one wave of
    // resident blocks per pass (measured 3% faster at 1M points than a
    // block per tile, which reloads the schedule in every block)
    h->inst_h = InstInfo{0, nl, nw, no, 0, 0, flux_blocks(nl), 0};
    h->sched = sched_view(h->d_inst, h->d_sched);
    h->point_block = default_point_block(h->fp32);
    h->point_grid = std::min((nl + h->point_block - 1) / h->point_block,
                             wave_blocks(h->dev, 0, h->point_block, 0, h->fp32));
    h->inner_grid = std::min((nl + h->point_block - 1) / h->point_block,
                             wave_blocks(h->dev, 1, h->point_block, 0, h->fp32));
    h->flux_grid = std::min(flux_grid_blocks(nl),
                            wave_blocks(h->dev, 2, 128,
                                        h->fp32 ? flux32_smem_bytes(kp) : flux_smem_bytes(kp),
                                        h->fp32));
    {
        const BatchRun run{-INFINITY, 0x7fffffff, 0};
        const int one = 1;
        sched_fill(h->h_sched, &h->inst_h, &one, 1);
        cudaError_t e = cudaMemcpy(h->d_inst, &h->inst_h, sizeof(InstInfo), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(h->d_run, &run, sizeof(BatchRun), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(h->d_sched, h->h_sched, sizeof(int) * SCHED_INTS, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            st = cuda_fail(h, e, "cudaMemcpy schedule");
            goto fail_create;
        }
    }
    {
        Ctl c{};
        c.it = 1;
        c.it_first = 1;
        c.restart = P.restart;
        c.plen = plen >= 0 ? plen : n;
        c.res_old = P.res_old;
        *h->h_ctl = c;
        cudaError_t e = cudaMemcpy(h->d_ctl, h->h_ctl, sizeof(Ctl), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            st = cuda_fail(h, e, "cudaMemcpy ctl");
            goto fail_create;
        }
    }
    // initial_conditions.F90:9-20: freestream everywhere
    {
        cudaError_t e;
        if (!h->fp32) {
            for (int p = 0; p < n; ++p)
                for (int c = 0; c < 4; ++c) h->h_stage[4 * (size_t)p + c] = h->q_inf[c];
            e = cudaMemcpy(h->d_prim[0], h->h_stage, sizeof(double) * 4 * (size_t)n,
                           cudaMemcpyHostToDevice);
        } else {
            float *fs = reinterpret_cast<float *>(h->h_stage);
            for (int p = 0; p < n; ++p)
                for (int c = 0; c < 4; ++c) fs[4 * (size_t)p + c] = (float)h->q_inf[c];
            e = cudaMemcpy(h->f_prim[0], fs, sizeof(float) * 4 * (size_t)n, cudaMemcpyHostToDevice);
        }
        if (e != cudaSuccess) {
            st = cuda_fail(h, e, "cudaMemcpy prim");
            goto fail_create;
        }
    }
    if ((st = upload_state_aux(h))) goto fail_create;
    {
        cudaError_t e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) {
            st = cuda_fail(h, e, "create sync");
            goto fail_create;
        }
    }
    *out = h;
    return MFCFD_OK;
fail_create:
    g_create_error = h->err;
    free_all(h);
    delete h;
    return st;
#undef ALLOC
}

extern "C" {

int mfcfd_destroy(mfcfd_t *h) {
    if (!h) return MFCFD_OK;
    cudaStreamSynchronize(h->stream);
    free_all(h);
    delete h;
    return MFCFD_OK;
}

int mfcfd_set_stream(mfcfd_t *h, void *stream) {
    if (!h) return MFCFD_ERR_ARG;
    h->stream = stream ? static_cast<cudaStream_t>(stream) : h->own;
    return MFCFD_OK;
}

}  // extern "C"

namespace {

// Runs fn(begin, end) over [0, n) split into contiguous ranges on up to 8
// host threads (the state copies between the caller's order and the
// renumbered staging buffer are host-memory bound); each range is written by
// one thread only, so the result does not depend on the split.  A thread
// that cannot be created runs its range on the calling thread.
template <class F>
void host_parallel_for(int n, F fn) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int nt = (int)std::min<long long>({8LL, (long long)hw, (long long)n / 65536 + 1});
    if (nt <= 1) {
        fn(0, n);
        return;
    }
    std::vector<std::thread> pool;
    std::vector<int> inline_ranges;
    const int chunk = (n + nt - 1) / nt;
    for (int t = 1; t < nt; ++t) {
        const int b = t * chunk, e = std::min(n, b + chunk);
        if (b >= e) break;
        try {
            pool.emplace_back(fn, b, e);
        } catch (...) {
            inline_ranges.push_back(t);
        }
    }
    fn(0, std::min(n, chunk));
    for (int t : inline_ranges) fn(t * chunk, std::min(n, t * chunk + chunk));
    for (auto &th : pool) th.join();
}

}  // namespace

extern "C" {

int mfcfd_set_state(mfcfd_t *h, const double *prim) {
    if (!h || !prim) return MFCFD_ERR_ARG;
    CK(cudaStreamSynchronize(h->stream));
    if (h->fp32) {
        float *fs = reinterpret_cast<float *>(h->h_stage);
        host_parallel_for(h->n, [&](int b, int e) {
            for (int p = b; p < e; ++p) {
                const double *src = prim + 4 * (size_t)h->perm[p];
                float *dst = fs + 4 * (size_t)p;
                dst[0] = (float)src[0]; dst[1] = (float)src[1]; dst[2] = (float)src[2];
                dst[3] = (float)src[3];
            }
        });
        CK(cudaMemcpyAsync(h->f_prim[h->cur], fs, sizeof(float) * 4 * (size_t)h->n,
                           cudaMemcpyHostToDevice, h->stream));
    } else {
        host_parallel_for(h->n, [&](int b, int e) {
            for (int p = b; p < e; ++p) {
                const double *src = prim + 4 * (size_t)h->perm[p];
                double *dst = h->h_stage + 4 * (size_t)p;
                dst[0] = src[0]; dst[1] = src[1]; dst[2] = src[2]; dst[3] = src[3];
            }
        });
        CK(cudaMemcpyAsync(h->d_prim[h->cur], h->h_stage, sizeof(double) * 4 * (size_t)h->n,
                           cudaMemcpyHostToDevice, h->stream));
    }
    int st = upload_state_aux(h);
    if (st) return st;
    CK(cudaStreamSynchronize(h->stream));
    return MFCFD_OK;
}

int mfcfd_get_state(mfcfd_t *h, double *prim) {
    if (!h || !prim) return MFCFD_ERR_ARG;
    if (h->fp32) {
        float *fs = reinterpret_cast<float *>(h->h_stage);
        CK(cudaMemcpyAsync(fs, h->f_prim[h->cur], sizeof(float) * 4 * (size_t)h->n,
                           cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        host_parallel_for(h->n, [&](int b, int e) {
            for (int p = b; p < e; ++p) {
                const float *src = fs + 4 * (size_t)p;
                double *dst = prim + 4 * (size_t)h->perm[p];
                dst[0] = src[0]; dst[1] = src[1]; dst[2] = src[2]; dst[3] = src[3];
            }
        });
        return MFCFD_OK;
    }
    CK(cudaMemcpyAsync(h->h_stage, h->d_prim[h->cur], sizeof(double) * 4 * (size_t)h->n,
                       cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    host_parallel_for(h->n, [&](int b, int e) {
        for (int p = b; p < e; ++p) {
            const double *src = h->h_stage + 4 * (size_t)p;
            double *dst = prim + 4 * (size_t)h->perm[p];
            dst[0] = src[0]; dst[1] = src[1]; dst[2] = src[2]; dst[3] = src[3];
        }
    });
    return MFCFD_OK;
}

int mfcfd_run(mfcfd_t *h, int it_first, int n_iters, double *residue, int *n_done) {
    if (n_done) *n_done = 0;
    if (!h || n_iters < 0) return MFCFD_ERR_ARG;
    if (h->n_local != h->n)
        return fail(h, MFCFD_ERR_STATE, "a partitioned grid runs with mfcfd_part_phase");
    if (n_iters == 0) return MFCFD_OK;
    // the history buffer and the graphs belong on the handle's device
    DevGuard dg(h->dev);
    CK(dg.err);
    if (n_iters > h->hist_cap) {
        if (h->d_hist) cudaFree(h->d_hist);
        h->d_hist = nullptr;
        h->hist_cap = 0;
        CK(dmalloc(&h->d_hist, (size_t)n_iters));
        h->hist_cap = n_iters;
        drop_graphs(h);  // the graphs hold the old history pointer
    }
    CK(cudaStreamSynchronize(h->stream));
    // reset it .. state and the schedule; res_old stays on the device
    if (int st = lskum_host::reset_run(h, it_first)) return st;
    int rem = n_iters;
    if (rem & 1) {
        if (!h->one_exec[h->cur][h->qcur]) {
            CK(cudaStreamSynchronize(h->stream));
            int st = build_one_graph(h);
            if (st) return st;
        }
        CK(cudaGraphLaunch(h->one_exec[h->cur][h->qcur], h->stream));
        const int c0 = h->cur, q0 = h->qcur;
        h->cur = h->one_next[c0][q0][0];
        h->qcur = h->one_next[c0][q0][1];
        h->launches += (long long)h->p.rks * (2 + h->p.inner_iterations) + 1;
        --rem;
    }
    if (rem > 0) {
        if (!h->pair_exec[h->cur][h->qcur]) {
            // capture on the handle's own stream, ordered after the work above
            CK(cudaStreamSynchronize(h->stream));
            int st = build_pair_graph(h);
            if (st) return st;
        }
        for (int k = 0; k < rem / 2; ++k) {
            CK(cudaGraphLaunch(h->pair_exec[h->cur][h->qcur], h->stream));
            h->launches += 2 * ((long long)h->p.rks * (2 + h->p.inner_iterations) + 1);
        }
    }
    CK(cudaMemcpyAsync(h->h_ctl, h->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    int done = h->h_ctl->done;
    if (residue && done > 0)
        CK(cudaMemcpy(residue, h->d_hist, sizeof(double) * done, cudaMemcpyDeviceToHost));
    if (n_done) *n_done = done;
    h->iters_done_total += done;
    if (h->h_ctl->halted) return fail(h, MFCFD_ERR_NONFINITE, "residue is NaN");
    return MFCFD_OK;
}

int mfcfd_forces(mfcfd_t *h, double *cl, double *cd, double *cm, double *cp) {
    if (!h) return MFCFD_ERR_ARG;
    const R4 *prim = h->d_prim[h->cur];
    if (h->fp32) {
        launch_widen(h->f_prim[h->cur], h->d_prim[0], h->n, h->stream);
        h->launches += 1;
        prim = h->d_prim[0];
    }
    launch_forces(h->shape, prim, h->p.mach, h->cos_t, h->sin_t, h->d_forces, h->stream);
    h->launches += 1;
    CK(cudaGetLastError());
    std::vector<double> o(3 * h->shapes + h->nshape);
    CK(cudaMemcpyAsync(o.data(), h->d_forces, o.size() * sizeof(double), cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (int s = 0; s < h->shapes; ++s) {
        if (cl) cl[s] = o[s];
        if (cd) cd[s] = o[h->shapes + s];
        if (cm) cm[s] = o[2 * h->shapes + s];
    }
    if (cp)
        for (int j = 0; j < h->nshape; ++j) cp[j] = o[3 * h->shapes + j];
    return MFCFD_OK;
}

int mfcfd_keep_diagnostics(mfcfd_t *h, int on) {
    if (!h) return MFCFD_ERR_ARG;
    bool want = on != 0;
    if (want && !h->d_flux_dbg) CK(dmalloc(&h->d_flux_dbg, (size_t)4 * h->n));
    if (want != h->keep_diag) drop_graphs(h);
    h->keep_diag = want;
    return MFCFD_OK;
}

int mfcfd_get_array(mfcfd_t *h, const char *name, double *out) {
    if (!h || !name || !out) return MFCFD_ERR_ARG;
    const double *src = nullptr;
    int w = 0;
    std::string s(name);
    const float *fsrc = nullptr;
    if (h->fp32) {
        if (s == "q") { fsrc = reinterpret_cast<const float *>(h->f_q[h->qcur ^ 1]); w = 4; }
        else if (s == "dq") { fsrc = h->f_dq[dq32_final(h->p.inner_iterations)]; w = 8; }
        else if (s == "qm") { fsrc = h->f_qm; w = 8; }
    }
    if (fsrc) {
        std::vector<float> ft((size_t)w * h->n);
        CK(cudaMemcpyAsync(ft.data(), fsrc, ft.size() * sizeof(float), cudaMemcpyDeviceToHost,
                           h->stream));
        CK(cudaStreamSynchronize(h->stream));
        for (int p = 0; p < h->n; ++p)
            for (int c = 0; c < w; ++c) {
                int cc = w == 8 ? (c % 4) * 2 + c / 4 : c;
                out[(size_t)w * h->perm[p] + cc] = ft[(size_t)w * p + c];
            }
        return MFCFD_OK;
    }
    if (s == "q") { src = reinterpret_cast<const double *>(h->d_q[h->qcur ^ 1]); w = 4; }
    else if (s == "dq") { src = h->d_dq[dq_final(h->p.inner_iterations)]; w = 8; }
    else if (s == "qm") { src = h->d_qm; w = 8; }
    else if (s == "delta") { src = h->d_delta; w = 1; }
    else if (s == "flux_res") {
        if (!h->d_flux_dbg) return fail(h, MFCFD_ERR_STATE, "flux_res needs mfcfd_keep_diagnostics");
        src = h->d_flux_dbg; w = 4;
    } else if (s == "nx" || s == "ny") {
        src = reinterpret_cast<const double *>(h->d_nrm); w = 2;
    } else {
        return fail(h, MFCFD_ERR_ARG, "unknown array name");
    }
    std::vector<double> tmp((size_t)w * h->n);
    CK(cudaMemcpyAsync(tmp.data(), src, tmp.size() * sizeof(double), cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (s == "nx" || s == "ny") {
        int off = s == "nx" ? 0 : 1;
        for (int p = 0; p < h->n; ++p) out[h->perm[p]] = tmp[2 * (size_t)p + off];
        return MFCFD_OK;
    }
    for (int p = 0; p < h->n; ++p)
        for (int c = 0; c < w; ++c) {
            int cc = c;
            if (w == 8) cc = (c % 4) * 2 + c / 4;  // [dx1..4, dy1..4] -> Fortran (2,4)
            out[(size_t)w * h->perm[p] + cc] = tmp[(size_t)w * p + c];
        }
    return MFCFD_OK;
}

int mfcfd_info(mfcfd_t *h, int *n, int *n_wall, int *n_outer, int *n_interior) {
    if (!h) return MFCFD_ERR_ARG;
    if (n) *n = h->n;
    if (n_wall) *n_wall = h->nw;
    if (n_outer) *n_outer = h->no;
    if (n_interior) *n_interior = h->nint;
    return MFCFD_OK;
}

long long mfcfd_launch_count(mfcfd_t *h) { return h ? h->launches : 0; }

int mfcfd_profile_iteration(mfcfd_t *h, int it, double *ms) {
    if (!h || !ms) return MFCFD_ERR_ARG;
    const int m = h->p.inner_iterations;
    const int nev = h->p.rks * (2 + m) + 2;
    std::vector<cudaEvent_t> ev(nev);
    for (auto &e : ev) CK(cudaEventCreate(&e));
    CK(cudaStreamSynchronize(h->stream));
    if (h->hist_cap < 1) {
        CK(dmalloc(&h->d_hist, 1));
        h->hist_cap = 1;
    }
    if (int st = lskum_host::reset_run(h, it)) return st;
    const int A = h->cur, B = h->cur ^ 1;
    int e = 0;
    CK(cudaEventRecord(ev[e++], h->stream));
    for (int rk = 1; rk <= h->p.rks; ++rk)
        launch_stage(h, h->stream, rk, A, B, [&] { cudaEventRecord(ev[e++], h->stream); });
    launch_residual(h->d_inst, 1, h->d_res_part, h->d_ctl, h->d_hist, 0, h->d_run, h->d_sched,
                    h->stream);
    CK(cudaEventRecord(ev[e++], h->stream));
    h->launches += 1;
    h->cur = B;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    double sum[4] = {0, 0, 0, 0};
    int cnt[4] = {0, 0, 0, 0};
    e = 1;
    auto span = [&](int k) {
        float t = 0.f;
        cudaEventElapsedTime(&t, ev[k - 1], ev[k]);
        return (double)t;
    };
    for (int rk = 1; rk <= h->p.rks; ++rk) {
        sum[0] += span(e++); cnt[0]++;
        for (int t = 1; t <= m; ++t) { sum[1] += span(e++); cnt[1]++; }
        sum[2] += span(e++); cnt[2]++;
    }
    sum[3] += span(e++); cnt[3]++;
    for (int k = 0; k < 4; ++k) ms[k] = cnt[k] ? sum[k] / cnt[k] : 0.0;
    float tot = 0.f;
    cudaEventElapsedTime(&tot, ev[0], ev[nev - 1]);
    ms[4] = tot;
    for (auto &x : ev) cudaEventDestroy(x);
    return MFCFD_OK;
}

const char *mfcfd_strerror(int status) {
    switch (status) {
    case MFCFD_OK: return "ok";
    case MFCFD_ERR_ARG: return "invalid argument";
    case MFCFD_ERR_CUDA: return "CUDA runtime error";
    case MFCFD_ERR_NONFINITE: return "residue became NaN";
    case MFCFD_ERR_TIMEOUT: return "bounded device wait timed out";
    case MFCFD_ERR_OOM: return "device out of memory";
    case MFCFD_ERR_GRID: return "invalid or singular grid";
    case MFCFD_ERR_NODEV: return "no usable CUDA device";
    case MFCFD_ERR_STATE: return "call not valid in this state";
    default: return "unknown status";
    }
}

const char *mfcfd_last_error(mfcfd_t *h) {
    return h ? h->err.c_str() : g_create_error.c_str();
}

}  // extern "C"

// ---------------------------------------------------------------------------
// mfcfd_run_noalloc: the pseudo-time loop without any device allocation.
// It launches the same kernels as mfcfd_run, one iteration after another
// (no graph instantiation), with the history written to the array above,
// whose address mfcfd_create resolved.  Every call on a device shares the
// array: each iteration writes its history entry before anything reads it,
// and calls that overlap on the GPU (two handles on concurrent streams) race
// on it.
extern "C" int mfcfd_run_noalloc(mfcfd_t *h, int it_first, int n_iters, double *residue,
                                 int *n_done) {
    if (n_done) *n_done = 0;
    if (!h || n_iters < 0) return MFCFD_ERR_ARG;
    if (n_iters > MFCFD_NOALLOC_MAX_ITERS)
        return fail(h, MFCFD_ERR_ARG,
                    "mfcfd_run_noalloc: n_iters exceeds MFCFD_NOALLOC_MAX_ITERS (65536); "
                    "split the run into several calls");
    if (h->n_local != h->n)
        return fail(h, MFCFD_ERR_STATE, "a partitioned grid runs with mfcfd_part_phase");
    if (n_iters == 0) return MFCFD_OK;
    double *hist = h->noalloc_hist;
    if (!hist) return fail(h, MFCFD_ERR_CUDA, h->noalloc_err);
    DevGuard dg(h->dev);
    CK(dg.err);
    CK(cudaStreamSynchronize(h->stream));
    if (int st = lskum_host::reset_run(h, it_first)) return st;
    for (int k = 0; k < n_iters; ++k)
        if (int st = enqueue_iteration_to(h, h->stream, hist)) return st;
    CK(cudaMemcpyAsync(h->h_ctl, h->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    const int done = h->h_ctl->done;
    if (residue && done > 0)
        CK(cudaMemcpy(residue, hist, sizeof(double) * done, cudaMemcpyDeviceToHost));
    if (n_done) *n_done = done;
    h->iters_done_total += done;
    if (h->h_ctl->halted) return fail(h, MFCFD_ERR_NONFINITE, "residue is NaN");
    return MFCFD_OK;
}

// ---------------------------------------------------------------------------
// A partitioned grid, one phase at a time (the reference's multi-rank
// fpi_solver, fpi_solver.F90:13-83 with the ghost updates of :34-52).  The
// handle owns points [0, n_local) of its grid; the rest are ghosts whose
// rows the caller refreshes from their owners between phases (PETSc's
// VecGhostUpdate): dq and qm after MFCFD_PHASE_GRAD, dq after each
// MFCFD_PHASE_INNER, prim after MFCFD_PHASE_FLUX followed by
// MFCFD_PHASE_GHOSTS.  Kernels are the single-grid ones over the owned
// points' tiles; ghost rows are read, never written, by them.
namespace {

int part_check(mfcfd_t *h) {
    if (!h) return MFCFD_ERR_ARG;
    if (h->fp32) return fail(h, MFCFD_ERR_STATE, "phases run the FP64 loop only");
    return MFCFD_OK;
}

}  // namespace

extern "C" int mfcfd_part_phase(mfcfd_t *h, int phase, int rk, int t, double *value) {
    if (int st = part_check(h)) return st;
    DevGuard dg(h->dev);
    CK(dg.err);
    cudaStream_t s = h->stream;
    const int m = h->p.inner_iterations;
    if (phase != MFCFD_PHASE_BEGIN && !h->part_in_iter)
        return fail(h, MFCFD_ERR_STATE, "phase outside an iteration (MFCFD_PHASE_BEGIN first)");
    if ((phase == MFCFD_PHASE_GRAD || phase == MFCFD_PHASE_INNER || phase == MFCFD_PHASE_FLUX) &&
        (rk < 1 || rk > h->p.rks))
        return fail(h, MFCFD_ERR_ARG, "rk out of range");
    const int A = h->part_A, B = A ^ 1;
    switch (phase) {
    case MFCFD_PHASE_BEGIN:
        if (!h->d_part_sum) CK(lskum_host::dmalloc(&h->d_part_sum, 1));
        h->part_A = h->cur;
        h->part_in_iter = true;
        return MFCFD_OK;
    case MFCFD_PHASE_GRAD:
        launch_grad(h->geom, h->consts, h->sched, h->d_q[h->qcur], h->d_spd, h->d_dq[0],
                    h->d_qm, h->d_delta, rk == 1, h->point_block, h->point_grid, s);
        h->part_dq = 0;
        break;
    case MFCFD_PHASE_INNER:
        if (t < 1 || t > m) return fail(h, MFCFD_ERR_ARG, "inner iteration t out of range");
        launch_inner(h->geom, h->consts, h->sched, h->d_dq[0], h->d_dq[dq_src(t)],
                     h->d_dq[dq_dst(t)], h->point_block, h->inner_grid, s);
        h->part_dq = dq_dst(t);
        break;
    case MFCFD_PHASE_FLUX: {
        StageBufs b;
        b.prim_in = rk == 1 ? h->d_prim[A] : h->d_prim[B];
        b.prim_out = h->d_prim[B];
        b.prim_old = h->d_prim[A];
        b.q_in = h->d_q[h->qcur];
        b.q_out = h->d_q[h->qcur ^ 1];
        b.dq = h->d_dq[dq_final(m)];
        b.qm = h->d_qm;
        b.delta = h->d_delta;
        b.spd = h->d_spd;
        b.res_part = h->d_res_part;
        b.flux_dbg = h->keep_diag ? h->d_flux_dbg : nullptr;
        launch_flux(h->geom, h->consts, h->sched, b, rk, rk == h->p.rks, h->flux_grid, s);
        h->qcur ^= 1;
        break;
    }
    case MFCFD_PHASE_GHOSTS:
        launch_init_rows(h->geom, h->d_prim[B], h->d_q[h->qcur], h->d_spd, h->n_local, h->n, s);
        break;
    case MFCFD_PHASE_END:
        launch_sum_parts(h->d_res_part, h->inst_h.ntiles, h->d_part_sum, s);
        CK(cudaGetLastError());
        if (value) {
            CK(cudaMemcpyAsync(value, h->d_part_sum, sizeof(double), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
        }
        h->cur = B;
        h->part_in_iter = false;
        h->launches += 1;
        h->iters_done_total += 1;
        return MFCFD_OK;
    default:
        return fail(h, MFCFD_ERR_ARG, "unknown phase");
    }
    h->launches += 1;
    CK(cudaGetLastError());
    return MFCFD_OK;
}

extern "C" int mfcfd_part_rows(mfcfd_t *h, const char *name, void **rows, int *row_doubles) {
    if (int st = part_check(h)) return st;
    if (!name || !rows) return fail(h, MFCFD_ERR_ARG, "NULL argument");
    const int B = h->part_in_iter ? (h->part_A ^ 1) : h->cur;
    if (!strcmp(name, "prim")) {
        *rows = h->d_prim[B];
        if (row_doubles) *row_doubles = 4;
    } else if (!strcmp(name, "dq")) {
        *rows = h->d_dq[h->part_dq];
        if (row_doubles) *row_doubles = 8;
    } else if (!strcmp(name, "qm")) {
        *rows = h->d_qm;
        if (row_doubles) *row_doubles = 8;
    } else {
        return fail(h, MFCFD_ERR_ARG, "rows: prim, dq or qm");
    }
    return MFCFD_OK;
}

extern "C" int mfcfd_part_index(mfcfd_t *h, int *internal) {
    if (!h || !internal) return MFCFD_ERR_ARG;
    for (int p = 0; p < h->n; ++p) internal[h->perm[p]] = p;
    return MFCFD_OK;
}
