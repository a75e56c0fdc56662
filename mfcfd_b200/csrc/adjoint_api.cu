// mfcfd_adjoint: reverse-mode derivative of the pseudo-time loop.
//
// Replaces the reference's q_lskum_chkpts_b + REVOLV driver
// (src_mpi_adjoint/sensitivity_files/q_lskum_chkpts_b.F90:23-300,
// src_mpi_adjoint/revolve.f:347-591) and FPI_SOLVER_B
// (fpi_solver_b.F90:28-156).  From the handle's current state prim_0 (held
// fixed) it runs n iterations, takes J = sum over shapes of Cl or Cd of the
// final state (the reference seeds vector_cost_funcb = 1 for J = Cd,
// objective_function_b.F90:22-33) and returns dJ/dx, dJ/dy per point.
//
// Checkpointing: prim snapshots (32 bytes a point) in HBM, placed by a
// binomial schedule (Griewank's reversal with s snapshots and t sweeps
// reverses C(s+t, t) iterations) within the caller's byte budget.  Each
// iteration is re-run forward from its snapshot with every stage input taped
// in HBM, then reversed stage by stage.
#include <cuda_runtime.h>

#include <algorithm>
#include <thread>
#include <vector>

#include "adjoint.h"
#include "handle.h"
#include "objective.h"

using namespace lskum;
using lskum_host::cuda_fail;
using lskum_host::dmalloc;
using lskum_host::fail;

struct AdjointState {
    int n = 0, kp = 0, m = 0, rks = 0;
    int *d_tptr = nullptr, *d_tlist = nullptr;
    int nshape = 0;
    int *d_sidx = nullptr, *d_sleft = nullptr, *d_sright = nullptr;
    double *d_snx = nullptr, *d_sny = nullptr;
    int nbnd = 0;
    int *d_bleft = nullptr, *d_bright = nullptr;
    // source lists of the gather forms of the force / normal reverses
    // (null: the single-thread kernels run)
    int *d_fptr = nullptr, *d_fsrc = nullptr, *d_nptr = nullptr, *d_nsrc = nullptr;
    R4 *tprim[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    R4 *tq[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    R4 *tfr[4] = {nullptr, nullptr, nullptr, nullptr};
    double *tdq = nullptr, *tqm = nullptr, *tdelta = nullptr, *tspd = nullptr;
    double *pb[2] = {nullptr, nullptr}, *pbA = nullptr;
    double *qb = nullptr, *dqb[2] = {nullptr, nullptr}, *qmb = nullptr, *deltab = nullptr;
    double *frb = nullptr, *xb = nullptr, *yb = nullptr, *nxb = nullptr, *nyb = nullptr;
    double *contrib = nullptr;
    // kinetic-state tape of the re-run (rks stages of [n][kp][KS_TAPE]); null
    // when it did not fit, and the reverse flux pass recomputes the states
    double *tks = nullptr;
    double *hist = nullptr;
    int hist_cap = 0;
    std::vector<R4 *> snaps;  // snapshot rows (n points each) in one device block
    R4 *snap_pool = nullptr;
    R4 *snap0 = nullptr;      // the initial state
    R4 *fin = nullptr;        // the final state
    // run bookkeeping
    int n_iters = 0, objective = 1;
    double J = 0.0;
    long long forward_iters = 0;
};

namespace {

double *dq_at(AdjointState *a, int rk, int t) {
    return a->tdq + ((size_t)(rk - 1) * (a->m + 1) + t) * 8 * (size_t)a->n;
}
double *qm_at(AdjointState *a, int rk) { return a->tqm + (size_t)(rk - 1) * 8 * (size_t)a->n; }

int adj_setup(mfcfd_t *h) {
    if (h->adj) return MFCFD_OK;
    AdjointState *a = new AdjointState();
    h->adj = a;
    const int n = h->n, kp = h->kp, m = h->p.inner_iterations, rks = h->p.rks;
    a->n = n;
    a->kp = kp;
    a->m = m;
    a->rks = rks;
    // transposed stencil: for each point k the (i, r) with conn[r][i] = k,
    // in increasing (i, r) order
    std::vector<int> hconn((size_t)kp * n), hnb(n);
    CK(cudaMemcpy(hconn.data(), h->d_conn, hconn.size() * sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(hnb.data(), h->d_nbhs, hnb.size() * sizeof(int), cudaMemcpyDeviceToHost));
    std::vector<int> tptr(n + 1, 0), tlist;
    for (int i = 0; i < n; ++i)
        for (int r = 0; r < hnb[i]; ++r) tptr[hconn[(size_t)r * n + i] + 1]++;
    for (int k = 0; k < n; ++k) tptr[k + 1] += tptr[k];
    tlist.resize(tptr[n]);
    std::vector<int> fill(tptr.begin(), tptr.end() - 1);
    for (int i = 0; i < n; ++i)
        for (int r = 0; r < hnb[i]; ++r) tlist[fill[hconn[(size_t)r * n + i]]++] = i * kp + r;
    CK(dmalloc(&a->d_tptr, n + 1));
    CK(dmalloc(&a->d_tlist, tlist.size()));
    CK(cudaMemcpy(a->d_tptr, tptr.data(), tptr.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(a->d_tlist, tlist.data(), tlist.size() * sizeof(int), cudaMemcpyHostToDevice));
    // renumbered ring neighbours and shape table
    std::vector<int> inv(n);
    for (int p = 0; p < n; ++p) inv[h->perm[p]] = p;
    a->nbnd = h->nw + h->no;
    std::vector<int> bl(std::max(a->nbnd, 1)), br(std::max(a->nbnd, 1));
    for (int p = 0; p < a->nbnd; ++p) {
        bl[p] = inv[h->left0[h->perm[p]] - 1];
        br[p] = inv[h->right0[h->perm[p]] - 1];
    }
    std::vector<double2> hnrm(n);
    CK(cudaMemcpy(hnrm.data(), h->d_nrm, n * sizeof(double2), cudaMemcpyDeviceToHost));
    std::vector<int> si, sl, sr;
    std::vector<double> snx, sny;
    for (int i = 0; i < n; ++i) {
        if (h->flag2_0[i] <= 0) continue;
        const int p = inv[i];
        si.push_back(p);
        sl.push_back(inv[h->left0[i] - 1]);
        sr.push_back(inv[h->right0[i] - 1]);
        snx.push_back(hnrm[p].x);
        sny.push_back(hnrm[p].y);
    }
    a->nshape = (int)si.size();
    const size_t ns = std::max(a->nshape, 1);
    CK(dmalloc(&a->d_bleft, bl.size()));
    CK(dmalloc(&a->d_bright, br.size()));
    CK(dmalloc(&a->d_sidx, ns));
    CK(dmalloc(&a->d_sleft, ns));
    CK(dmalloc(&a->d_sright, ns));
    CK(dmalloc(&a->d_snx, ns));
    CK(dmalloc(&a->d_sny, ns));
    CK(cudaMemcpy(a->d_bleft, bl.data(), bl.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(a->d_bright, br.data(), br.size() * sizeof(int), cudaMemcpyHostToDevice));
    if (a->nshape) {
        CK(cudaMemcpy(a->d_sidx, si.data(), ns * sizeof(int), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(a->d_sleft, sl.data(), ns * sizeof(int), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(a->d_sright, sr.data(), ns * sizeof(int), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(a->d_snx, snx.data(), ns * sizeof(double), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(a->d_sny, sny.data(), ns * sizeof(double), cudaMemcpyHostToDevice));
    }
    // per boundary point q, the entries j of the force and normal reverses
    // that add to xb[q] / yb[q], in the serial loops' order (ascending j, and
    // within one j the order of its statements)
    {
        const int nb = a->nbnd;
        std::vector<std::vector<int>> nl(std::max(nb, 1)), fl(std::max(nb, 1));
        bool n_ok = nb > 0, f_ok = nb > 0;
        for (int j = 0; j < nb && n_ok; ++j) {
            if (br[j] < 0 || br[j] >= nb || bl[j] < 0 || bl[j] >= nb) n_ok = false;
            else {
                nl[br[j]].push_back(2 * j);
                nl[bl[j]].push_back(2 * j + 1);
            }
        }
        for (int j = 0; j < a->nshape && f_ok; ++j) {
            const int tgt[3] = {si[j], sl[j], sr[j]};
            for (int role = 0; role < 3; ++role) {
                if (tgt[role] < 0 || tgt[role] >= nb) { f_ok = false; break; }
                fl[tgt[role]].push_back(3 * j + role);
            }
        }
        auto upload_csr = [&](const std::vector<std::vector<int>> &lists, int **d_ptr,
                              int **d_src) -> int {
            std::vector<int> ptr(nb + 1, 0), src;
            for (int q = 0; q < nb; ++q) {
                ptr[q + 1] = ptr[q] + (int)lists[q].size();
                src.insert(src.end(), lists[q].begin(), lists[q].end());
            }
            if (src.empty()) src.push_back(0);
            CK(dmalloc(d_ptr, ptr.size()));
            CK(dmalloc(d_src, src.size()));
            CK(cudaMemcpy(*d_ptr, ptr.data(), ptr.size() * sizeof(int), cudaMemcpyHostToDevice));
            CK(cudaMemcpy(*d_src, src.data(), src.size() * sizeof(int), cudaMemcpyHostToDevice));
            return MFCFD_OK;
        };
        int st = MFCFD_OK;
        if (n_ok && (st = upload_csr(nl, &a->d_nptr, &a->d_nsrc))) return st;
        if (f_ok && (st = upload_csr(fl, &a->d_fptr, &a->d_fsrc))) return st;
    }
    // tape of one iteration and the adjoint arrays
    for (int s = 0; s <= rks; ++s) {
        CK(dmalloc(&a->tprim[s], n));
        CK(dmalloc(&a->tq[s], n));
    }
    for (int s = 0; s < rks; ++s) CK(dmalloc(&a->tfr[s], n));
    CK(dmalloc(&a->tdq, (size_t)rks * (m + 1) * 8 * n));
    CK(dmalloc(&a->tqm, (size_t)rks * 8 * n));
    CK(dmalloc(&a->tdelta, n));
    CK(dmalloc(&a->tspd, n));
    for (int b = 0; b < 2; ++b) {
        CK(dmalloc(&a->pb[b], (size_t)4 * n));
        CK(dmalloc(&a->dqb[b], (size_t)8 * n));
    }
    CK(dmalloc(&a->pbA, (size_t)4 * n));
    CK(dmalloc(&a->qb, (size_t)4 * n));
    CK(dmalloc(&a->qmb, (size_t)8 * n));
    CK(dmalloc(&a->deltab, n));
    CK(dmalloc(&a->frb, (size_t)4 * n));
    CK(dmalloc(&a->xb, n));
    CK(dmalloc(&a->yb, n));
    CK(dmalloc(&a->nxb, n));
    CK(dmalloc(&a->nyb, n));
    CK(dmalloc(&a->contrib, (size_t)n * kp * ADJ_CW));
    if (dmalloc(&a->tks, (size_t)rks * n * kp * KS_TAPE) != cudaSuccess) {
        a->tks = nullptr;
        cudaGetLastError();  // an allocation failure is not sticky; clear it
    }
    CK(dmalloc(&a->snap0, n));
    CK(dmalloc(&a->fin, n));
    cudaError_t e = init_adjoint_kernels();
    if (e != cudaSuccess) return cuda_fail(h, e, "init_adjoint_kernels");
    return MFCFD_OK;
}

int reset_ctl(mfcfd_t *h) { return lskum_host::reset_run(h, 1); }

// The kinetic-state tape of stage rk (1-based), or nullptr.
double *ks_at(AdjointState *a, int rk) {
    return a->tks ? a->tks + (size_t)(rk - 1) * a->n * a->kp * KS_TAPE : nullptr;
}

// Runs k plain iterations from state `from` and stores the result in `to`.
int advance(mfcfd_t *h, AdjointState *a, const R4 *from, int k, R4 *to) {
    const size_t bytes = sizeof(R4) * (size_t)a->n;
    CK(cudaMemcpyAsync(h->d_prim[h->cur], from, bytes, cudaMemcpyDeviceToDevice, h->stream));
    int st = lskum_host::upload_state_aux(h);
    if (st) return st;
    if ((st = reset_ctl(h))) return st;
    for (int j = 0; j < k; ++j) {
        if ((st = lskum_host::enqueue_iteration_to(h, h->stream, a->hist))) return st;
    }
    a->forward_iters += k;
    CK(cudaMemcpyAsync(to, h->d_prim[h->cur], bytes, cudaMemcpyDeviceToDevice, h->stream));
    return MFCFD_OK;
}

// One forward iteration from `from` with every stage input taped.
int record(mfcfd_t *h, AdjointState *a, const R4 *from) {
    const size_t bytes = sizeof(R4) * (size_t)a->n;
    const int m = a->m, rks = a->rks;
    int st = reset_ctl(h);
    if (st) return st;
    CK(cudaMemcpyAsync(a->tprim[0], from, bytes, cudaMemcpyDeviceToDevice, h->stream));
    launch_init_state(h->geom, a->tprim[0], a->tq[0], a->tspd, h->stream);
    for (int rk = 1; rk <= rks; ++rk) {
        launch_grad(h->geom, h->consts, h->sched, a->tq[rk - 1], a->tspd, dq_at(a, rk, 0),
                    qm_at(a, rk), a->tdelta, rk == 1, h->point_block, h->point_grid, h->stream);
        for (int t = 1; t <= m; ++t)
            launch_inner(h->geom, h->consts, h->sched, dq_at(a, rk, 0), dq_at(a, rk, t - 1),
                         dq_at(a, rk, t), h->point_block, h->inner_grid, h->stream);
        StageBufs b;
        b.prim_in = a->tprim[rk - 1];
        b.prim_out = a->tprim[rk];
        b.prim_old = a->tprim[0];
        b.q_in = a->tq[rk - 1];
        b.q_out = a->tq[rk];
        b.dq = dq_at(a, rk, m);
        b.qm = qm_at(a, rk);
        b.delta = a->tdelta;
        // tspd keeps the input state's spd for the reverse of func_delta; the
        // last stage's spd of the output goes to the handle's own buffer
        // (rebuilt when the adjoint restores the state)
        b.spd = h->d_spd;
        b.res_part = h->d_res_part;
        b.flux_dbg = reinterpret_cast<double *>(a->tfr[rk - 1]);
        b.kstape = ks_at(a, rk);
        launch_flux(h->geom, h->consts, h->sched, b, rk, rk == rks, h->flux_grid, h->stream);
    }
    h->launches += 1 + (long long)rks * (2 + m);
    a->forward_iters += 1;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(h, e, "adjoint record launch");
    return MFCFD_OK;
}

// Reverse of one taped iteration: pb[0] holds the adjoint of its output on
// entry and of its input on exit.
int reverse_taped(mfcfd_t *h, AdjointState *a) {
    const int n = a->n, m = a->m, rks = a->rks;
    cudaStream_t s = h->stream;
    AdjConsts ac{{h->q_inf[0], h->q_inf[1], h->q_inf[2], h->q_inf[3]}};
    CK(cudaMemsetAsync(a->pbA, 0, sizeof(double) * 4 * n, s));
    CK(cudaMemsetAsync(a->deltab, 0, sizeof(double) * n, s));
    int out = 0;  // pb[out] = adjoint of the current stage's output
    for (int rk = rks; rk >= 1; --rk) {
        double *pb_out = a->pb[out];
        double *pb_in = rk == 1 ? a->pbA : a->pb[out ^ 1];
        if (rk != 1) CK(cudaMemsetAsync(pb_in, 0, sizeof(double) * 4 * n, s));
        launch_update_b(h->geom, h->consts, ac, a->tprim[rk - 1], a->tprim[0], a->tfr[rk - 1],
                        pb_out, pb_in, a->pbA, a->frb, a->nxb, a->nyb, rk, s);
        CK(cudaMemsetAsync(a->qb, 0, sizeof(double) * 4 * n, s));
        CK(cudaMemsetAsync(a->qmb, 0, sizeof(double) * 8 * n, s));
        CK(cudaMemsetAsync(a->dqb[m & 1], 0, sizeof(double) * 8 * n, s));
        launch_flux_b(h->geom, h->consts, a->tq[rk - 1], dq_at(a, rk, m), qm_at(a, rk), a->tdelta,
                      a->frb, a->qb, a->dqb[m & 1], a->qmb, a->xb, a->yb, a->nxb, a->nyb,
                      a->deltab, a->contrib, a->contrib + (size_t)n * a->kp * NBREC, a->d_tptr,
                      a->d_tlist, ks_at(a, rk), s);
        for (int t = m; t >= 1; --t) {
            launch_inner_b(h->geom, a->tq[rk - 1], dq_at(a, rk, t - 1), a->dqb[t & 1],
                           a->dqb[(t - 1) & 1], a->qb, a->xb, a->yb, a->contrib, s);
            launch_gather(n, a->kp, a->d_tptr, a->d_tlist, a->contrib, ADJ_GATHER_INNER, a->qb,
                          a->dqb[(t - 1) & 1], nullptr, a->xb, a->yb, s);
        }
        launch_grad_b(h->geom, h->consts, a->tq[rk - 1], a->tprim[0], a->tspd, a->dqb[0],
                      a->qmb, a->deltab, rk == 1, a->qb, a->pbA, a->xb, a->yb, a->contrib,
                      a->d_tptr, a->d_tlist, s);
        launch_qvar_b(n, a->tprim[rk - 1], a->qb, pb_in, s);
        h->launches += 7 + 2LL * m;
        out ^= 1;
    }
    CK(cudaMemcpyAsync(a->pb[0], a->pbA, sizeof(double) * 4 * n, cudaMemcpyDeviceToDevice, s));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(h, e, "adjoint reverse launch");
    return MFCFD_OK;
}

// Reverse of iteration k from its input state: tapes it; the last iteration
// also seeds the adjoint from the objective of its output.
int reverse_iteration(mfcfd_t *h, AdjointState *a, int k, const R4 *state) {
    int st = record(h, a, state);
    if (st) return st;
    if (k == a->n_iters - 1) {
        const int n = a->n;
        cudaStream_t s = h->stream;
        CK(cudaMemsetAsync(a->pb[0], 0, sizeof(double) * 4 * n, s));
        if (a->objective == MFCFD_OBJ_CL || a->objective == MFCFD_OBJ_CD) {
            AdjShape t{a->nshape, a->d_sidx, a->d_sleft, a->d_sright, a->d_snx, a->d_sny};
            const AdjGather gth{a->nbnd, a->d_fptr, a->d_fsrc, a->d_nptr, a->d_nsrc};
            launch_forces_b(t, gth, a->tprim[a->rks], h->d_xy, h->p.mach, h->cos_t, h->sin_t,
                            a->objective, a->pb[0], a->xb, a->yb, a->nxb, a->nyb, s);
        } else {
            lskum_host::launch_objective_b(h, a->objective, a->tprim[a->rks], a->pb[0], a->xb,
                                           a->yb, a->contrib, s);
            if (a->objective == MFCFD_OBJ_ENSTROPHY) {
                launch_gather(n, a->kp, a->d_tptr, a->d_tlist, a->contrib, ADJ_GATHER_GRAD, a->qb,
                              nullptr, a->pb[0], a->xb, a->yb, s);
                h->launches += 1;
            }
        }
        // keep the final state: the handle holds it at the end, as after mfcfd_run
        CK(cudaMemcpyAsync(a->fin, a->tprim[a->rks], sizeof(R4) * (size_t)n,
                           cudaMemcpyDeviceToDevice, s));
        h->launches += 1;
    }
    return reverse_taped(h, a);
}

long long binom(int s, int t) {
    long long r = 1;
    for (int j = 1; j <= t; ++j) {
        r = r * (s + j) / j;
        if (r > (1LL << 40)) return 1LL << 40;
    }
    return r;
}

// Reverses iterations [lo, hi) whose input state lo is held in `state`.
int reverse_range(mfcfd_t *h, AdjointState *a, int lo, int hi, R4 *state,
                  std::vector<R4 *> &free_slots, R4 *scratch) {
    const int n = hi - lo;
    if (n <= 0) return MFCFD_OK;
    if (n == 1) return reverse_iteration(h, a, lo, state);
    const int s = (int)free_slots.size();
    if (s == 0) {
        for (int k = hi - 1; k >= lo; --k) {
            int st = advance(h, a, state, k - lo, scratch);
            if (st) return st;
            if ((st = reverse_iteration(h, a, k, scratch))) return st;
        }
        return MFCFD_OK;
    }
    int t = 1;
    while (binom(s, t) < n) ++t;
    const long long right = binom(s - 1, t);
    const int d = (int)std::max<long long>(1, n - std::min<long long>(right, n - 1));
    R4 *slot = free_slots.back();
    free_slots.pop_back();
    int st = advance(h, a, state, d, slot);
    if (!st) st = reverse_range(h, a, lo + d, hi, slot, free_slots, scratch);
    free_slots.push_back(slot);
    if (st) return st;
    return reverse_range(h, a, lo, lo + d, state, free_slots, scratch);
}

}  // namespace

void lskum_host::free_adjoint(mfcfd_t *h) {
    AdjointState *a = h->adj;
    if (!a) return;
    void *bufs[] = {a->d_tptr, a->d_tlist, a->d_sidx, a->d_sleft, a->d_sright, a->d_snx,
                    a->d_sny, a->d_bleft, a->d_bright, a->d_fptr, a->d_fsrc, a->d_nptr,
                    a->d_nsrc, a->tdq, a->tqm, a->tdelta, a->tspd,
                    a->pb[0], a->pb[1], a->pbA, a->qb, a->dqb[0], a->dqb[1], a->qmb,
                    a->deltab, a->frb, a->xb, a->yb, a->nxb, a->nyb, a->contrib, a->hist,
                    a->snap0, a->fin, a->tks};
    for (void *b : bufs)
        if (b) cudaFree(b);
    for (int s = 0; s < 5; ++s) {
        if (a->tprim[s]) cudaFree(a->tprim[s]);
        if (a->tq[s]) cudaFree(a->tq[s]);
    }
    for (int s = 0; s < 4; ++s)
        if (a->tfr[s]) cudaFree(a->tfr[s]);
    if (a->snap_pool) cudaFree(a->snap_pool);
    a->snaps.clear();
    delete a;
    h->adj = nullptr;
}

namespace {

bool adjoint_args_ok(const mfcfd_t *h, int objective, int n_iters) {
    return h && n_iters >= 1 && objective >= MFCFD_OBJ_CL && objective <= MFCFD_OBJ_STAGNATION;
}

// Allocation half of mfcfd_adjoint: the tape, the transposed stencil, the
// residue history and the snapshot pool (within ckpt_bytes, the initial state
// counting); returns the number of snapshot rows in *nsnap.
int adjoint_prepare(mfcfd_t *h, int objective, int n_iters, size_t ckpt_bytes, int *nsnap) {
    if (h->fp32) return fail(h, MFCFD_ERR_ARG, "mfcfd_adjoint: FP64 handles only");
    if (h->p.power != 0.0)
        return fail(h, MFCFD_ERR_ARG,
                    "mfcfd_adjoint: LSQ weights with power != 0 are not differentiated");
    int st = adj_setup(h);
    if (st) return st;
    AdjointState *a = h->adj;
    const size_t row = sizeof(R4) * (size_t)h->n;
    a->n_iters = n_iters;
    a->objective = objective;
    a->forward_iters = 0;
    if (a->hist_cap < n_iters) {
        if (a->hist) cudaFree(a->hist);
        a->hist = nullptr;
        CK(dmalloc(&a->hist, (size_t)n_iters));
        a->hist_cap = n_iters;
    }
    const long long want = ckpt_bytes > row ? (long long)(ckpt_bytes / row) - 1 : 0;
    *nsnap = (int)std::min<long long>(want, n_iters - 1);
    if ((int)a->snaps.size() < *nsnap + 1) {  // + one scratch row; one allocation
        if (a->snap_pool) cudaFree(a->snap_pool);
        a->snap_pool = nullptr;
        a->snaps.clear();
        CK(dmalloc(&a->snap_pool, (size_t)h->n * (*nsnap + 1)));
        for (int j = 0; j <= *nsnap; ++j) a->snaps.push_back(a->snap_pool + (size_t)j * h->n);
    }
    return MFCFD_OK;
}

// Run half: allocates no device memory (the objective values 2-4 excepted);
// everything is ordered on the handle's stream.
int adjoint_execute(mfcfd_t *h, int nsnap, double *J, double *dJdx, double *dJdy,
                    int *n_forward) {
    AdjointState *a = h->adj;
    const int n = h->n;
    const size_t row = sizeof(R4) * (size_t)n;
    std::vector<R4 *> free_slots(a->snaps.begin(), a->snaps.begin() + nsnap);
    R4 *scratch = a->snaps[nsnap];
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpyAsync(a->snap0, h->d_prim[h->cur], row, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemsetAsync(a->xb, 0, sizeof(double) * n, h->stream));
    CK(cudaMemsetAsync(a->yb, 0, sizeof(double) * n, h->stream));
    CK(cudaMemsetAsync(a->nxb, 0, sizeof(double) * n, h->stream));
    CK(cudaMemsetAsync(a->nyb, 0, sizeof(double) * n, h->stream));
    int st = reverse_range(h, a, 0, a->n_iters, a->snap0, free_slots, scratch);
    if (st) return st;
    const AdjGather gth{a->nbnd, a->d_fptr, a->d_fsrc, a->d_nptr, a->d_nsrc};
    launch_normals_b(a->nbnd, gth, a->d_bleft, a->d_bright, h->d_xy, a->nxb, a->nyb, a->xb,
                     a->yb, h->stream);
    h->launches += 1;
    CK(cudaGetLastError());
    // leave the final state current, as mfcfd_run would
    CK(cudaMemcpyAsync(h->d_prim[h->cur], a->fin, row, cudaMemcpyDeviceToDevice, h->stream));
    if ((st = lskum_host::upload_state_aux(h))) return st;
    std::vector<double> xb(n), yb(n);
    CK(cudaMemcpyAsync(xb.data(), a->xb, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(yb.data(), a->yb, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (int p = 0; p < n; ++p) {
        dJdx[h->perm[p]] = xb[p];
        dJdy[h->perm[p]] = yb[p];
    }
    if (J && (st = lskum_host::objective_value(h, a->objective, h->d_prim[h->cur], J)))
        return st;
    if (n_forward) *n_forward = (int)a->forward_iters;
    return MFCFD_OK;
}

}  // namespace

extern "C" int mfcfd_adjoint(mfcfd_t *h, int objective, int n_iters, size_t ckpt_bytes,
                             double *J, double *dJdx, double *dJdy, int *n_forward) {
    if (!adjoint_args_ok(h, objective, n_iters) || !dJdx || !dJdy) return MFCFD_ERR_ARG;
    int nsnap = 0;
    int st = adjoint_prepare(h, objective, n_iters, ckpt_bytes, &nsnap);
    if (st) return st;
    return adjoint_execute(h, nsnap, J, dJdx, dJdy, n_forward);
}

// Handles at least this large run their sweeps in sequence (see below).
constexpr int ADJ_OVERLAP_POINTS = 65536;

extern "C" int mfcfd_adjoint_many(int n_handles, mfcfd_t *const *handles, int objective,
                                  int n_iters, size_t ckpt_bytes, double *J,
                                  double *const *dJdx, double *const *dJdy, int *n_forward,
                                  int *status) {
    if (n_handles < 1 || n_handles > MFCFD_ADJOINT_MANY_MAX || !handles || !dJdx || !dJdy)
        return MFCFD_ERR_ARG;
    for (int i = 0; i < n_handles; ++i) {
        if (!adjoint_args_ok(handles[i], objective, n_iters) || !dJdx[i] || !dJdy[i])
            return MFCFD_ERR_ARG;
        for (int j = 0; j < i; ++j)
            if (handles[j] == handles[i] || handles[j]->stream == handles[i]->stream)
                return fail(handles[i], MFCFD_ERR_ARG,
                            "mfcfd_adjoint_many: handles must be distinct, on distinct streams");
    }
    std::vector<int> st(n_handles, MFCFD_OK), nsnap(n_handles, 0);
    // the CUDA device is per host thread: each handle's work runs with the
    // handle's device current, and the caller's device is restored at the end
    int caller_dev = 0;
    if (cudaGetDevice(&caller_dev) != cudaSuccess) caller_dev = handles[0]->dev;
    auto use_dev = [&](int i) -> int {
        const cudaError_t e = cudaSetDevice(handles[i]->dev);
        return e == cudaSuccess ? MFCFD_OK : cuda_fail(handles[i], e, "cudaSetDevice");
    };
    // every allocation first, one handle after the other
    for (int i = 0; i < n_handles; ++i) {
        st[i] = use_dev(i);
        if (!st[i]) st[i] = adjoint_prepare(handles[i], objective, n_iters, ckpt_bytes, &nsnap[i]);
        if (st[i]) {
            if (status)
                for (int k = 0; k < n_handles; ++k) status[k] = k == i ? st[i] : MFCFD_OK;
            cudaSetDevice(caller_dev);
            return st[i];
        }
    }
    // then the sweeps: a handle of ADJ_OVERLAP_POINTS points or more fills the
    // GPU on its own (its flux launches are several waves deep), so those run
    // one after another on one host thread; each smaller handle gets a thread
    // of its own, and its latency-bound sweep overlaps that chain on its own
    // stream.  Running all large sweeps at once only made them contend.
    auto run = [&](int i) {
        st[i] = use_dev(i);
        if (st[i]) return;
        st[i] = adjoint_execute(handles[i], nsnap[i], J ? J + i : nullptr, dJdx[i], dJdy[i],
                                n_forward ? n_forward + i : nullptr);
    };
    std::vector<int> large, small;
    for (int i = 0; i < n_handles; ++i)
        (handles[i]->n >= ADJ_OVERLAP_POINTS ? large : small).push_back(i);
    auto run_large = [&] {
        for (int i : large) run(i);
    };
    // a thread that cannot be created runs its work on the calling thread
    std::vector<std::thread> pool;
    std::vector<int> inline_small;
    bool large_inline = false;
    try {
        pool.reserve(n_handles + 1);
    } catch (...) {
    }
    for (int i : small) {
        try {
            pool.emplace_back(run, i);
        } catch (...) {
            inline_small.push_back(i);
        }
    }
    if (!large.empty()) {
        try {
            pool.emplace_back(run_large);
        } catch (...) {
            large_inline = true;
        }
    }
    for (int i : inline_small) run(i);
    if (large_inline) run_large();
    for (auto &t : pool) t.join();
    cudaSetDevice(caller_dev);
    int first = MFCFD_OK;
    for (int i = 0; i < n_handles; ++i) {
        if (status) status[i] = st[i];
        if (!first && st[i]) first = st[i];
    }
    return first;
}
