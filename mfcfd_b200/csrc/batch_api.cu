// C ABI of batched runs: many independent grids advanced together on one GPU.
//
// Each instance is set up exactly as mfcfd_create sets up a single grid
// (lskum_host::prepare_grid) and its renumbered arrays are placed one after
// the other in shared device arrays, every instance starting on a TILE (16
// point) boundary.  A pass of the pseudo-time loop is one grid-stride launch
// over the tiles of the instances still running (batch.cuh); the per-instance
// residual kernel retires an instance on the device (NaN residue, residue <=
// tol, or max_iters iterations) and rebuilds the schedule without it for the
// next iteration's passes.  Two iterations are captured per CUDA graph; the
// host only polls the active-instance count every 16 iterations.
//
// A single-instance handle runs the same kernels on a schedule of one
// instance, and nothing an instance computes depends on the other instances
// or on the launch shape, so its states and residues are bit-identical to
// those of a handle created from its grid alone.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <string>
#include <vector>

#include "handle.h"
#include "mfcfd_b200.h"
#include "primal.h"

using namespace lskum;

static_assert(MFCFD_BATCH_MAX == MAX_BATCH, "batch size limits differ");
static_assert(MFCFD_BATCH_CONVERGED == BATCH_CONVERGED && MFCFD_BATCH_MAX_ITERS == BATCH_MAX_ITERS &&
                  MFCFD_BATCH_NONFINITE == BATCH_NONFINITE,
              "batch states differ");

namespace {

struct BatchInst {
    int n = 0, nw = 0, no = 0, base = 0;
    int shapes = 1, nshape = 0, sh_off = 0;  // rows of the shape tables
    double mach = 0, cos_t = 1, sin_t = 0, q_inf[4] = {0, 0, 0, 0};
    std::vector<int> perm;  // instance-local new index -> caller index
};

constexpr int POLL_PAIRS = 8;  // graph launches (2 iterations each) between polls

}  // namespace

struct mfcfd_batch {
    int dev = 0, n_inst = 0, ntot = 0, kp = 1, ntiles = 0, max_n = 0, max_forces = 1;
    long long npoints = 0;
    mfcfd_params p{};
    bool fp32 = false;
    std::vector<BatchInst> inst;
    Geom geom{};
    Consts consts{};
    Sched sched{};

    double2 *d_xy = nullptr, *d_nrm = nullptr;
    double *d_eps2 = nullptr, *d_obc = nullptr;
    int *d_conn = nullptr, *d_nbhs = nullptr;
    unsigned long long *d_mx = nullptr, *d_my = nullptr;
    int *d_hoff = nullptr, *d_hrow = nullptr;  // tile halos of the D and I passes
    unsigned char *d_hloc = nullptr;
    R4 *d_prim[2] = {nullptr, nullptr}, *d_q[2] = {nullptr, nullptr};
    double *d_dq[3] = {nullptr, nullptr, nullptr};
    double *d_qm = nullptr;
    float4 *f_prim[2] = {nullptr, nullptr}, *f_q[2] = {nullptr, nullptr};
    float *f_dq[3] = {nullptr, nullptr, nullptr};
    float *f_qm = nullptr, *f_eps2 = nullptr;
    float2 *f_dxy = nullptr;
    float *f_w = nullptr;
    float4 *f_lsq = nullptr, *f_flsq = nullptr;
    Geom32 geom32{};
    double *d_delta = nullptr, *d_spd = nullptr, *d_res_part = nullptr, *d_hist = nullptr;
    double *d_forces = nullptr;
    int hist_cap = 0;
    std::vector<InstInfo> info;  // host copy of d_inst
    InstInfo *d_inst = nullptr;
    int *d_sched = nullptr;      // SCHED_INTS
    BatchRun *d_run = nullptr;
    Ctl *d_ctl = nullptr;
    int *d_sh_idx = nullptr, *d_sh_shape = nullptr;
    double *d_sh_geo = nullptr, *d_sh_my = nullptr;

    Ctl *h_ctl = nullptr;      // pinned [n_inst]
    int *h_nact = nullptr;     // pinned [2]
    int *h_sched = nullptr;    // pinned SCHED_INTS
    BatchRun *h_run = nullptr; // pinned
    double *h_stage = nullptr; // pinned [max_n][4]
    cudaEvent_t ev[2] = {nullptr, nullptr};

    int cur = 0, qcur = 0;
    cudaStream_t own = nullptr, stream = nullptr;
    cudaGraphExec_t pair_exec[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    int point_block = 256, point_grid = 0, flux_grid = 0;  // effective launch shape
    int inner_grid = 0;
    long long launches = 0;
    std::string err;
};

namespace {

int bfail(mfcfd_batch_t *b, int code, const std::string &m) {
    if (b) b->err = m;
    else lskum_host::fail(nullptr, code, m);
    return code;
}

int bcuda(mfcfd_batch_t *b, cudaError_t e, const char *where) {
    return bfail(b, e == cudaErrorMemoryAllocation ? MFCFD_ERR_OOM : MFCFD_ERR_CUDA,
                 std::string(where) + ": " + cudaGetErrorString(e));
}

#define BK(call)                                                 \
    do {                                                         \
        cudaError_t e_ = (call);                                 \
        if (e_ != cudaSuccess) return bcuda(b, e_, #call);       \
    } while (0)

template <class T>
cudaError_t dalloc(T **p, size_t count) {
    return cudaMalloc(reinterpret_cast<void **>(p), count * sizeof(T) + (count == 0 ? 16 : 0));
}

void drop_graphs(mfcfd_batch_t *b) {
    for (auto &row : b->pair_exec)
        for (auto &g : row)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
}

void free_batch(mfcfd_batch_t *b) {
    drop_graphs(b);
    void *bufs[] = {b->d_xy, b->d_nrm, b->d_eps2, b->d_obc, b->d_conn, b->d_nbhs, b->d_mx,
                    b->d_my, b->d_hoff, b->d_hrow, b->d_hloc, b->d_prim[0], b->d_prim[1], b->d_q[0], b->d_q[1], b->d_dq[0],
                    b->d_dq[1], b->d_dq[2], b->d_qm, b->f_prim[0], b->f_prim[1], b->f_q[0], b->f_q[1],
                    b->f_dq[0], b->f_dq[1], b->f_dq[2], b->f_qm, b->f_eps2, b->f_dxy, b->f_w, b->f_lsq,
                    b->f_flsq, b->d_delta, b->d_spd,
                    b->d_res_part, b->d_hist, b->d_forces, b->d_inst, b->d_sched, b->d_run,
                    b->d_ctl, b->d_sh_idx, b->d_sh_shape, b->d_sh_geo, b->d_sh_my};
    for (void *p : bufs)
        if (p) cudaFree(p);
    void *pinned[] = {b->h_ctl, b->h_nact, b->h_sched, b->h_run, b->h_stage};
    for (void *p : pinned)
        if (p) cudaFreeHost(p);
    for (auto &e : b->ev)
        if (e) cudaEventDestroy(e);
    if (b->own) cudaStreamDestroy(b->own);
}

// blocks in one wave of resident blocks of a batched pass
int batch_wave(const mfcfd_batch_t *b, int kind, int block) {
    if (kind < 2) return wave_blocks(b->dev, kind, block, 0, b->fp32);
    size_t smem = 0;
    if (kind == 2) smem = b->fp32 ? flux32_smem_bytes(b->kp) : flux_smem_bytes(b->kp);
    return wave_blocks(b->dev, kind, block, smem, b->fp32);
}

// Launch shape from (block, waves) or (block, points per thread): waves > 0
// sizes every pass to that many waves of resident blocks; otherwise ppt
// (1, 2, 4) gives each thread of the point passes ppt points and each warp
// of the flux pass ppt chunks of two tiles (ppt 1: every point its thread).
void set_shape(mfcfd_batch_t *b, int block, int waves, int ppt = 1) {
    b->point_block = block;
    const int fmax = flux_grid_blocks(b->ntiles * TILE);
    if (waves > 0) {
        b->point_grid = waves * batch_wave(b, 0, block);
        b->inner_grid = waves * batch_wave(b, 1, block);
        b->flux_grid = waves * batch_wave(b, 2, 128);
    } else {
        ppt = std::max(1, ppt);
        b->point_grid = (b->ntot + block * ppt - 1) / (block * ppt);
        b->inner_grid = b->point_grid;
        b->flux_grid = (fmax + ppt - 1) / ppt;
    }
    b->point_grid = std::max(1, std::min(b->point_grid, (b->ntot + block - 1) / block));
    b->inner_grid = std::max(1, std::min(b->inner_grid, (b->ntot + block - 1) / block));
    b->flux_grid = std::max(1, std::min(b->flux_grid, fmax));
}

// One pseudo-time stage over all active instances (launch_stage of the
// single-instance driver, with the batched kernels).
void batch_stage(mfcfd_batch_t *b, cudaStream_t s, int rk, int A, int B) {
    const int m = b->p.inner_iterations;
    const bool last = rk == b->p.rks;
    const int pb = b->point_block, pg = b->point_grid, ig = b->inner_grid, fg = b->flux_grid;
    if (!b->fp32) {
        const R4 *q_in = b->d_q[b->qcur];
        launch_grad(b->geom, b->consts, b->sched, q_in, b->d_spd, b->d_dq[0], b->d_qm,
                    b->d_delta, rk == 1, pb, pg, s);
        for (int t = 1; t <= m; ++t)
            launch_inner(b->geom, b->consts, b->sched, b->d_dq[0], b->d_dq[dq_src(t)],
                         b->d_dq[dq_dst(t)], pb, ig, s);
        StageBufs sb;
        sb.prim_in = rk == 1 ? b->d_prim[A] : b->d_prim[B];
        sb.prim_out = b->d_prim[B];
        sb.prim_old = b->d_prim[A];
        sb.q_in = q_in;
        sb.q_out = b->d_q[b->qcur ^ 1];
        sb.dq = b->d_dq[dq_final(m)];
        sb.qm = b->d_qm;
        sb.delta = b->d_delta;
        sb.spd = b->d_spd;
        sb.res_part = b->d_res_part;
        sb.flux_dbg = nullptr;
        launch_flux(b->geom, b->consts, b->sched, sb, rk, last, fg, s);
    } else {
        const float4 *q_in = b->f_q[b->qcur];
        launch_grad32(b->geom, b->consts, b->geom32, b->sched, q_in, b->d_spd, b->f_dq[0],
                      b->f_qm, b->d_delta, rk == 1, pb, pg, s);
        for (int t = 1; t <= m; ++t)
            launch_inner32(b->geom, b->consts, b->geom32, b->sched, b->f_dq[0],
                           b->f_dq[dq32_src(t)], b->f_dq[dq32_dst(t)], pb, ig, s);
        StageBufs32 sb;
        sb.prim_in = rk == 1 ? b->f_prim[A] : b->f_prim[B];
        sb.prim_out = b->f_prim[B];
        sb.prim_old = b->f_prim[A];
        sb.q_in = q_in;
        sb.q_out = b->f_q[b->qcur ^ 1];
        sb.dq = b->f_dq[dq32_final(m)];
        sb.qm = b->f_qm;
        sb.eps2f = b->f_eps2;
        sb.delta = b->d_delta;
        sb.spd = b->d_spd;
        sb.res_part = b->d_res_part;
        sb.flux_dbg = nullptr;
        sb.f = b->geom32;
        launch_flux32(b->geom, b->consts, b->sched, sb, rk, last, fg, s);
    }
    b->qcur ^= 1;
    b->launches += 2 + m;
}

int batch_iteration(mfcfd_batch_t *b, cudaStream_t s) {
    const int A = b->cur, B = b->cur ^ 1;
    for (int rk = 1; rk <= b->p.rks; ++rk) batch_stage(b, s, rk, A, B);
    launch_residual(b->d_inst, b->n_inst, b->d_res_part, b->d_ctl, b->d_hist, b->hist_cap,
                    b->d_run, b->d_sched, s);
    b->launches += 1;
    b->cur = B;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return bcuda(b, e, "kernel launch");
    return MFCFD_OK;
}

long long launches_per_iteration(const mfcfd_batch_t *b) {
    return (long long)b->p.rks * (2 + b->p.inner_iterations) + 1;
}

// Two iterations in one graph; the prim and q parities return to where they
// started (as in the single-instance driver).
int build_pair_graph(mfcfd_batch_t *b) {
    const int cur0 = b->cur, q0 = b->qcur;
    cudaGraphExec_t &slot = b->pair_exec[cur0][q0];
    if (slot) {
        cudaGraphExecDestroy(slot);
        slot = nullptr;
    }
    const long long l0 = b->launches;
    cudaGraph_t graph;
    BK(cudaStreamBeginCapture(b->own, cudaStreamCaptureModeThreadLocal));
    int st = batch_iteration(b, b->own);
    if (st == MFCFD_OK) st = batch_iteration(b, b->own);
    cudaError_t e = cudaStreamEndCapture(b->own, &graph);
    b->cur = cur0;
    b->qcur = q0;
    b->launches = l0;
    if (st != MFCFD_OK) return st;
    if (e != cudaSuccess) return bcuda(b, e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&slot, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return bcuda(b, e, "cudaGraphInstantiate");
    return MFCFD_OK;
}

int ensure_hist(mfcfd_batch_t *b, int iters) {
    if (iters <= b->hist_cap) return MFCFD_OK;
    BK(cudaStreamSynchronize(b->stream));
    if (b->d_hist) cudaFree(b->d_hist);
    b->d_hist = nullptr;
    b->hist_cap = 0;
    BK(dalloc(&b->d_hist, (size_t)b->n_inst * iters));
    b->hist_cap = iters;
    drop_graphs(b);  // the graphs hold the old history pointer and stride
    return MFCFD_OK;
}

// q and spd of instance i from its prim rows (set_state, create)
int init_instance(mfcfd_batch_t *b, int i) {
    const BatchInst &in = b->inst[i];
    Geom g = b->geom;
    g.n = in.n;
    if (b->fp32)
        launch_init_state32(g, b->f_prim[b->cur] + in.base, b->f_q[b->qcur] + in.base,
                            b->d_spd + in.base, b->stream);
    else
        launch_init_state(g, b->d_prim[b->cur] + in.base, b->d_q[b->qcur] + in.base,
                          b->d_spd + in.base, b->stream);
    b->launches += 1;
    BK(cudaGetLastError());
    return MFCFD_OK;
}

int upload_instance_state(mfcfd_batch_t *b, int i, const double *prim_caller) {
    const BatchInst &in = b->inst[i];
    BK(cudaStreamSynchronize(b->stream));
    if (b->fp32) {
        float *fs = reinterpret_cast<float *>(b->h_stage);
        for (int p = 0; p < in.n; ++p) {
            const double *src = prim_caller ? prim_caller + 4 * (size_t)in.perm[p] : in.q_inf;
            for (int c = 0; c < 4; ++c) fs[4 * (size_t)p + c] = (float)src[c];
        }
        BK(cudaMemcpyAsync(b->f_prim[b->cur] + in.base, fs, sizeof(float4) * (size_t)in.n,
                           cudaMemcpyHostToDevice, b->stream));
    } else {
        for (int p = 0; p < in.n; ++p) {
            const double *src = prim_caller ? prim_caller + 4 * (size_t)in.perm[p] : in.q_inf;
            for (int c = 0; c < 4; ++c) b->h_stage[4 * (size_t)p + c] = src[c];
        }
        BK(cudaMemcpyAsync(b->d_prim[b->cur] + in.base, b->h_stage, sizeof(R4) * (size_t)in.n,
                           cudaMemcpyHostToDevice, b->stream));
    }
    int st = init_instance(b, i);
    if (st) return st;
    BK(cudaStreamSynchronize(b->stream));
    return MFCFD_OK;
}

// Copies the state rows of instances whose last iteration left them in the
// other buffer parity back into the current buffers.
int normalise_parity(mfcfd_batch_t *b) {
    for (int i = 0; i < b->n_inst; ++i) {
        const BatchInst &in = b->inst[i];
        const int done = b->h_ctl[i].done;
        const bool prim_odd = done & 1, q_odd = ((long long)done * b->p.rks) & 1;
        if (b->fp32) {
            if (prim_odd)
                BK(cudaMemcpyAsync(b->f_prim[b->cur] + in.base, b->f_prim[b->cur ^ 1] + in.base,
                                   sizeof(float4) * in.n, cudaMemcpyDeviceToDevice, b->stream));
            if (q_odd)
                BK(cudaMemcpyAsync(b->f_q[b->qcur] + in.base, b->f_q[b->qcur ^ 1] + in.base,
                                   sizeof(float4) * in.n, cudaMemcpyDeviceToDevice, b->stream));
        } else {
            if (prim_odd)
                BK(cudaMemcpyAsync(b->d_prim[b->cur] + in.base, b->d_prim[b->cur ^ 1] + in.base,
                                   sizeof(R4) * in.n, cudaMemcpyDeviceToDevice, b->stream));
            if (q_odd)
                BK(cudaMemcpyAsync(b->d_q[b->qcur] + in.base, b->d_q[b->qcur ^ 1] + in.base,
                                   sizeof(R4) * in.n, cudaMemcpyDeviceToDevice, b->stream));
        }
    }
    return MFCFD_OK;
}

// Enqueues iterations until no instance is active or max_iters iterations
// were enqueued; h_ctl must hold the control blocks of the run (uploaded
// here with the schedule of its active instances).
int run_loop(mfcfd_batch_t *b, int max_iters) {
    std::vector<int> active(b->n_inst);
    for (int i = 0; i < b->n_inst; ++i) active[i] = b->h_ctl[i].active;
    sched_fill(b->h_sched, b->info.data(), active.data(), b->n_inst);
    BK(cudaMemcpyAsync(b->d_ctl, b->h_ctl, sizeof(Ctl) * b->n_inst, cudaMemcpyHostToDevice,
                       b->stream));
    BK(cudaMemcpyAsync(b->d_sched, b->h_sched, sizeof(int) * SCHED_INTS, cudaMemcpyHostToDevice,
                       b->stream));
    if (!b->pair_exec[b->cur][b->qcur]) {
        BK(cudaStreamSynchronize(b->stream));
        int st = build_pair_graph(b);
        if (st) return st;
    }
    cudaGraphExec_t g = b->pair_exec[b->cur][b->qcur];
    int enq = 0, pairs = 0, pending = -1;
    while (enq < max_iters) {
        BK(cudaGraphLaunch(g, b->stream));
        b->launches += 2 * launches_per_iteration(b);
        enq += 2;
        if (++pairs % POLL_PAIRS == 0 && enq < max_iters) {
            const int slot = (pairs / POLL_PAIRS) & 1;
            BK(cudaMemcpyAsync(b->h_nact + slot, b->d_sched + SCHED_NACT, sizeof(int),
                               cudaMemcpyDeviceToHost, b->stream));
            BK(cudaEventRecord(b->ev[slot], b->stream));
            if (pending >= 0) {
                BK(cudaEventSynchronize(b->ev[pending]));
                if (b->h_nact[pending] == 0) break;
            }
            pending = slot;
        }
    }
    return MFCFD_OK;
}

int check_inst(mfcfd_batch_t *b, int i) {
    if (i < 0 || i >= b->n_inst) return bfail(b, MFCFD_ERR_ARG, "instance index out of range");
    return MFCFD_OK;
}

}  // namespace

extern "C" {

int mfcfd_batch_create(int n_inst, const mfcfd_grid *const *grids, const mfcfd_params *params,
                       mfcfd_batch_t **out) {
    if (!out) return bfail(nullptr, MFCFD_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (n_inst < 1 || n_inst > MFCFD_BATCH_MAX)
        return bfail(nullptr, MFCFD_ERR_ARG, "n_inst must be in [1, MFCFD_BATCH_MAX]");
    if (!grids || !params) return bfail(nullptr, MFCFD_ERR_ARG, "grids or params is NULL");
    const mfcfd_params &P0 = params[0];
    for (int i = 0; i < n_inst; ++i) {
        if (!grids[i]) return bfail(nullptr, MFCFD_ERR_ARG, "grids[i] is NULL");
        const mfcfd_params &P = params[i];
        if (P.cfl != P0.cfl || P.power != P0.power || P.rks != P0.rks || P.euler != P0.euler ||
            P.inner_iterations != P0.inner_iterations || P.precision != P0.precision)
            return bfail(nullptr, MFCFD_ERR_ARG,
                         "params[" + std::to_string(i) +
                             "] differs from params[0] in cfl, power, rks, euler, "
                             "inner_iterations or precision");
    }
    // host set-up of every instance, as mfcfd_create does it
    std::vector<HostGrid> hg(n_inst);
    for (int i = 0; i < n_inst; ++i) {
        int st = lskum_host::prepare_grid(*grids[i], params[i], hg[i]);
        if (st) {
            std::string m = mfcfd_last_error(nullptr);
            return bfail(nullptr, st, "instance " + std::to_string(i) + ": " + m);
        }
    }
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0)
        return bfail(nullptr, MFCFD_ERR_NODEV, "no CUDA device");
    {
        cudaError_t e = init_kernels();
        if (e == cudaSuccess) e = init_kernels32();
        if (e != cudaSuccess) return bfail(nullptr, MFCFD_ERR_CUDA, cudaGetErrorString(e));
    }
    mfcfd_batch_t *b = new (std::nothrow) mfcfd_batch();
    if (!b) return bfail(nullptr, MFCFD_ERR_OOM, "host allocation failed");
    b->n_inst = n_inst;
    b->p = P0;
    b->fp32 = P0.precision == MFCFD_FP32_MIXED;
    cudaGetDevice(&b->dev);

    // placement
    b->inst.resize(n_inst);
    std::vector<InstInfo> info(n_inst);
    long long pos = 0, obc_rows = 0, sh_rows = 0;
    for (int i = 0; i < n_inst; ++i) {
        BatchInst &in = b->inst[i];
        const HostGrid &h = hg[i];
        in.n = h.n;
        in.nw = h.nw;
        in.no = h.no;
        in.base = (int)pos;
        in.shapes = h.shapes;
        in.nshape = h.nshape;
        in.sh_off = (int)sh_rows;
        in.mach = params[i].mach;
        in.cos_t = h.cos_t;
        in.sin_t = h.sin_t;
        for (int c = 0; c < 4; ++c) in.q_inf[c] = h.q_inf[c];
        info[i] = InstInfo{in.base, h.n, h.nw, h.no, (int)obc_rows, in.base / TILE,
                           (h.n + TILE - 1) / TILE, 0};
        pos += (long long)info[i].ntiles * TILE;
        obc_rows += h.no;
        sh_rows += h.nshape;
        b->kp = std::max(b->kp, h.kp);
        b->max_n = std::max(b->max_n, h.n);
        b->max_forces = std::max(b->max_forces, 3 * h.shapes + std::max(h.nshape, 1));
        b->npoints += h.n;
    }
    if (pos > (1LL << 30)) {
        free_batch(b);
        delete b;
        return bfail(nullptr, MFCFD_ERR_ARG, "batch too large (more than 2^30 points)");
    }
    const int N = (int)pos, kp = b->kp;
    b->ntot = N;
    b->ntiles = N / TILE;

    // concatenated host arrays
    std::vector<double2> xy(N, make_double2(0.0, 0.0)), nrm(N, make_double2(0.0, 1.0));
    std::vector<double> eps2(N, 0.0), obc((size_t)8 * std::max<long long>(obc_rows, 1), 0.0);
    std::vector<int> conn((size_t)kp * N), nbhs(N, 0);
    std::vector<unsigned long long> mx(N, 0), my(N, 0);
    std::vector<int> sidx, sshape;
    std::vector<double> sgeo, smy;
    // FP32-mixed geometry (per slot [kp][N], per point, per point and list)
    const bool weighted = b->fp32 && P0.power != 0.0;
    std::vector<float2> dxy(b->fp32 ? (size_t)kp * N : 0, make_float2(0.f, 0.f));
    std::vector<float> wslot(weighted ? (size_t)kp * N : 0, 0.f);
    std::vector<float4> lsq(b->fp32 ? N : 0, make_float4(0.f, 0.f, 0.f, 0.f));
    std::vector<float4> flsq(b->fp32 ? 2 * (size_t)N : 0, make_float4(0.f, 0.f, 0.f, 0.f));
    for (int p = 0; p < N; ++p)
        for (int r = 0; r < kp; ++r) conn[(size_t)r * N + p] = p;
    for (int i = 0; i < n_inst; ++i) {
        HostGrid &h = hg[i];
        const int base = b->inst[i].base;
        for (int p = 0; p < h.n; ++p) {
            xy[base + p] = h.xy[p];
            nrm[base + p] = h.nrm[p];
            eps2[base + p] = h.eps2[p];
            nbhs[base + p] = h.nbhs[p];
            mx[base + p] = h.mx[p];
            my[base + p] = h.my[p];
            for (int r = 0; r < h.kp; ++r)
                conn[(size_t)r * N + base + p] = base + h.conn[(size_t)r * h.n + p];
            if (b->fp32) {
                for (int r = 0; r < h.kp; ++r) {
                    dxy[(size_t)r * N + base + p] = h.dxy[(size_t)r * h.n + p];
                    if (weighted) wslot[(size_t)r * N + base + p] = h.wslot[(size_t)r * h.n + p];
                }
                lsq[base + p] = h.lsq[p];
                flsq[2 * (size_t)(base + p)] = h.flsq[2 * (size_t)p];
                flsq[2 * (size_t)(base + p) + 1] = h.flsq[2 * (size_t)p + 1];
            }
        }
        std::copy(h.obc.begin(), h.obc.begin() + (size_t)8 * h.no,
                  obc.begin() + (size_t)8 * info[i].obc_off);
        for (int s : h.sidx) sidx.push_back(base + s);
        sshape.insert(sshape.end(), h.sshape.begin(), h.sshape.end());
        sgeo.insert(sgeo.end(), h.sgeo.begin(), h.sgeo.end());
        smy.insert(smy.end(), h.smy.begin(), h.smy.end());
        b->inst[i].perm = std::move(h.perm);
        h = HostGrid();
    }

    HostHalo halo;  // tile halos of the D and I passes
    int st = MFCFD_OK;
    auto up = [&](auto *d, const auto &v) -> int {
        if (v.empty()) return MFCFD_OK;
        cudaError_t e = cudaMemcpy(d, v.data(), v.size() * sizeof(v[0]), cudaMemcpyHostToDevice);
        return e == cudaSuccess ? MFCFD_OK : bcuda(b, e, "cudaMemcpy");
    };
#define BALLOC(ptr, cnt)                                          \
    do {                                                          \
        cudaError_t e_ = dalloc(&(ptr), (size_t)(cnt));           \
        if (e_ != cudaSuccess) {                                  \
            st = bcuda(b, e_, "cudaMalloc " #ptr);                \
            goto fail_create;                                     \
        }                                                         \
    } while (0)
    {
        cudaError_t e = cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev[0], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev[1], cudaEventDisableTiming);
        if (e != cudaSuccess) {
            st = bcuda(b, e, "stream/event create");
            goto fail_create;
        }
        b->stream = b->own;
    }
    BALLOC(b->d_xy, N);
    BALLOC(b->d_nrm, N);
    BALLOC(b->d_eps2, N);
    BALLOC(b->d_obc, obc.size());
    BALLOC(b->d_conn, (size_t)kp * N);
    BALLOC(b->d_nbhs, N);
    BALLOC(b->d_mx, N);
    BALLOC(b->d_my, N);
    {
        std::vector<std::pair<int, int>> ranges;
        for (int i = 0; i < n_inst; ++i) ranges.emplace_back(b->inst[i].base, info[i].n);
        lskum_host::build_halo(N, kp, conn.data(), nbhs.data(), ranges, halo);
        BALLOC(b->d_hoff, halo.off.size());
        BALLOC(b->d_hrow, halo.rows.size());
        BALLOC(b->d_hloc, halo.loc.size());
    }
    if (!b->fp32) {
        for (int k = 0; k < 2; ++k) {
            BALLOC(b->d_prim[k], N);
            BALLOC(b->d_q[k], N);
        }
        for (int k = 0; k < 3; ++k) BALLOC(b->d_dq[k], (size_t)8 * N);
        BALLOC(b->d_qm, (size_t)8 * N);
    } else {
        BALLOC(b->d_prim[0], N);  // FP64 copy of the state for the force sums
        for (int k = 0; k < 2; ++k) {
            BALLOC(b->f_prim[k], N);
            BALLOC(b->f_q[k], N);
        }
        for (int k = 0; k < 3; ++k) BALLOC(b->f_dq[k], (size_t)8 * N);
        BALLOC(b->f_qm, (size_t)8 * N);
        BALLOC(b->f_eps2, N);
        BALLOC(b->f_dxy, (size_t)kp * N);
        if (weighted) BALLOC(b->f_w, (size_t)kp * N);
        BALLOC(b->f_lsq, N);
        BALLOC(b->f_flsq, 2 * (size_t)N);
    }
    BALLOC(b->d_delta, N);
    BALLOC(b->d_spd, N);
    BALLOC(b->d_res_part, b->ntiles);
    BALLOC(b->d_forces, b->max_forces);
    BALLOC(b->d_inst, n_inst);
    BALLOC(b->d_sched, SCHED_INTS);
    BALLOC(b->d_run, 1);
    BALLOC(b->d_ctl, n_inst);
    BALLOC(b->d_sh_idx, std::max<size_t>(sidx.size(), 1));
    BALLOC(b->d_sh_shape, std::max<size_t>(sshape.size(), 1));
    BALLOC(b->d_sh_geo, std::max<size_t>(sgeo.size(), 1));
    BALLOC(b->d_sh_my, std::max<size_t>(smy.size(), 1));
    {
        cudaError_t e = cudaMallocHost(reinterpret_cast<void **>(&b->h_ctl), sizeof(Ctl) * n_inst);
        if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void **>(&b->h_nact), 2 * sizeof(int));
        if (e == cudaSuccess)
            e = cudaMallocHost(reinterpret_cast<void **>(&b->h_sched), sizeof(int) * SCHED_INTS);
        if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void **>(&b->h_run), sizeof(BatchRun));
        if (e == cudaSuccess)
            e = cudaMallocHost(reinterpret_cast<void **>(&b->h_stage),
                               sizeof(double) * 4 * (size_t)b->max_n);
        if (e != cudaSuccess) {
            st = bcuda(b, e, "cudaMallocHost");
            goto fail_create;
        }
    }
    if ((st = up(b->d_xy, xy)) || (st = up(b->d_nrm, nrm)) || (st = up(b->d_eps2, eps2)) ||
        (st = up(b->d_obc, obc)) || (st = up(b->d_conn, conn)) || (st = up(b->d_nbhs, nbhs)) ||
        (st = up(b->d_mx, mx)) || (st = up(b->d_my, my)) || (st = up(b->d_inst, info)) ||
        (st = up(b->d_sh_idx, sidx)) || (st = up(b->d_sh_shape, sshape)) ||
        (st = up(b->d_sh_geo, sgeo)) || (st = up(b->d_sh_my, smy)))
        goto fail_create;
    if (b->d_hoff && ((st = up(b->d_hoff, halo.off)) || (st = up(b->d_hrow, halo.rows)) ||
                      (st = up(b->d_hloc, halo.loc))))
        goto fail_create;
    if (b->fp32) {
        std::vector<float> feps(eps2.begin(), eps2.end());
        if ((st = up(b->f_eps2, feps)) || (st = up(b->f_dxy, dxy)) || (st = up(b->f_lsq, lsq)) ||
            (st = up(b->f_flsq, flsq)))
            goto fail_create;
        if (weighted && (st = up(b->f_w, wslot))) goto fail_create;
        b->geom32 = Geom32{b->f_dxy, b->f_w, b->f_lsq, b->f_flsq};
    }
    b->geom = Geom{N, kp, 0, 0, b->d_xy, b->d_nrm, b->d_eps2, b->d_conn, b->d_nbhs,
                   b->d_mx, b->d_my, b->d_obc};
    if (b->d_hoff) {
        b->geom.hoff = b->d_hoff;
        b->geom.hrow = b->d_hrow;
        b->geom.hloc = b->d_hloc;
        b->geom.hkp = halo.hkp;
        b->geom.hc = halo.hc;
    }
    b->consts.cfl = P0.cfl;
    b->consts.power = P0.power;
    b->consts.euler = P0.euler;
    b->consts.pi = 4.0 * atan(1.0);
    b->consts.gm1 = 1.4 - 1;
    b->consts.power_zero = P0.power == 0.0 ? 1 : 0;
    b->consts.rks = P0.rks;
    b->sched = sched_view(b->d_inst, b->d_sched);
    b->info = info;
    for (int i = 0; i < n_inst; ++i) {
        Ctl c{};
        c.it = 1;
        c.it_first = 1;
        c.restart = params[i].restart;
        c.plen = b->inst[i].n;
        c.res_old = params[i].res_old;
        b->h_ctl[i] = c;
    }
    {
        cudaError_t e = cudaMemcpy(b->d_ctl, b->h_ctl, sizeof(Ctl) * n_inst, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            st = bcuda(b, e, "cudaMemcpy ctl");
            goto fail_create;
        }
    }
    // initial_conditions.F90:9-20: freestream everywhere
    for (int i = 0; i < n_inst; ++i)
        if ((st = upload_instance_state(b, i, nullptr))) goto fail_create;
    set_shape(b, default_point_block(b->fp32), 1);
    *out = b;
    return MFCFD_OK;
fail_create:
    {
        std::string m = b->err;
        free_batch(b);
        delete b;
        return bfail(nullptr, st, m);
    }
#undef BALLOC
}

int mfcfd_batch_destroy(mfcfd_batch_t *b) {
    if (!b) return MFCFD_OK;
    cudaStreamSynchronize(b->stream);
    free_batch(b);
    delete b;
    return MFCFD_OK;
}

int mfcfd_batch_set_stream(mfcfd_batch_t *b, void *stream) {
    if (!b) return MFCFD_ERR_ARG;
    b->stream = stream ? static_cast<cudaStream_t>(stream) : b->own;
    return MFCFD_OK;
}

int mfcfd_batch_set_state(mfcfd_batch_t *b, int i, const double *prim) {
    if (!b || !prim) return MFCFD_ERR_ARG;
    if (int st = check_inst(b, i)) return st;
    return upload_instance_state(b, i, prim);
}

int mfcfd_batch_get_state(mfcfd_batch_t *b, int i, double *prim) {
    if (!b || !prim) return MFCFD_ERR_ARG;
    if (int st = check_inst(b, i)) return st;
    const BatchInst &in = b->inst[i];
    BK(cudaStreamSynchronize(b->stream));
    if (b->fp32) {
        float *fs = reinterpret_cast<float *>(b->h_stage);
        BK(cudaMemcpyAsync(fs, b->f_prim[b->cur] + in.base, sizeof(float4) * (size_t)in.n,
                           cudaMemcpyDeviceToHost, b->stream));
        BK(cudaStreamSynchronize(b->stream));
        for (int p = 0; p < in.n; ++p)
            for (int c = 0; c < 4; ++c)
                prim[4 * (size_t)in.perm[p] + c] = fs[4 * (size_t)p + c];
        return MFCFD_OK;
    }
    BK(cudaMemcpyAsync(b->h_stage, b->d_prim[b->cur] + in.base, sizeof(R4) * (size_t)in.n,
                       cudaMemcpyDeviceToHost, b->stream));
    BK(cudaStreamSynchronize(b->stream));
    for (int p = 0; p < in.n; ++p)
        for (int c = 0; c < 4; ++c) prim[4 * (size_t)in.perm[p] + c] = b->h_stage[4 * (size_t)p + c];
    return MFCFD_OK;
}

int mfcfd_batch_run(mfcfd_batch_t *b, double tol, int max_iters, int *iters_done, int *state,
                    double *residue) {
    if (!b) return MFCFD_ERR_ARG;
    if (max_iters < 0 || isnan(tol)) return bfail(b, MFCFD_ERR_ARG, "max_iters < 0 or tol NaN");
    for (int i = 0; i < b->n_inst; ++i) {
        if (iters_done) iters_done[i] = 0;
        if (state) state[i] = MFCFD_BATCH_RUNNING;
    }
    if (max_iters == 0) return MFCFD_OK;
    if (int st = ensure_hist(b, max_iters)) return st;
    BK(cudaStreamSynchronize(b->stream));
    BK(cudaMemcpy(b->h_ctl, b->d_ctl, sizeof(Ctl) * b->n_inst, cudaMemcpyDeviceToHost));
    for (int i = 0; i < b->n_inst; ++i) {
        Ctl &c = b->h_ctl[i];
        c.it_first = c.it;
        c.done = 0;
        c.halted = 0;
        c.active = 1;
        c.state = BATCH_RUNNING;
    }
    b->h_run->tol = tol;
    b->h_run->max_iters = max_iters;
    BK(cudaMemcpyAsync(b->d_run, b->h_run, sizeof(BatchRun), cudaMemcpyHostToDevice, b->stream));
    if (int st = run_loop(b, max_iters)) return st;
    BK(cudaMemcpyAsync(b->h_ctl, b->d_ctl, sizeof(Ctl) * b->n_inst, cudaMemcpyDeviceToHost,
                       b->stream));
    BK(cudaStreamSynchronize(b->stream));
    if (int st = normalise_parity(b)) return st;
    bool nan = false;
    for (int i = 0; i < b->n_inst; ++i) {
        if (iters_done) iters_done[i] = b->h_ctl[i].done;
        if (state) state[i] = b->h_ctl[i].state;
        nan = nan || b->h_ctl[i].state == BATCH_NONFINITE;
    }
    if (residue) {
        std::vector<double> hist((size_t)b->n_inst * b->hist_cap);
        BK(cudaMemcpyAsync(hist.data(), b->d_hist, hist.size() * sizeof(double),
                           cudaMemcpyDeviceToHost, b->stream));
        BK(cudaStreamSynchronize(b->stream));
        for (int i = 0; i < b->n_inst; ++i)
            for (int k = 0; k < b->h_ctl[i].done; ++k)
                residue[(size_t)i * max_iters + k] = hist[(size_t)i * b->hist_cap + k];
    }
    BK(cudaStreamSynchronize(b->stream));
    if (nan) return bfail(b, MFCFD_ERR_NONFINITE, "an instance's residue is NaN");
    return MFCFD_OK;
}

int mfcfd_batch_forces(mfcfd_batch_t *b, int i, double *cl, double *cd, double *cm, double *cp) {
    if (!b) return MFCFD_ERR_ARG;
    if (int st = check_inst(b, i)) return st;
    const BatchInst &in = b->inst[i];
    const R4 *prim = b->d_prim[b->cur];
    if (b->fp32) {
        launch_widen(b->f_prim[b->cur] + in.base, b->d_prim[0] + in.base, in.n, b->stream);
        b->launches += 1;
        prim = b->d_prim[0];
    }
    ShapeTab t{in.nshape, in.shapes, b->d_sh_idx + in.sh_off, b->d_sh_shape + in.sh_off,
               b->d_sh_geo + 4 * (size_t)in.sh_off, b->d_sh_my + in.sh_off};
    launch_forces(t, prim, in.mach, in.cos_t, in.sin_t, b->d_forces, b->stream);
    b->launches += 1;
    BK(cudaGetLastError());
    std::vector<double> o(3 * in.shapes + in.nshape);
    BK(cudaMemcpyAsync(o.data(), b->d_forces, o.size() * sizeof(double), cudaMemcpyDeviceToHost,
                       b->stream));
    BK(cudaStreamSynchronize(b->stream));
    for (int s = 0; s < in.shapes; ++s) {
        if (cl) cl[s] = o[s];
        if (cd) cd[s] = o[in.shapes + s];
        if (cm) cm[s] = o[2 * in.shapes + s];
    }
    if (cp)
        for (int k = 0; k < in.nshape; ++k) cp[k] = o[3 * in.shapes + k];
    return MFCFD_OK;
}

int mfcfd_batch_set_launch(mfcfd_batch_t *b, int point_block, int point_grid, int flux_grid) {
    if (!b) return MFCFD_ERR_ARG;
    if ((point_block != 128 && point_block != 256) || point_grid < 0 || flux_grid < 0)
        return bfail(b, MFCFD_ERR_ARG, "point_block must be 128 or 256, grids >= 0");
    BK(cudaStreamSynchronize(b->stream));
    set_shape(b, point_block, 1);
    if (point_grid > 0)
        b->point_grid = b->inner_grid =
            std::min(point_grid, (b->ntot + point_block - 1) / point_block);
    if (flux_grid > 0) b->flux_grid = std::min(flux_grid, flux_grid_blocks(b->ntiles * TILE));
    drop_graphs(b);
    return MFCFD_OK;
}

int mfcfd_batch_tune(mfcfd_batch_t *b, int iters, double *ms_per_iter) {
    if (!b) return MFCFD_ERR_ARG;
    if (iters < 2) return bfail(b, MFCFD_ERR_ARG, "iters must be >= 2");
    iters += iters & 1;
    if (int st = ensure_hist(b, iters + 2)) return st;
    BK(cudaStreamSynchronize(b->stream));
    // saved state: prim, q and spd rows and the control blocks
    const size_t rows = (size_t)b->ntot;
    void *save_prim = nullptr, *save_q = nullptr, *save_spd = nullptr;
    const size_t row_bytes = b->fp32 ? sizeof(float4) : sizeof(R4);
    void *prim = b->fp32 ? (void *)b->f_prim[b->cur] : (void *)b->d_prim[b->cur];
    void *q = b->fp32 ? (void *)b->f_q[b->qcur] : (void *)b->d_q[b->qcur];
    std::vector<Ctl> ctl0(b->n_inst);
    int st = MFCFD_OK;
    double best_ms = 0.0;
    int best_block = b->point_block, best_pg = b->point_grid, best_fg = b->flux_grid;
    int best_ig = b->inner_grid;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    auto restore = [&]() -> int {
        BK(cudaMemcpyAsync(prim, save_prim, rows * row_bytes, cudaMemcpyDeviceToDevice, b->stream));
        BK(cudaMemcpyAsync(q, save_q, rows * row_bytes, cudaMemcpyDeviceToDevice, b->stream));
        BK(cudaMemcpyAsync(b->d_spd, save_spd, rows * sizeof(double), cudaMemcpyDeviceToDevice,
                           b->stream));
        for (int i = 0; i < b->n_inst; ++i) b->h_ctl[i] = ctl0[i];
        BK(cudaMemcpyAsync(b->d_ctl, b->h_ctl, sizeof(Ctl) * b->n_inst, cudaMemcpyHostToDevice,
                           b->stream));
        BK(cudaStreamSynchronize(b->stream));
        return MFCFD_OK;
    };
    {
        cudaError_t e = cudaMalloc(&save_prim, rows * row_bytes);
        if (e == cudaSuccess) e = cudaMalloc(&save_q, rows * row_bytes);
        if (e == cudaSuccess) e = cudaMalloc(&save_spd, rows * sizeof(double));
        if (e == cudaSuccess) e = cudaEventCreate(&t0);
        if (e == cudaSuccess) e = cudaEventCreate(&t1);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(save_prim, prim, rows * row_bytes, cudaMemcpyDeviceToDevice, b->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(save_q, q, rows * row_bytes, cudaMemcpyDeviceToDevice, b->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(save_spd, b->d_spd, rows * sizeof(double), cudaMemcpyDeviceToDevice,
                                b->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(ctl0.data(), b->d_ctl, sizeof(Ctl) * b->n_inst,
                                cudaMemcpyDeviceToHost, b->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
        if (e != cudaSuccess) st = bcuda(b, e, "tune set-up");
    }
    // candidates: 1, 2, 4 waves of resident blocks, and 1, 2, 4 points per
    // thread (chunks per flux warp), for blocks of 256 and 128 threads
    const int blocks[2] = {256, 128};
    const int waves[6] = {1, 2, 4, 0, 0, 0}, ppts[6] = {0, 0, 0, 1, 2, 4};
    for (int bi = 0; bi < 2 && st == MFCFD_OK; ++bi)
        for (int wi = 0; wi < 6 && st == MFCFD_OK; ++wi) {
            set_shape(b, blocks[bi], waves[wi], ppts[wi]);
            drop_graphs(b);
            if ((st = restore())) break;
            for (int i = 0; i < b->n_inst; ++i) {
                Ctl &c = b->h_ctl[i];
                c.it_first = c.it;
                c.done = 0;
                c.halted = 0;
                c.active = 1;
                c.state = BATCH_RUNNING;
            }
            b->h_run->tol = -INFINITY;
            b->h_run->max_iters = iters + 2;
            cudaError_t e = cudaMemcpyAsync(b->d_run, b->h_run, sizeof(BatchRun),
                                            cudaMemcpyHostToDevice, b->stream);
            if (e != cudaSuccess) {
                st = bcuda(b, e, "tune upload");
                break;
            }
            if ((st = run_loop(b, 2))) break;  // warm-up pair (builds the graph)
            e = cudaEventRecord(t0, b->stream);
            for (int k = 0; k < iters / 2 && e == cudaSuccess; ++k) {
                e = cudaGraphLaunch(b->pair_exec[b->cur][b->qcur], b->stream);
                b->launches += 2 * launches_per_iteration(b);
            }
            if (e == cudaSuccess) e = cudaEventRecord(t1, b->stream);
            if (e == cudaSuccess) e = cudaEventSynchronize(t1);
            float ms = 0.f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
            if (e != cudaSuccess) {
                st = bcuda(b, e, "tune timing");
                break;
            }
            const double per = ms / iters;
            if (best_ms == 0.0 || per < best_ms) {
                best_ms = per;
                best_block = b->point_block;
                best_pg = b->point_grid;
                best_ig = b->inner_grid;
                best_fg = b->flux_grid;
            }
        }
    if (save_prim && save_q && save_spd && st == MFCFD_OK) st = restore();
    b->point_block = best_block;
    b->point_grid = best_pg;
    b->inner_grid = best_ig;
    b->flux_grid = best_fg;
    drop_graphs(b);
    if (save_prim) cudaFree(save_prim);
    if (save_q) cudaFree(save_q);
    if (save_spd) cudaFree(save_spd);
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    if (st == MFCFD_OK && ms_per_iter) *ms_per_iter = best_ms;
    return st;
}

int mfcfd_batch_info(mfcfd_batch_t *b, int *n_inst, long long *n_points, int *point_block,
                     int *point_grid, int *flux_grid) {
    if (!b) return MFCFD_ERR_ARG;
    if (n_inst) *n_inst = b->n_inst;
    if (n_points) *n_points = b->npoints;
    if (point_block) *point_block = b->point_block;
    if (point_grid) *point_grid = b->point_grid;
    if (flux_grid) *flux_grid = b->flux_grid;
    return MFCFD_OK;
}

const char *mfcfd_batch_last_error(mfcfd_batch_t *b) {
    if (!b) return mfcfd_last_error(nullptr);
    return b->err.c_str();
}

long long mfcfd_batch_launch_count(mfcfd_batch_t *b) { return b ? b->launches : 0; }

}  // extern "C"
