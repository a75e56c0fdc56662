// Internal: the handle behind mfcfd_t, shared by the C ABI files.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <utility>
#include <vector>

#include "mfcfd_b200.h"
#include "primal.h"

using namespace lskum;

struct AdjointState;  // adjoint buffers (adjoint_api.cu), created on first use

struct mfcfd {
    int dev = 0;
    int n = 0, kp = 1, nw = 0, no = 0, nint = 0, shapes = 1, nshape = 0;
    int n_local = 0;  // owned points; [n_local, n) are ghosts of a partitioned grid
    mfcfd_params p{};
    std::vector<int> perm;  // new index -> caller index
    double pi = 0, theta = 0, cos_t = 0, sin_t = 0, q_inf[4] = {0, 0, 0, 0};

    Geom geom{};
    Consts consts{};
    ShapeTab shape{};

    // device buffers
    double2 *d_xy = nullptr, *d_nrm = nullptr;
    double *d_eps2 = nullptr, *d_obc = nullptr;
    int *d_conn = nullptr, *d_nbhs = nullptr;
    unsigned long long *d_mx = nullptr, *d_my = nullptr;
    int *d_hoff = nullptr, *d_hrow = nullptr;  // tile halos of the D and I passes
    unsigned char *d_hloc = nullptr;
    R4 *d_prim[2] = {nullptr, nullptr}, *d_q[2] = {nullptr, nullptr};
    double *d_dq[3] = {nullptr, nullptr, nullptr};  // D-pass result, then the inner iterations'
    double *d_qm = nullptr, *d_delta = nullptr, *d_spd = nullptr, *d_res_part = nullptr;
    double *d_flux_dbg = nullptr, *d_hist = nullptr, *d_forces = nullptr;
    int hist_cap = 0;
    Ctl *d_ctl = nullptr;
    Ctl *h_ctl = nullptr;  // pinned
    int *d_sh_idx = nullptr, *d_sh_shape = nullptr;
    double *d_sh_geo = nullptr, *d_sh_my = nullptr;
    double *h_stage = nullptr;  // pinned staging [n][4]
    // FP32-mixed state (precision == MFCFD_FP32_MIXED)
    bool fp32 = false;
    float4 *f_prim[2] = {nullptr, nullptr}, *f_q[2] = {nullptr, nullptr};
    float *f_dq[3] = {nullptr, nullptr, nullptr};
    float *f_qm = nullptr, *f_eps2 = nullptr;
    float2 *f_dxy = nullptr;
    float *f_w = nullptr;
    float4 *f_lsq = nullptr, *f_flsq = nullptr;
    Geom32 geom32{};

    // the handle's grid as a schedule of one instance (kernels are shared
    // with batched runs)
    InstInfo inst_h{};
    InstInfo *d_inst = nullptr;
    int *d_sched = nullptr;    // SCHED_INTS
    int *h_sched = nullptr;    // pinned SCHED_INTS
    BatchRun *d_run = nullptr; // no retirement but on a NaN residue
    Sched sched{};
    int point_block = 256, point_grid = 1, flux_grid = 1;  // launch shape
    int inner_grid = 1;  // I pass (its residency differs from the D pass's)

    int cur = 0;   // prim buffer holding the state
    int qcur = 0;  // q buffer holding q of the state
    int iters_done_total = 0;
    cudaStream_t own = nullptr, stream = nullptr;
    cudaGraphExec_t pair_exec[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [cur][qcur]
    // one iteration as a graph (for odd iteration counts), and the (cur, qcur)
    // it leaves current
    cudaGraphExec_t one_exec[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    int one_next[2][2][2] = {};
    bool keep_diag = false;
    long long launches = 0;
    std::string err;
    std::vector<double> shape_cp;
    AdjointState *adj = nullptr;
    // device address of the fixed residue-history array of mfcfd_run_noalloc
    // on this handle's device, resolved by mfcfd_create (nullptr if that
    // lookup failed; noalloc_err then says why)
    double *noalloc_hist = nullptr;
    std::string noalloc_err;
    // phase-by-phase iteration of a partitioned grid (mfcfd_part_phase)
    bool part_in_iter = false;
    int part_A = 0;                // prim buffer the iteration started from
    int part_dq = 0;               // dq buffer the last D or I pass wrote
    double *d_part_sum = nullptr;  // the rank's sum of res_sqr
    // caller-order ring neighbours of every point (for the adjoint set-up)
    std::vector<int> left0, right0, flag2_0;
};


// Renumbered host arrays of one grid (the host half of mfcfd_create).
struct HostGrid {
    int n = 0, n_local = 0, kp = 1, nw = 0, no = 0, shapes = 1, nshape = 0;
    double pi = 0, theta = 0, cos_t = 0, sin_t = 0, q_inf[4] = {0, 0, 0, 0};
    std::vector<int> perm;  // new index -> caller index
    std::vector<double2> xy, nrm;
    std::vector<double> eps2, obc;  // obc: 8 per outer point (at least 8)
    std::vector<int> conn, nbhs;    // conn[r * n + p], renumbered, padded with p
    std::vector<unsigned long long> mx, my;
    std::vector<int> sidx, sshape;  // shape points in caller order
    std::vector<double> sgeo, smy;
    // FP32-mixed geometry (precision MFCFD_FP32_MIXED only)
    std::vector<float2> dxy;    // [kp][n] offsets to the stencil neighbours
    std::vector<float> wslot;   // [kp][n] least-squares weights (power != 0 only)
    std::vector<float4> lsq;    // [n] inverse normal matrix of the full stencil
    std::vector<float4> flsq;   // [2n] per split list, two solve coefficients
};

// Tile halos (Geom::hoff, hrow, hloc) of a renumbered point set of n points
// with ELL stencils conn[r * n + p] (nbhs[p] slots used), for the tiles of
// the point ranges [b, b + m) of `ranges` (each b a multiple of TILE); every
// other tile gets an empty halo.
struct HostHalo {
    std::vector<int> off, rows;
    std::vector<unsigned char> loc;
    int hkp = 0, hc = 0;
};

namespace lskum_host {
void build_halo(int n, int kp, const int *conn, const int *nbhs,
                const std::vector<std::pair<int, int>> &ranges, HostHalo &out);
// n_local < 0: every point is owned; else points [n_local, n) are ghosts
int prepare_grid(const mfcfd_grid &G, const mfcfd_params &P, HostGrid &hg, int n_local = -1);
int fail(mfcfd_t *h, int code, const std::string &msg);
int cuda_fail(mfcfd_t *h, cudaError_t e, const char *where);
int enqueue_iteration_to(mfcfd_t *h, cudaStream_t s, double *hist);
int upload_state_aux(mfcfd_t *h);
// Control block and schedule for a run starting at iteration it_first
// (enqueued on the handle's stream).
int reset_run(mfcfd_t *h, int it_first);
void free_adjoint(mfcfd_t *h);
template <class T>
inline cudaError_t dmalloc(T **p, size_t count) {
    return cudaMalloc(reinterpret_cast<void **>(p), count * sizeof(T) + (count == 0 ? 16 : 0));
}
}  // namespace lskum_host

// Makes `dev` the calling thread's current device for the scope of a call
// and gives the caller's device back afterwards, so that a handle's work
// (allocations, launches, symbol lookups) lands on the handle's own GPU
// whatever device the caller has current.
struct DevGuard {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit DevGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) err = cudaSetDevice(dev);
    }
    ~DevGuard() {
        int now = -1;
        if (prev >= 0 && cudaGetDevice(&now) == cudaSuccess && now != prev) cudaSetDevice(prev);
    }
    DevGuard(const DevGuard &) = delete;
    DevGuard &operator=(const DevGuard &) = delete;
};

#define CK(call)                                                                   \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) return lskum_host::cuda_fail(h, e_, #call);         \
    } while (0)
