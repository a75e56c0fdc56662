// Tile halos of the point passes (the D and I passes of both precisions).
//
// The halo of a TILE-point tile is the sorted set of rows its points read:
// the points themselves and their stencil neighbours (Geom::hoff, hrow,
// hloc, built once per grid on the host).  A warp takes chunks of two
// scheduled tiles, copies both tiles' halo rows into shared memory with
// cp.async -- every row once, consecutive lanes copying consecutive 16-byte
// pieces of a row array, so that the runs of neighbouring rows an O-grid
// ring order gives come in whole 128-byte lines -- waits, and computes one
// point per lane from shared memory.  Shared memory holds one 16-byte array
// per piece of a row (stride hc rows, one more than a multiple of eight, so
// the pieces of a row fall on different banks and a warp's reads of
// neighbouring rows on distinct banks).  A tile whose halo was too large to
// stage (an empty hrow range) reads its rows from global memory.
#pragma once

#include "batch.cuh"

namespace lskum {

__device__ __forceinline__ void halo_cp16(void *dst, const void *src) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void halo_cp8(void *dst, const void *src) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
// Waits for every cp.async this thread issued.
__device__ __forceinline__ void halo_wait() {
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// The row indices of a warp's two tiles: lane l holds those of pair rows l,
// l + 32, l + 64 and l + 96 (row u of the pair being row u of the first
// tile's halo, hrow[h0 + u], or row u - hn0 of the second's).
struct HaloIdx {
    int h0 = 0, hn0 = 0, h1 = 0, hn1 = 0;
    int kr[2 * HALO_CAP / 32] = {0, 0, 0, 0};
};

// One chunk: both tiles' halo ranges and row indices, and this lane's point
// (i < 0: none), its stencil size and the size of its tile's halo.
struct HaloChunk {
    HaloIdx x;
    int i = -1, nb = 0, hn = 0;
};

__device__ __forceinline__ void halo_chunk(const Geom &g, const Sched &s, const SchedSmem &ss,
                                           int ntiles, int ch, int lane, HaloChunk &c) {
    c = HaloChunk();
    if (2 * ch >= ntiles) return;
    const int half = lane / TILE, jl = lane % TILE;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int v = 2 * ch + h;
        if (v >= ntiles) break;
        const TileRef t = sched_tile(s, ss, v);
        const int h0 = __ldg(g.hoff + t.tile), hn = __ldg(g.hoff + t.tile + 1) - h0;
        if (h == 0) {
            c.x.h0 = h0;
            c.x.hn0 = hn;
        } else {
            c.x.h1 = h0;
            c.x.hn1 = hn;
        }
        if (h == half) {
            c.hn = hn;
            if (t.j0 + jl < t.n) {
                c.i = t.base + t.j0 + jl;
                c.nb = __ldg(g.nbhs + c.i);
            }
        }
    }
    const int hnt = c.x.hn0 + c.x.hn1;
#pragma unroll
    for (int w = 0; w < 2 * HALO_CAP / 32; ++w) {
        const int u = 32 * w + lane;
        c.x.kr[w] = u < hnt ? __ldg(g.hrow + (u < c.x.hn0 ? c.x.h0 + u : c.x.h1 + u - c.x.hn0))
                            : 0;
    }
}

// Copies NP 16-byte pieces of every halo row of an array (row k at base + k *
// row_bytes) into shared arrays a0 .. a0 + NP - 1: piece p of pair row u to
// (u < hn0 ? sm0 + u : sm1 + u - hn0) + (a0 + p) * hc.  A copy takes its row
// index from the lane holding it (a shuffle whose source register is the
// same for the whole warp).
template <int NP>
__device__ __forceinline__ void stage_array(const void *base, int row_bytes, const HaloIdx &x,
                                            int lane, double2 *sm0, double2 *sm1, int hc,
                                            int a0) {
    const int hn0 = x.hn0, hn = x.hn0 + x.hn1;
    const char *b = static_cast<const char *>(base);
#pragma unroll
    for (int t = 0; t < 2 * HALO_CAP * NP / 32; ++t) {
        if (32 * t >= NP * hn) break;
        const int pc = 32 * t + lane, u = pc / NP, part = pc % NP;
        const int k = NP == 1 ? x.kr[t] : __shfl_sync(0xffffffffu, x.kr[t / NP], u & 31);
        double2 *d = (u < hn0 ? sm0 + u : sm1 + (u - hn0)) + (a0 + part) * hc;
        if (u < hn) halo_cp16(d, b + (size_t)k * row_bytes + 16 * part);
    }
}

// An 8-byte value per halo row (row k at base + 8 k) into the first half of
// shared array a.
__device__ __forceinline__ void stage_array8(const void *base, const HaloIdx &x, int lane,
                                             double2 *sm0, double2 *sm1, int hc, int a) {
    const int hn0 = x.hn0, hn = x.hn0 + x.hn1;
    const char *b = static_cast<const char *>(base);
#pragma unroll
    for (int t = 0; t < 2 * HALO_CAP / 32; ++t) {
        if (32 * t >= hn) break;
        const int u = 32 * t + lane;
        double2 *d = (u < hn0 ? sm0 + u : sm1 + (u - hn0)) + a * hc;
        if (u < hn) halo_cp8(d, b + 8 * (size_t)x.kr[t]);
    }
}

// A point's local rows: hloc[i * hkp + r] for its slots r, hloc[i * hkp + hkp
// - 1] its own row (hkp <= 24: three 8-byte words).
struct HaloLoc {
    unsigned long long w0 = 0ull, w1 = 0ull, w2 = 0ull;
    int own = 0;
    // i < 0: no point (nothing is loaded)
    __device__ __forceinline__ HaloLoc(const Geom &g, int i) {
        if (i < 0) return;
        const unsigned long long *lw =
            reinterpret_cast<const unsigned long long *>(g.hloc + (size_t)i * g.hkp);
        w0 = __ldg(lw);
        if (g.hkp > 8) w1 = __ldg(lw + 1);
        if (g.hkp > 16) w2 = __ldg(lw + 2);
        const unsigned long long last = g.hkp > 16 ? w2 : (g.hkp > 8 ? w1 : w0);
        own = (int)(last >> 56);
    }
    __device__ __forceinline__ int slot(int r) const {
        const unsigned long long w = r < 8 ? w0 : (r < 16 ? w1 : w2);
        return (int)((w >> (8 * (r & 7))) & 0xffull);
    }
};

// dynamic shared memory of a halo kernel: nA arrays of hc 16-byte rows per
// tile, two tiles a warp
inline size_t halo_bytes(int warps, int nA, int hc) {
    return (size_t)warps * 2 * nA * hc * sizeof(double2);
}

}  // namespace lskum
