// Device side of the schedule: which tiles of which instances the
// grid-stride kernels of a pass visit.
//
// Instances are concatenated in device memory, each starting on a TILE
// boundary (padding points are never computed); a single grid is one
// instance.  The schedule lists the instances still running (in instance
// order) and the prefix sums of their tile counts; a kernel maps its virtual
// tile v to (instance, tile) by binary search over those prefix sums, held
// in shared memory.
#pragma once

#include "primal.h"

namespace lskum {

struct SchedSmem {
    int nact;
    int pre[MAX_BATCH + 1];
    int act[MAX_BATCH];
};

// Whole block: copies the current schedule into shared memory.
__device__ __forceinline__ void load_sched(const Sched &s, SchedSmem &ss) {
    const int na = *s.nact;
    for (int t = threadIdx.x; t <= na; t += blockDim.x) ss.pre[t] = s.pre[t];
    for (int t = threadIdx.x; t < na; t += blockDim.x) ss.act[t] = s.act[t];
    if (threadIdx.x == 0) ss.nact = na;
    __syncthreads();
}

// Active slot holding virtual tile v: the largest a with pre[a] <= v.
__device__ __forceinline__ int find_slot(const SchedSmem &ss, int v) {
    int lo = 0, hi = ss.nact - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (ss.pre[mid] <= v) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

struct TileRef {
    int base, n, nw, no, obc_off;  // the instance (InstInfo)
    int tile;                      // global tile index
    int j0;                        // instance-local index of the tile's first point
};

__device__ __forceinline__ TileRef sched_tile(const Sched &s, const SchedSmem &ss, int v) {
    const int a = find_slot(ss, v);
    const InstInfo &in = s.inst[ss.act[a]];
    const int k = v - ss.pre[a];
    return TileRef{in.base, in.n, in.nw, in.no, in.obc_off, in.tile0 + k, k * TILE};
}

// sched_tile with the schedule read from global memory (through L1) instead
// of a shared-memory copy: for kernels whose shared memory bounds residency.
__device__ __forceinline__ TileRef sched_tile_global(const Sched &s, int v) {
    int lo = 0, hi = __ldg(s.nact) - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(s.pre + mid) <= v) lo = mid;
        else hi = mid - 1;
    }
    const InstInfo &in = s.inst[__ldg(s.act + lo)];
    const int k = v - __ldg(s.pre + lo);
    return TileRef{in.base, in.n, in.nw, in.no, in.obc_off, in.tile0 + k, k * TILE};
}

// Global point of virtual point vp, or -1 for a padding point.
__device__ __forceinline__ int sched_point(const Sched &s, const SchedSmem &ss, int vp) {
    const int v = vp / TILE;
    const int a = find_slot(ss, v);
    const InstInfo &in = s.inst[ss.act[a]];
    const int j = (v - ss.pre[a]) * TILE + vp % TILE;
    return j < in.n ? in.base + j : -1;
}

}  // namespace lskum
