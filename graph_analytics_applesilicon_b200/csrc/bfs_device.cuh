// bfs_device.cuh -- device helpers shared by the persistent BFS kernels.
#pragma once

#include "common.cuh"

namespace gb {

// Exclusive scan of one value per thread over a block of NT threads; *total
// gets the block sum.  All threads of the block must call it.
template <int NT>
__device__ __forceinline__ uint32_t blockScan(uint32_t v, uint32_t* total, uint32_t* sm) {
    constexpr int W = NT / 32;
    const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(kFull, x, o);
        if ((int)lane >= o) x += y;
    }
    if (lane == 31) sm[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = lane < W ? sm[lane] : 0u, incl = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(kFull, incl, o);
            if ((int)lane >= o) incl += y;
        }
        if (lane < W) sm[lane] = incl - w;
        if (lane == W - 1) sm[W] = incl;
    }
    __syncthreads();
    uint32_t r = sm[wid] + x - v;
    *total = sm[W];
    __syncthreads();
    return r;
}

// Largest i in [lo, hi] with off[i] <= e (the owner of edge e in an
// exclusive scan of degrees; zero-degree entries are skipped).
template <class T>
__device__ __forceinline__ uint32_t ownerOf(const T* off, uint32_t lo, uint32_t hi, T e) {
    while (lo < hi) {
        uint32_t mid = (lo + hi + 1) >> 1;
        if (off[mid] <= e) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// ownerOf for one warp: all 32 lanes call it with the same arguments and all
// get the result.  Each round probes 32 evenly spaced entries at once, so a
// search over R entries costs ceil(log32 R) + 1 dependent loads instead of
// log2 R (a hub list of 1,700 entries: 3 instead of 11).  Needs off[lo] <= e
// and off non-decreasing on [lo, hi].
template <class T>
__device__ __forceinline__ uint32_t warpOwnerOf(const T* off, uint32_t lo, uint32_t hi, T e) {
    const unsigned lane = threadIdx.x & 31u;
    while (hi - lo >= 32u) {
        const uint32_t step = (hi - lo) / 32u + 1u;  // 32 * step covers [lo, hi]
        const uint32_t i = lo + lane * step;
        const unsigned b = __ballot_sync(kFull, i <= hi && off[i] <= e);  // a prefix of the lanes, lane 0 set
        lo += (31u - __clz(b)) * step;
        hi = min(hi, lo + step - 1u);
    }
    const uint32_t i = lo + lane;
    const unsigned b = __ballot_sync(kFull, i <= hi && off[i] <= e);
    return lo + (31u - __clz(b));
}

}  // namespace gb
