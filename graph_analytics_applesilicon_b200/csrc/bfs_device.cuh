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

}  // namespace gb
