// selector.cuh -- the learned per-level strategy selector.
//
// A two-hidden-layer ReLU MLP maps the on-device frontier counters of a BFS
// level to a predicted log2 run time (us) per strategy (gb_strategy); the
// persistent kernel runs the argmin.  No counterpart in the reference, whose
// direction choice is the alpha/beta rule of src/metal/bfs_gpu.mm:354-357,
// :416-420 (kept here as the fallback and as the judge).
#pragma once

#include "common.cuh"

namespace gb {

constexpr int kSelFeatures = 8;
constexpr int kSelHidden = 32;
constexpr int kSelOutputs = GB_NUM_STRATS;
constexpr int kSelParams = kSelHidden * kSelFeatures + kSelHidden + kSelHidden * kSelHidden + kSelHidden +
                           kSelOutputs * kSelHidden + kSelOutputs;

// Feature vector of a level (the same on host and device, all inputs exact
// integers from the level counters):
//   0 log2(1+frontier vertices)/32   1 log2(1+frontier edges)/32
//   2 log2(1+unexplored edges)/32    3 log2(1+unvisited vertices)/32
//   4 log2(1+n)/32                   5 log2(1+m)/32
//   6 min(level,255)/256             7 log2(1+frontier edges/frontier vertices)/16
__host__ __device__ inline void selectorFeatures(double frontier, double fedges, double unexplored,
                                                 double unvisited, double n, double m, double level,
                                                 float* f) {
    f[0] = (float)(log2(1.0 + frontier) / 32.0);
    f[1] = (float)(log2(1.0 + fedges) / 32.0);
    f[2] = (float)(log2(1.0 + unexplored) / 32.0);
    f[3] = (float)(log2(1.0 + unvisited) / 32.0);
    f[4] = (float)(log2(1.0 + n) / 32.0);
    f[5] = (float)(log2(1.0 + m) / 32.0);
    f[6] = (float)((level < 255.0 ? level : 255.0) / 256.0);
    f[7] = (float)(log2(1.0 + fedges / (frontier > 1.0 ? frontier : 1.0)) / 16.0);
}

#ifdef __CUDACC__
// Copy the parameters (layout: W1[32][8], b1, W2[32][32], b2, W3[5][32], b3,
// row-major, as trained) into shared memory with every weight matrix
// transposed, so that in selectorArgmin the 32 lanes of a warp read 32
// consecutive words per step (conflict-free) instead of one bank 32 times.
__device__ __forceinline__ void selectorStage(float* S, const float* P, unsigned tid, unsigned nthreads) {
    constexpr int oW1 = 0, oB1 = oW1 + kSelHidden * kSelFeatures, oW2 = oB1 + kSelHidden,
                  oB2 = oW2 + kSelHidden * kSelHidden, oW3 = oB2 + kSelHidden, oB3 = oW3 + kSelOutputs * kSelHidden;
    for (unsigned i = tid; i < (unsigned)kSelParams; i += nthreads) {
        unsigned dst = i;
        if (i < (unsigned)oB1) {  // W1[j][k] -> [k][j]
            const unsigned j = i / kSelFeatures, k = i % kSelFeatures;
            dst = oW1 + k * kSelHidden + j;
        } else if (i >= (unsigned)oW2 && i < (unsigned)oB2) {  // W2[j][k] -> [k][j]
            const unsigned r = i - oW2, j = r / kSelHidden, k = r % kSelHidden;
            dst = oW2 + k * kSelHidden + j;
        } else if (i >= (unsigned)oW3 && i < (unsigned)oB3) {  // W3[o][k] -> [k][o]
            const unsigned r = i - oW3, o = r / kSelHidden, k = r % kSelHidden;
            dst = oW3 + k * kSelOutputs + o;
        }
        S[dst] = P[i];
    }
}

// One warp evaluates the MLP (lane j owns hidden unit j) and returns the
// strategy with the smallest predicted time, or -1 if an output is not finite.
// S is the shared-memory copy written by selectorStage.  Every lane returns
// the same value; the result depends only on the parameters and f, so every
// block of a grid that calls it on the same counters agrees.
__device__ __forceinline__ int selectorArgmin(const float* S, const float* f, unsigned lane) {
    const float* w1 = S;  // [k][j]
    const float* b1 = w1 + kSelHidden * kSelFeatures;
    const float* w2 = b1 + kSelHidden;  // [k][j]
    const float* b2 = w2 + kSelHidden * kSelHidden;
    const float* w3 = b2 + kSelHidden;  // [k][o]
    const float* b3 = w3 + kSelOutputs * kSelHidden;
    float h1 = b1[lane];
#pragma unroll
    for (int k = 0; k < kSelFeatures; ++k) h1 = fmaf(w1[k * kSelHidden + lane], f[k], h1);
    h1 = fmaxf(h1, 0.0f);
    float h2 = b2[lane];
#pragma unroll
    for (int k = 0; k < kSelHidden; ++k) h2 = fmaf(w2[k * kSelHidden + lane], __shfl_sync(kFull, h1, k), h2);
    h2 = fmaxf(h2, 0.0f);
    const unsigned o = lane < kSelOutputs ? lane : 0;
    float out = b3[o];
#pragma unroll
    for (int k = 0; k < kSelHidden; ++k) out = fmaf(w3[k * kSelOutputs + o], __shfl_sync(kFull, h2, k), out);
    bool bad = lane < kSelOutputs && !isfinite(out);
    float key = lane < kSelOutputs ? out : 3.0e38f;
    int idx = (int)lane;
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        float k2 = __shfl_xor_sync(kFull, key, s);
        int i2 = __shfl_xor_sync(kFull, idx, s);
        if (k2 < key || (k2 == key && i2 < idx)) {
            key = k2;
            idx = i2;
        }
    }
    return __any_sync(kFull, bad) ? -1 : idx;
}
#endif

}  // namespace gb
