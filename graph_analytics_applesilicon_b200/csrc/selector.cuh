// selector.cuh -- the learned per-level strategy selector.
//
// A two-hidden-layer ReLU MLP maps the on-device frontier counters of a BFS
// level to a predicted log2 run time (us) per strategy (gb_strategy); the
// persistent kernel runs the argmin.  No counterpart in the reference, whose
// direction choice is the alpha/beta rule of src/metal/bfs_gpu.mm:354-357,
// :416-420 (kept here as the fallback and as the judge).
#pragma once

#include <cmath>

#include "common.cuh"

namespace gb {

constexpr int kSelFeatures = 8;
constexpr int kSelHidden = 32;
constexpr int kSelOutputs = GB_NUM_STRATS;
constexpr int kSelParams = kSelHidden * kSelFeatures + kSelHidden + kSelHidden * kSelHidden + kSelHidden +
                           kSelOutputs * kSelHidden + kSelOutputs;

// Feature vector of a level (the same function on host and device; inputs
// are exact integer counters, converted to float first, and only float
// arithmetic follows, so a device level costs a few instructions per feature):
//   0 log2(1+frontier vertices)/32   1 log2(1+frontier edges)/32
//   2 log2(1+unexplored edges)/32    3 log2(1+unvisited vertices)/32
//   4 log2(1+n)/32                   5 log2(1+m)/32
//   6 min(level,255)/256             7 log2(1+frontier edges/frontier vertices)/16
__host__ __device__ inline void selectorFeatures(double frontier, double fedges, double unexplored,
                                                 double unvisited, double n, double m, double level,
                                                 float* f) {
    const float fr = (float)frontier, fe = (float)fedges;
    f[0] = log2f(1.0f + fr) * (1.0f / 32.0f);
    f[1] = log2f(1.0f + fe) * (1.0f / 32.0f);
    f[2] = log2f(1.0f + (float)unexplored) * (1.0f / 32.0f);
    f[3] = log2f(1.0f + (float)unvisited) * (1.0f / 32.0f);
    f[4] = log2f(1.0f + (float)n) * (1.0f / 32.0f);
    f[5] = log2f(1.0f + (float)m) * (1.0f / 32.0f);
    f[6] = (level < 255.0 ? (float)level : 255.0f) * (1.0f / 256.0f);
    f[7] = log2f(1.0f + fe / (fr > 1.0f ? fr : 1.0f)) * (1.0f / 16.0f);
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

// The same copy issued as asynchronous 4-byte copies (cp.async), so the
// threads go on with other work while the parameters arrive; the caller waits
// with selectorStageWait (each thread for its own copies) and a block barrier
// before the first evaluation.
__device__ __forceinline__ void selectorStageAsync(float* S, const float* P, unsigned tid, unsigned nthreads) {
    constexpr int oW1 = 0, oB1 = oW1 + kSelHidden * kSelFeatures, oW2 = oB1 + kSelHidden,
                  oB2 = oW2 + kSelHidden * kSelHidden, oW3 = oB2 + kSelHidden, oB3 = oW3 + kSelOutputs * kSelHidden;
    for (unsigned i = tid; i < (unsigned)kSelParams; i += nthreads) {
        unsigned dst = i;
        if (i < (unsigned)oB1) {
            const unsigned j = i / kSelFeatures, k = i % kSelFeatures;
            dst = oW1 + k * kSelHidden + j;
        } else if (i >= (unsigned)oW2 && i < (unsigned)oB2) {
            const unsigned r = i - oW2, j = r / kSelHidden, k = r % kSelHidden;
            dst = oW2 + k * kSelHidden + j;
        } else if (i >= (unsigned)oW3 && i < (unsigned)oB3) {
            const unsigned r = i - oW3, o = r / kSelHidden, k = r % kSelHidden;
            dst = oW3 + k * kSelOutputs + o;
        }
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(S + dst)),
                     "l"(P + i)
                     : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void selectorStageWait() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// One warp evaluates the MLP (lane j owns hidden unit j) on the features of
// a level and returns the strategy to run, or -1 if an output is not finite.
// ruleBU is the alpha/beta rule's direction; with margin 0 (and mayGoBU) the
// result is the strategy of smallest predicted time.  mayGoBU = false keeps a
// top-down level top-down (the caller's trust region around the rule).
// S is the shared-memory copy written by selectorStage.  Every lane returns
// the same value; the result depends only on the parameters and f, so every
// block of a grid that calls it on the same counters agrees.
__device__ __forceinline__ int selectorChoose(const float* S, const float* f, unsigned lane, bool ruleBU,
                                              float margin, bool mayGoBU = true) {
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
    // 32-term dot products in four independent partial sums (shorter dependency chains)
    float p2[4] = {b2[lane], 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int k = 0; k < kSelHidden; ++k) p2[k & 3] = fmaf(w2[k * kSelHidden + lane], __shfl_sync(kFull, h1, k), p2[k & 3]);
    const float h2 = fmaxf((p2[0] + p2[1]) + (p2[2] + p2[3]), 0.0f);
    const unsigned o = lane < kSelOutputs ? lane : 0;
    float p3[4] = {b3[o], 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int k = 0; k < kSelHidden; ++k) p3[k & 3] = fmaf(w3[k * kSelOutputs + o], __shfl_sync(kFull, h2, k), p3[k & 3]);
    const float out = (p3[0] + p3[1]) + (p3[2] + p3[3]);
    if (__any_sync(kFull, lane < kSelOutputs && !isfinite(out))) return -1;
    // the fastest top-down strategy (GB_STRAT_TD_EPT1..TD_WARP = 0..3), then
    // the direction: the rule's unless the other one is predicted faster by
    // more than `margin` (log2 time)
    float key = lane < GB_STRAT_BU ? out : 3.0e38f;
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
    const float tBU = __shfl_sync(kFull, out, GB_STRAT_BU);
    if (ruleBU) return key + margin < tBU ? idx : GB_STRAT_BU;
    return mayGoBU && tBU + margin < key ? GB_STRAT_BU : idx;
}
#endif

}  // namespace gb
