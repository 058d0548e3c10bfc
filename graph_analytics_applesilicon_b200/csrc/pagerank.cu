// pagerank.cu -- PageRank on the GPU: push, scalar / vector / degree-adaptive
// pull, in-place (Gauss-Seidel) sweeps and a double-precision pull oracle.
//
// Definition (src/cpu/pagerank_cpu.hpp:4-8): d = 0.85, r0 = 1/n,
//   r_new[v] = (1-d)/n + d * (sum_{u in in(v)} r[u]/outdeg[u] + dangling/n).
// Precision (FP32 ranks): per-vertex sums are Kahan-compensated (the star's
// hub has 100k equal terms, src/shaders/pagerank.metal:27-42); the dangling
// mass is a float-float (TwoSum) accumulation; the L1 residual and the
// in-place renormalisation sum are FP64.  push uses compensated float atomics
// (TwoSum error into a second accumulator, src/shaders/pagerank.metal:196-226).
//
// Structure (B200): one kernel per Jacobi iteration does the gather, the
// store, the next iteration's contributions r/outdeg, the dangling mass and
// (tol mode) the residual; its last block to finish (ticket on the control
// block) reduces the per-block partials in a fixed order and advances the
// iteration control on the device.  Iterations are therefore independent of
// the host and replayed as CUDA graphs: fixed mode is one graph, tol mode
// graphs of 8 iterations with one host check per batch (the reference
// synchronises every iteration, src/metal/pagerank_gpu.mm:384-405).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>

#include "pagerank.hpp"

namespace gb {
namespace {

constexpr int kMaxGrid = 4096;
constexpr int kGraphBatch = 8;

struct PrArgs {
    const uint32_t* rp;
    const uint32_t* ci;
    const uint32_t* outdeg;
    float* r[2];
    float* contrib[2];
    double* r64[2];
    double* contrib64[2];
    float* acc;
    float* accLo;
    const uint32_t* list;  // GS natural: the list to sweep
    GbPrControl* ctl;
    float* partF;
    double* partD;
    uint32_t n;
    float damping, base, invN;
    double base64, invN64, damping64;
    uint32_t lo, hi;  // GS colored: id range of the set
    // split vertices: chunk table, per-hub (first, count), tickets, partials
    const uint4* chunks;
    const uint32_t* hubFirst;
    unsigned* hubDone;
    float* hubPart;   // indexed by global chunk index
    uint32_t nChunks;
    uint32_t chunkBase;  // global chunk index of chunks[0]
    // degree classes of the relabeled layout: ids [binLo, binHi) use groups of binG lanes
    uint32_t binLo[8], binHi[8], binG[8];
    int nBins;
};

struct Kahan {
    float sum = 0.f, comp = 0.f;
    __device__ __forceinline__ void add(float x) {
        float y = x - comp;
        float t = sum + y;
        comp = (t - sum) - y;
        sum = t;
    }
};

// float-float accumulator: (hi, lo) with |lo| << |hi|, combined by TwoSum.
struct FF {
    float hi = 0.f, lo = 0.f;
    __device__ __forceinline__ void add(float x) {
        float s = hi + x;
        float bp = s - hi;
        float err = (hi - (s - bp)) + (x - bp);
        hi = s;
        lo += err;
    }
    __device__ __forceinline__ void add(FF o) {
        add(o.hi);
        lo += o.lo;
    }
};

__device__ __forceinline__ int ldvi(const int* p) { return *reinterpret_cast<const volatile int*>(p); }

__device__ __forceinline__ float prValue(const PrArgs& a, float s, float dang) {
    return a.base + a.damping * (s + dang * a.invN);  // pr_value, src/shaders/pagerank.metal:45-48
}

// Per-thread accumulators of one iteration.
struct IterAcc {
    FF dang;
    double dsum = 0;
    float dmax = 0;
    double d64 = 0;
};

// Store of vertex v in a Jacobi iteration: r_new, the next contribution, the
// dangling mass and the residual against the previous iterate.
__device__ __forceinline__ void storeJacobi(const PrArgs& a, int cur, bool withDelta, uint32_t v, float val,
                                            IterAcc& acc) {
    a.r[cur ^ 1][v] = val;
    const uint32_t od = a.outdeg[v];
    a.contrib[cur ^ 1][v] = od ? val / (float)od : 0.0f;
    if (!od) acc.dang.add(val);
    if (withDelta) {
        const float o = a.r[cur][v];
        const double d = fabs((double)val - (double)o);
        acc.dsum += d;
        acc.dmax = fmaxf(acc.dmax, (float)d / fmaxf(val, a.invN));
    }
}

// Block-wide reduction of IterAcc into thread 0 (fixed order: deterministic).
__device__ __forceinline__ IterAcc blockReduceAcc(IterAcc acc) {
    __shared__ float sHi[32], sLo[32], sMax[32];
    __shared__ double sSum[32], s64[32];
    const unsigned lane = laneId(), wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        FF other;
        other.hi = __shfl_xor_sync(kFull, acc.dang.hi, o);
        other.lo = __shfl_xor_sync(kFull, acc.dang.lo, o);
        if (lane < (unsigned)o) acc.dang.add(other);  // lane 0 ends with the exact warp total
        acc.dsum += __shfl_xor_sync(kFull, acc.dsum, o);
        acc.d64 += __shfl_xor_sync(kFull, acc.d64, o);
        acc.dmax = fmaxf(acc.dmax, __shfl_xor_sync(kFull, acc.dmax, o));
    }
    if (lane == 0) {
        sHi[wid] = acc.dang.hi;
        sLo[wid] = acc.dang.lo;
        sSum[wid] = acc.dsum;
        s64[wid] = acc.d64;
        sMax[wid] = acc.dmax;
    }
    __syncthreads();
    IterAcc t;
    if (threadIdx.x == 0) {
        for (unsigned w = 0; w < nw; ++w) {
            FF x;
            x.hi = sHi[w];
            x.lo = sLo[w];
            t.dang.add(x);
            t.dsum += sSum[w];
            t.d64 += s64[w];
            t.dmax = fmaxf(t.dmax, sMax[w]);
        }
    }
    __syncthreads();
    return t;
}

// Each block writes its partials; the last block to finish (ticket on the
// control block) reduces all partials in a fixed order and updates the
// control block:
//   kind 0: Jacobi iteration (dangling + residual + iteration advance)
//   kind 1: contribution pass (dangling only)
//   kind 2: renormalisation sum (sum64 only)
//   kind 3: in-place scale (residual + iteration advance)
//   kind 4: FP64 Jacobi iteration (dang64 + residual + advance)
//   kind 5: FP64 initialisation (dang64 only)
template <int KIND>
__device__ void finishBlock(const PrArgs& a, IterAcc acc) {
    __shared__ bool sLast;
    IterAcc b = blockReduceAcc(acc);
    if (threadIdx.x == 0) {
        a.partF[2 * blockIdx.x] = b.dang.hi;
        a.partF[2 * blockIdx.x + 1] = b.dang.lo;
        a.partD[3 * blockIdx.x] = b.dsum;
        a.partD[3 * blockIdx.x + 1] = b.d64;
        a.partD[3 * blockIdx.x + 2] = b.dmax;
        __threadfence();
        sLast = atomicAdd(&a.ctl->done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!sLast) return;
    __threadfence();
    IterAcc p;
    for (unsigned k = threadIdx.x; k < gridDim.x; k += blockDim.x) {
        FF x;
        x.hi = __ldcg(&a.partF[2 * k]);
        x.lo = __ldcg(&a.partF[2 * k + 1]);
        p.dang.add(x);
        p.dsum += __ldcg(&a.partD[3 * k]);
        p.d64 += __ldcg(&a.partD[3 * k + 1]);
        p.dmax = fmaxf(p.dmax, (float)__ldcg(&a.partD[3 * k + 2]));
    }
    IterAcc t = blockReduceAcc(p);
    if (threadIdx.x != 0) return;
    GbPrControl* c = a.ctl;
    c->done = 0;
    if (KIND == 0 || KIND == 1) {
        c->dangHi = t.dang.hi;
        c->dangLo = t.dang.lo;
    }
    if (KIND == 4 || KIND == 5) c->dang64 = t.d64;
    if (KIND == 2) c->sum64 = t.dsum;
    if (KIND == 0 || KIND == 3 || KIND == 4) {
        c->iters += 1;
        c->cur ^= 1;
        if (c->withDelta) {
            const double sum = t.dsum;
            const float mx = t.dmax;
            c->lastDelta = sum;
            c->lastMaxRel = mx;
            if (sum < c->tol && (c->tolRel <= 0 || mx < c->tolRel)) {
                c->stopped = 1;
            } else if (sum < c->best) {
                c->best = sum;
                c->sinceBest = 0;
            } else if (++c->sinceBest >= 5) {
                c->stopped = 1;
                c->floorStop = 1;
            }
        }
        if (c->iters >= c->cap) c->stopped = 1;
    }
}

// r = 1/n, contrib = r/outdeg, dangling mass.
__global__ void prInitKernel(PrArgs a) {
    IterAcc acc;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < a.n; base += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t v = base + threadIdx.x;
        if (v < a.n) {
            a.r[0][v] = a.invN;
            const uint32_t od = a.outdeg[v];
            a.contrib[0][v] = od ? a.invN / (float)od : 0.0f;
            if (!od) acc.dang.add(a.invN);
        }
    }
    finishBlock<1>(a, acc);
}

__global__ void prInit64Kernel(PrArgs a) {
    IterAcc acc;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < a.n; base += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t v = base + threadIdx.x;
        if (v < a.n) {
            a.r64[0][v] = a.invN64;
            const uint32_t od = a.outdeg[v];
            a.contrib64[0][v] = od ? a.invN64 / (double)od : 0.0;
            if (!od) acc.d64 += a.invN64;
        }
    }
    finishBlock<5>(a, acc);
}

// Kahan sum of contrib over v's in-list [b, e), lanes of a group of G threads
// striding it; 16-byte aligned vector loads of col_idx (entries outside
// [b, e) are masked; the array is padded so the last vector stays in bounds).
// Adjacency (col_idx) is read once per sweep: load it without allocating in
// L1, so L1 keeps the contributions that many rows gather (hub-first order
// puts the most-gathered ones together).
__device__ __forceinline__ uint4 ldStream4(const uint32_t* p) {
    uint4 v;
    asm("ld.global.nc.L1::no_allocate.v4.u32 {%0, %1, %2, %3}, [%4];"
        : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
        : "l"(p));
    return v;
}
__device__ __forceinline__ uint32_t ldStream(const uint32_t* p) {
    uint32_t v;
    asm("ld.global.nc.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

template <bool COHERENT>
__device__ __forceinline__ float ldContrib(const float* p) {
    if (COHERENT) return *reinterpret_cast<const volatile float*>(p);  // rewritten during the sweep
    return __ldg(p);
}

template <int G, bool COHERENT = false>
__device__ __forceinline__ float gatherStrided(const uint32_t* __restrict__ ci, const float* contrib, uint32_t b,
                                               uint32_t e, unsigned rank) {
    Kahan k;
    for (uint32_t i = (b & ~3u) + 4 * rank; i < e; i += 4 * G) {
        const uint4 q = ldStream4(ci + i);
        if (i >= b) k.add(ldContrib<COHERENT>(contrib + q.x));
        if (i + 1 >= b && i + 1 < e) k.add(ldContrib<COHERENT>(contrib + q.y));
        if (i + 2 >= b && i + 2 < e) k.add(ldContrib<COHERENT>(contrib + q.z));
        if (i + 3 >= b && i + 3 < e) k.add(ldContrib<COHERENT>(contrib + q.w));
    }
    return k.sum;
}

template <bool COHERENT = false>
__device__ __forceinline__ float gatherSerial(const uint32_t* __restrict__ ci, const float* contrib, uint32_t b,
                                              uint32_t e) {
    Kahan k;
    for (uint32_t i = b; i < e; ++i) k.add(ldContrib<COHERENT>(contrib + ldStream(ci + i)));
    return k.sum;
}

// Kahan sum of contrib over [b, e) by group rank `rank` of G lanes (runtime
// G), 16-byte aligned vector loads of col_idx.
template <bool COHERENT>
__device__ __forceinline__ float gatherGroup(const uint32_t* __restrict__ ci, const float* contrib, uint32_t b,
                                             uint32_t e, unsigned rank, unsigned G) {
    // Two 16-byte vectors per lane per step (8 gathers in flight); entries
    // are added in the same per-lane order as a one-vector loop.
    Kahan k;
    const uint32_t step = 4 * G;
    for (uint32_t i = (b & ~3u) + 4 * rank; i < e; i += 2 * step) {
        const uint32_t j = i + step;
        const uint4 q = ldStream4(ci + i);
        const uint4 r = j < e ? ldStream4(ci + j) : make_uint4(0, 0, 0, 0);
        const float a0 = (i >= b) ? ldContrib<COHERENT>(contrib + q.x) : 0.f;
        const float a1 = (i + 1 >= b && i + 1 < e) ? ldContrib<COHERENT>(contrib + q.y) : 0.f;
        const float a2 = (i + 2 >= b && i + 2 < e) ? ldContrib<COHERENT>(contrib + q.z) : 0.f;
        const float a3 = (i + 3 >= b && i + 3 < e) ? ldContrib<COHERENT>(contrib + q.w) : 0.f;
        const float b0 = (j < e) ? ldContrib<COHERENT>(contrib + r.x) : 0.f;
        const float b1 = (j + 1 < e) ? ldContrib<COHERENT>(contrib + r.y) : 0.f;
        const float b2 = (j + 2 < e) ? ldContrib<COHERENT>(contrib + r.z) : 0.f;
        const float b3 = (j + 3 < e) ? ldContrib<COHERENT>(contrib + r.w) : 0.f;
        k.add(a0);
        k.add(a1);
        k.add(a2);
        k.add(a3);
        k.add(b0);
        k.add(b1);
        k.add(b2);
        k.add(b3);
    }
    return k.sum;
}

// One warp chunk of a split vertex: the warp's sum goes to the chunk's
// partial; the warp finishing the vertex's last chunk (ticket per vertex)
// adds the partials in chunk order (Kahan) and stores the vertex.  All 32
// lanes call it; store() runs on lane 0.
template <bool COHERENT, class Store>
__device__ __forceinline__ void chunkTask(const PrArgs& a, uint32_t t, const float* contrib, Store store) {
    const uint4 c = a.chunks[t];  // vertex, start, end, hub
    float s = gatherGroup<COHERENT>(a.ci, contrib, c.y, c.z, laneId(), 32);
    s = warpSum(s);
    if (laneId() == 0) {
        a.hubPart[a.chunkBase + t] = s;
        __threadfence();
        const uint32_t first = a.hubFirst[2 * c.w], cnt = a.hubFirst[2 * c.w + 1];
        if (atomicAdd(&a.hubDone[c.w], 1u) == cnt - 1) {
            __threadfence();
            Kahan k;
            for (uint32_t i = 0; i < cnt; ++i) k.add(__ldcg(&a.hubPart[first + i]));
            a.hubDone[c.w] = 0;
            store(c.x, k.sum);
        }
    }
}

// Jacobi pull iteration.  MODE 0: thread per vertex (gpu_pull_scalar);
// 1: warp per vertex (gpu_pull_vector); 2: degree-adaptive over the three
// in-degree bins in one launch (block per large, warp per medium, thread per
// small vertex; gpu_pull_adaptive).  INPLACE: the sweep of an in-place
// variant -- contributions are read and rewritten in contrib[0] as vertices
// are updated, and dangling / residual / control are left to the
// contribution, sum and scale kernels.
template <int MODE, bool INPLACE>
__global__ void prPullKernel(PrArgs a) {
    const GbPrControl* c = a.ctl;
    if (ldvi(&c->stopped)) return;
    const int cur = c->cur;
    const float dang = c->dangHi + c->dangLo;
    const bool withDelta = !INPLACE && c->withDelta;
    const float* contrib = INPLACE ? a.contrib[0] : a.contrib[cur];
    IterAcc acc;
    auto store = [&](uint32_t v, float s) {
        const float val = prValue(a, s, dang);
        if (INPLACE) {
            a.r[cur ^ 1][v] = val;
            const uint32_t od = a.outdeg[v];
            a.contrib[0][v] = od ? val / (float)od : 0.0f;
        } else {
            storeJacobi(a, cur, withDelta, v, val, acc);
        }
    };
    const uint64_t gthreads = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t gtid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (MODE == 0) {
        for (uint64_t v = gtid; v < a.n; v += gthreads)
            store((uint32_t)v, gatherSerial<INPLACE>(a.ci, contrib, a.rp[v], a.rp[v + 1]));
    } else if (MODE == 1) {
        const uint64_t nwarps = gthreads >> 5;
        for (uint64_t v = gtid >> 5; v < a.n; v += nwarps) {
            float s = gatherStrided<32, INPLACE>(a.ci, contrib, a.rp[v], a.rp[v + 1], laneId());
            s = warpSum(s);
            if (laneId() == 0) store((uint32_t)v, s);
        }
    } else {
        // degree-adaptive over the hub-first relabeled graph: task space =
        // chunks of split vertices, then warp tasks of each degree class
        uint64_t total = a.nChunks;
        for (int b = 0; b < a.nBins; ++b) total += ((uint64_t)(a.binHi[b] - a.binLo[b]) * a.binG[b] + 31) / 32;
        const uint64_t nwarps = gthreads >> 5;
        const unsigned lane = laneId();
        for (uint64_t t = gtid >> 5; t < total; t += nwarps) {  // warp-uniform
            if (t < a.nChunks) {
                chunkTask<INPLACE>(a, (uint32_t)t, contrib, store);
                continue;
            }
            uint64_t tb = t - a.nChunks;
            int b = 0;
            for (; b < a.nBins; ++b) {
                const uint64_t nt = ((uint64_t)(a.binHi[b] - a.binLo[b]) * a.binG[b] + 31) / 32;
                if (tb < nt) break;
                tb -= nt;
            }
            const unsigned G = a.binG[b];
            const uint32_t v = a.binLo[b] + (uint32_t)tb * (32 / G) + lane / G;
            const bool active = v < a.binHi[b];
            float s = active ? gatherGroup<INPLACE>(a.ci, contrib, a.rp[v], a.rp[v + 1], lane & (G - 1), G) : 0.f;
            for (unsigned o = G >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
            if (active && (lane & (G - 1)) == 0) store(v, s);
        }
    }
    if (!INPLACE) finishBlock<0>(a, acc);
}

// In-place sweep over a vertex list, warp per vertex (natural GS order; the
// deferred mutual-pair partners form a second list swept afterwards).
// Vertices with >= kGsHubMin in-edges are swept by gsHubKernel instead.
__global__ void gsSweepListKernel(PrArgs a, uint32_t count) {
    const GbPrControl* c = a.ctl;
    if (ldvi(&c->stopped)) return;
    const int cur = c->cur;
    const float dang = c->dangHi + c->dangLo;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < count; i += nwarps) {
        const uint32_t v = a.list[i];
        const uint32_t b = a.rp[v], e = a.rp[v + 1];
        if (e - b >= kGsHubMin) continue;  // warp-uniform
        float s = gatherGroup<true>(a.ci, a.contrib[0], b, e, laneId(), 32);
        s = warpSum(s);
        if (laneId() == 0) {
            const float val = prValue(a, s, dang);
            a.r[cur ^ 1][v] = val;
            const uint32_t od = a.outdeg[v];
            a.contrib[0][v] = od ? val / (float)od : 0.0f;
        }
    }
}

// In-place sweep of the split vertices (natural GS order), warp per chunk.
__global__ void gsHubKernel(PrArgs a) {
    const GbPrControl* c = a.ctl;
    if (ldvi(&c->stopped)) return;
    const int cur = c->cur;
    const float dang = c->dangHi + c->dangLo;
    auto store = [&](uint32_t v, float s) {
        const float val = prValue(a, s, dang);
        a.r[cur ^ 1][v] = val;
        const uint32_t od = a.outdeg[v];
        a.contrib[0][v] = od ? val / (float)od : 0.0f;
    };
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t t = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < a.nChunks; t += nwarps)
        chunkTask<true>(a, (uint32_t)t, a.contrib[0], store);
}

// In-place variants: contributions and dangling mass of the current iterate.
__global__ void gsContribKernel(PrArgs a) {
    const GbPrControl* c = a.ctl;
    if (ldvi(&c->stopped)) return;
    const int cur = c->cur;
    IterAcc acc;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < a.n; base += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t v = base + threadIdx.x;
        if (v < a.n) {
            const float r = a.r[cur][v];
            const uint32_t od = a.outdeg[v];
            a.contrib[0][v] = od ? r / (float)od : 0.0f;
            if (!od) acc.dang.add(r);
        }
    }
    finishBlock<1>(a, acc);
}

// FP64 sum of the new iterate (renormalisation, src/shaders/pagerank.metal:86-117).
__global__ void prSumKernel(PrArgs a) {
    const GbPrControl* c = a.ctl;
    if (ldvi(&c->stopped)) return;
    const float* rn = a.r[c->cur ^ 1];
    IterAcc acc;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < a.n; v += (uint64_t)gridDim.x * blockDim.x)
        acc.dsum += (double)rn[v];
    finishBlock<2>(a, acc);
}

// Scale the new iterate to sum 1 (FP64 division), residual, advance.
__global__ void prScaleKernel(PrArgs a) {
    const GbPrControl* c = a.ctl;
    if (ldvi(&c->stopped)) return;
    const int cur = c->cur;
    const double sum = c->sum64;
    const bool withDelta = c->withDelta;
    IterAcc acc;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < a.n; base += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t v = base + threadIdx.x;
        if (v < a.n) {
            const float val = (float)((double)a.r[cur ^ 1][v] / sum);
            a.r[cur ^ 1][v] = val;
            if (withDelta) {
                const float o = a.r[cur][v];
                const double d = fabs((double)val - (double)o);
                acc.dsum += d;
                acc.dmax = fmaxf(acc.dmax, (float)d / fmaxf(val, a.invN));
            }
        }
    }
    finishBlock<3>(a, acc);
}

// gpu_push: thread per source vertex scatters its contribution with float
// atomics.  When every active lane of a warp targets the same vertex (a hub's
// in-neighbours), the lanes sum first and issue one atomic.  Each atomic's
// rounding error is recovered exactly by TwoSum against the returned old
// value and, when it exceeds 2^-16 of the term, added to a second
// accumulator (src/shaders/pagerank.metal:196-226).
__device__ __forceinline__ void addCompensated(float* acc, float* accLo, uint32_t t, float x) {
    const float old = atomicAdd(&acc[t], x);
    const float s = old + x;
    const float bp = s - old;
    const float err = (old - (s - bp)) + (x - bp);
    if (fabsf(err) > fabsf(x) * 0x1p-16f) atomicAdd(&accLo[t], err);
}

__global__ void prPushKernel(PrArgs a, const uint32_t* __restrict__ rowOut, const uint32_t* __restrict__ colOut) {
    const GbPrControl* c = a.ctl;
    if (ldvi(&c->stopped)) return;
    const float* contrib = a.contrib[c->cur];
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < a.n; base += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t u = base + threadIdx.x;
        const bool active = u < a.n;
        const float cu = active ? contrib[u] : 0.0f;
        const uint32_t b = active ? rowOut[u] : 0u;
        const uint32_t deg = (active && cu != 0.0f) ? rowOut[u + 1] - b : 0u;
        const uint32_t rounds = __reduce_max_sync(kFull, deg);
        for (uint32_t k = 0; k < rounds; ++k) {
            const bool has = k < deg;
            const uint32_t t = has ? colOut[b + k] : 0xFFFFFFFFu;
            const uint32_t lead = __reduce_min_sync(kFull, t);
            if (__all_sync(kFull, !has || t == lead)) {
                const float s = warpSum(has ? cu : 0.0f);
                if (laneId() == 0) addCompensated(a.acc, a.accLo, lead, s);
            } else if (has) {
                addCompensated(a.acc, a.accLo, t, cu);
            }
        }
    }
}

__global__ void prPushFinalizeKernel(PrArgs a) {
    const GbPrControl* c = a.ctl;
    if (ldvi(&c->stopped)) return;
    const int cur = c->cur;
    const float dang = c->dangHi + c->dangLo;
    const bool withDelta = c->withDelta;
    IterAcc acc;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < a.n; base += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t v = base + threadIdx.x;
        if (v < a.n) {
            const float val = prValue(a, a.acc[v] + a.accLo[v], dang);
            a.acc[v] = 0.0f;
            a.accLo[v] = 0.0f;
            storeJacobi(a, cur, withDelta, (uint32_t)v, val, acc);
        }
    }
    finishBlock<0>(a, acc);
}

// ---------------------------------------------------------------- blocked pull
// Rows in row blocks whose sums live in shared memory, columns in parts of
// kBlkPart vertices whose contributions are staged in shared memory, so no
// gather reaches L2: an edge costs 4 bytes of a streamed tile, one shared-
// memory gather and one shared-memory float atomic add.  One CUDA block of
// kBlkThreads per row block (one per SM at the graph sizes this form is for),
// warp-specialized:
//   warp 0, one thread: the producer.  It walks the block's non-empty tiles
//     (row block k, part p), parts in an order rotated by k so the SMs stage
//     different contributions at once, and issues TMA bulk copies
//     (cp.async.bulk) of part p's contributions into a ring of kBlkCStages
//     stages and of the tile's packed edge words, in chunks of at most
//     kBlkChunk words, into a ring of kBlkEStages stages.  Each copy completes
//     on its stage's `full` mbarrier; a stage is refilled only after every
//     consumer warp has arrived on its `empty` mbarrier.
//   warps 1..kBlkConsumerWarps: the consumers.  For every chunk each thread
//     takes one 16-byte word (four edges) from the edge ring and adds the
//     staged contributions into the row sums.  Warps wait only on the stages
//     they read, so they drift across parts and row blocks; no block barrier
//     runs per part.  A named barrier among the consumers separates row
//     blocks (sums stored, then zeroed for the next block).
// The producer runs up to kBlkCStages parts and kBlkEStages chunks ahead,
// across row-block boundaries.  Rows with kBlkHub or more in-edges are summed
// afterwards by one block each with Kahan-compensated per-thread sums
// combined as float-float; the other rows' sums are plain FP32 (fewer than
// kBlkHub terms).  Every mbarrier wait is bounded: a thread whose wait gives
// up raises the block's failure flag and stops issuing or consuming; the
// others then time out on the stages it no longer fills or frees, the
// consumers agree at their named barrier, the producer waits (bounded) for
// the copies it has in flight, and the block records the error and leaves.
struct BlkArgs {
    const uint4* edges;     // tiles of packed (row in block << 16 | column in part) words, 0xFFFFFFFF padding
    const uint32_t* off;    // 16-byte-word offset of tile (k, p) at k * nParts + p, then the end
    const uint32_t* hubs;
    uint32_t nRowBlocks, rowsPer, nParts, nHubs;
    unsigned long long spinLimit;
};

__device__ __forceinline__ uint32_t smemAddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Waits for the given phase parity of an mbarrier; gives up after `limit` polls.
__device__ __forceinline__ bool blkWait(unsigned long long* mbar, uint32_t parity, unsigned long long limit) {
    const uint32_t addr = smemAddr(mbar);
    for (unsigned long long i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void blkArrive(unsigned long long* mbar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smemAddr(mbar)) : "memory");
}

// One bulk copy of `bytes` (a multiple of 16, both addresses 16-byte
// aligned) from global memory into shared memory, completing on `mbar`.
__device__ __forceinline__ void blkCopy(void* dst, const void* src, uint32_t bytes, unsigned long long* mbar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smemAddr(mbar)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smemAddr(dst)),
                 "l"(src), "r"(bytes), "r"(smemAddr(mbar))
                 : "memory");
}

// Named barrier 1 among the consumer threads; returns whether any of them
// passed `pred`.
__device__ __forceinline__ bool consumersOr(bool pred) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbarrier.cta.red.or.pred q, 1, %2, p;\n\tselp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)pred), "n"(kBlkConsumerWarps * 32)
        : "memory");
    return r != 0;
}

// The four edges of one 16-byte word into the row sums.
__device__ __forceinline__ void blkAdd(float* sums, const float* part, uint4 w) {
    if (w.x != 0xFFFFFFFFu) atomicAdd(&sums[w.x >> 16], part[w.x & 0xFFFFu]);
    if (w.y != 0xFFFFFFFFu) atomicAdd(&sums[w.y >> 16], part[w.y & 0xFFFFu]);
    if (w.z != 0xFFFFFFFFu) atomicAdd(&sums[w.z >> 16], part[w.z & 0xFFFFu]);
    if (w.w != 0xFFFFFFFFu) atomicAdd(&sums[w.w >> 16], part[w.w & 0xFFFFu]);
}

__global__ void __launch_bounds__(kBlkThreads, 1) prBlockedKernel(PrArgs a, BlkArgs b) {
    // [contribution ring][edge ring][row sums]
    extern __shared__ __align__(128) float blkSmem[];
    float* cring = blkSmem;
    uint4* ering = reinterpret_cast<uint4*>(blkSmem + kBlkCStages * kBlkPart);
    float* sums = reinterpret_cast<float*>(ering + kBlkEStages * kBlkChunk);
    __shared__ __align__(8) unsigned long long cFull[kBlkCStages], cEmpty[kBlkCStages];
    __shared__ __align__(8) unsigned long long eFull[kBlkEStages], eEmpty[kBlkEStages];
    __shared__ int sFailed;
    const GbPrControl* c = a.ctl;
    if (ldvi(&c->stopped)) return;
    const int cur = c->cur;
    const bool withDelta = c->withDelta;
    const float dang = c->dangHi + c->dangLo;
    const float* contrib = a.contrib[cur];
    const unsigned tid = threadIdx.x, warp = tid >> 5;
    if (tid == 0) {
        for (int i = 0; i < kBlkCStages; ++i) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smemAddr(&cFull[i])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddr(&cEmpty[i])),
                         "r"(kBlkConsumerWarps)
                         : "memory");
        }
        for (int i = 0; i < kBlkEStages; ++i) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smemAddr(&eFull[i])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddr(&eEmpty[i])),
                         "r"(kBlkConsumerWarps)
                         : "memory");
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        sFailed = 0;
    }
    __syncthreads();
    auto tileOf = [&](uint32_t k, uint32_t j, uint32_t& w0, uint32_t& w1) {
        const uint32_t rot = (uint32_t)((uint64_t)k * b.nParts / b.nRowBlocks);
        const uint32_t p = j + rot < b.nParts ? j + rot : j + rot - b.nParts;
        const uint64_t g = (uint64_t)k * b.nParts + p;
        w0 = b.off[g];
        w1 = b.off[g + 1];
        return p;
    };
    IterAcc acc;
    if (warp == 0) {
        if (tid == 0) {
            // producer: parts staged (ci) and chunks issued (ei) so far
            uint32_t ci = 0, ei = 0;
            bool ok = true;
            for (uint32_t k = blockIdx.x; k < b.nRowBlocks && ok; k += gridDim.x) {
                for (uint32_t j = 0; j < b.nParts && ok; ++j) {
                    uint32_t w0, w1;
                    const uint32_t p = tileOf(k, j, w0, w1);
                    if (w0 == w1) continue;
                    const uint32_t cs = ci % kBlkCStages;
                    if (ci >= kBlkCStages) ok = blkWait(&cEmpty[cs], (ci / kBlkCStages - 1) & 1u, b.spinLimit);
                    if (!ok) break;
                    // whole 16-byte groups: the contribution arrays carry 4 floats of slack past n
                    const uint32_t first = p * kBlkPart;
                    const uint32_t bytes = ((min(kBlkPart, (uint32_t)a.n - first) * 4u) + 15u) & ~15u;
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    blkCopy(cring + cs * kBlkPart, contrib + first, bytes, &cFull[cs]);
                    ++ci;
                    for (uint32_t w = w0; w < w1; w += kBlkChunk) {
                        const uint32_t es = ei % kBlkEStages;
                        if (ei >= kBlkEStages) ok = blkWait(&eEmpty[es], (ei / kBlkEStages - 1) & 1u, b.spinLimit);
                        if (!ok) break;
                        const uint32_t words = min(kBlkChunk, w1 - w);
                        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                        blkCopy(ering + es * kBlkChunk, b.edges + w, words * 16u, &eFull[es]);
                        ++ei;
                    }
                }
            }
            if (!ok) atomicOr(&sFailed, 1);
            // every copy issued must land before the block's shared memory is
            // released: wait for the last fill of each stage (bounded)
            for (uint32_t x = ci > kBlkCStages ? ci - kBlkCStages : 0; x < ci; ++x)
                if (!blkWait(&cFull[x % kBlkCStages], (x / kBlkCStages) & 1u, b.spinLimit)) atomicOr(&sFailed, 1);
            for (uint32_t x = ei > kBlkEStages ? ei - kBlkEStages : 0; x < ei; ++x)
                if (!blkWait(&eFull[x % kBlkEStages], (x / kBlkEStages) & 1u, b.spinLimit)) atomicOr(&sFailed, 1);
        }
        __syncwarp();  // lanes 1-31 wait for the producer thread
    } else {
        // consumers: thread ct of kBlkConsumerWarps * 32
        const unsigned ct = tid - 32, lane = tid & 31;
        constexpr unsigned kCons = kBlkConsumerWarps * 32;
        uint32_t ci = 0, ei = 0;
        bool ok = true;
        for (uint32_t k = blockIdx.x; k < b.nRowBlocks; k += gridDim.x) {
            const uint32_t r0 = k * b.rowsPer, rows = min((uint32_t)a.n - r0, b.rowsPer);
            for (uint32_t i = ct; i < rows; i += kCons) sums[i] = 0.0f;
            if (consumersOr(!ok)) break;  // sums zeroed (and the previous block's stored)
            for (uint32_t j = 0; j < b.nParts && ok; ++j) {
                uint32_t w0, w1;
                tileOf(k, j, w0, w1);
                if (w0 == w1) continue;
                const uint32_t cs = ci % kBlkCStages;
                ok = __all_sync(kFull, blkWait(&cFull[cs], (ci / kBlkCStages) & 1u, b.spinLimit));
                if (!ok) break;
                const float* part = cring + cs * kBlkPart;
                for (uint32_t w = w0; w < w1; w += kBlkChunk) {
                    const uint32_t es = ei % kBlkEStages;
                    ok = __all_sync(kFull, blkWait(&eFull[es], (ei / kBlkEStages) & 1u, b.spinLimit));
                    if (!ok) break;
                    const uint32_t words = min(kBlkChunk, w1 - w);
                    for (uint32_t q = ct; q < words; q += kCons) blkAdd(sums, part, ering[es * kBlkChunk + q]);
                    __syncwarp();
                    if (lane == 0) blkArrive(&eEmpty[es]);
                    ++ei;
                }
                if (!ok) break;
                __syncwarp();
                if (lane == 0) blkArrive(&cEmpty[cs]);
                ++ci;
            }
            if (consumersOr(!ok)) break;  // every edge of row block k is in the sums
            for (uint32_t i = ct; i < rows; i += kCons) {
                const uint32_t v = r0 + i;
                if (a.rp[v + 1] - a.rp[v] >= kBlkHub) continue;
                storeJacobi(a, cur, withDelta, v, prValue(a, sums[i], dang), acc);
            }
        }
        if (!ok && lane == 0) atomicOr(&sFailed, 1);
    }
    __syncthreads();
    if (sFailed) {
        if (tid == 0) atomicOr(&a.ctl->error, 1);
        return;
    }
    // rows with kBlkHub or more in-edges: one block each
    __shared__ float hubHi[kBlkThreads / 32], hubLo[kBlkThreads / 32];
    for (uint32_t h = blockIdx.x; h < b.nHubs; h += gridDim.x) {
        const uint32_t v = b.hubs[h];
        Kahan ks;
        for (uint32_t e = a.rp[v] + tid; e < a.rp[v + 1]; e += kBlkThreads) ks.add(__ldg(contrib + ldStream(a.ci + e)));
        FF f;
        f.add(ks.sum);
        f.add(-ks.comp);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            FF other;
            other.hi = __shfl_xor_sync(kFull, f.hi, o);
            other.lo = __shfl_xor_sync(kFull, f.lo, o);
            if (laneId() < (unsigned)o) f.add(other);
        }
        if (laneId() == 0) {
            hubHi[tid >> 5] = f.hi;
            hubLo[tid >> 5] = f.lo;
        }
        __syncthreads();
        if (tid == 0) {
            FF t2;
            for (int w = 0; w < kBlkThreads / 32; ++w) {
                FF x;
                x.hi = hubHi[w];
                x.lo = hubLo[w];
                t2.add(x);
            }
            storeJacobi(a, cur, withDelta, v, prValue(a, t2.hi + t2.lo, dang), acc);
        }
        __syncthreads();
    }
    finishBlock<0>(a, acc);
}

// Double-precision Jacobi pull (warp per vertex): the GPU oracle against
// which FP32 runs are measured at sizes where the CPU reference is slow.
__global__ void prPullF64Kernel(PrArgs a) {
    const GbPrControl* c = a.ctl;
    if (ldvi(&c->stopped)) return;
    const int cur = c->cur;
    const double add = a.base64 + a.damping64 * c->dang64 * a.invN64;
    const bool withDelta = c->withDelta;
    const double* contrib = a.contrib64[cur];
    IterAcc acc;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t v = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < a.n; v += nwarps) {
        double s = 0;
        for (uint32_t j = a.rp[v] + laneId(); j < a.rp[v + 1]; j += 32) s += contrib[a.ci[j]];
        s = warpSum(s);
        if (laneId() == 0) {
            const double val = add + a.damping64 * s;
            a.r64[cur ^ 1][v] = val;
            const uint32_t od = a.outdeg[v];
            a.contrib64[cur ^ 1][v] = od ? val / od : 0.0;
            if (!od) acc.d64 += val;
            if (withDelta) {
                const double d = fabs(val - a.r64[cur][v]);
                acc.dsum += d;
                acc.dmax = fmaxf(acc.dmax, (float)(d / fmax(val, a.invN64)));
            }
        }
    }
    finishBlock<4>(a, acc);
}

}  // namespace
}  // namespace gb

using namespace gb;

gb_pr::~gb_pr() { invalidateGraphs(); }

// Cached graphs hold buffer addresses: drop them whenever a buffer they may
// reference is (re)allocated.
void gb_pr::invalidateGraphs() {
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
    graphs.clear();
}

namespace {

PrArgs makeArgs(gb_pr& h, bool relabeled) {
    PrArgs a{};
    a.rp = relabeled ? h.rowGS.get() : h.rowIn.get();
    a.ci = relabeled ? h.colGS.get() : h.colIn.get();
    a.outdeg = relabeled ? h.outdegGS.get() : h.outdeg.get();
    for (int i = 0; i < 2; ++i) {
        a.r[i] = h.r[i].get();
        a.contrib[i] = h.contrib[i].get();
        a.r64[i] = h.r64[i].get();
        a.contrib64[i] = h.contrib64[i].get();
    }
    a.acc = h.acc.get();
    a.accLo = h.accLo.get();
    a.ctl = h.ctl.get();
    a.partF = h.partF.get();
    a.partD = h.partD.get();
    a.n = (uint32_t)h.n;
    return a;
}

uint32_t gridFor(uint64_t work, uint32_t threads) {
    uint64_t b = (work + threads - 1) / threads;
    uint64_t cap = std::min<uint64_t>(kMaxGrid, (uint64_t)deviceSmCount() * (2048 / threads));
    return (uint32_t)std::max<uint64_t>(1, std::min(b, cap));
}

// Grid of exactly the blocks that can be resident at once (grid-stride
// kernels: a second, partly filled wave would only add a tail).
template <class K>
uint32_t residentGrid(K kernel, uint64_t work, uint32_t threads) {
    static std::map<std::pair<const void*, uint32_t>, int> cache;
    auto key = std::make_pair((const void*)kernel, threads);
    auto it = cache.find(key);
    int perSm;
    if (it == cache.end()) {
        GB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, (int)threads, 0));
        perSm = std::max(perSm, 1);
        cache[key] = perSm;
    } else {
        perSm = it->second;
    }
    uint64_t b = (work + threads - 1) / threads;
    uint64_t cap = std::min<uint64_t>(kMaxGrid, (uint64_t)deviceSmCount() * perSm);
    return (uint32_t)std::max<uint64_t>(1, std::min(b, cap));
}

}  // namespace

// Dynamic shared memory of prBlockedKernel (the staging ring, row sums);
// the opt-in limit is raised once per process.
static size_t blkSmemBytes() {
    static const size_t bytes = [] {
        const size_t b = ((size_t)kBlkCStages * kBlkPart + kBlkRowCap) * sizeof(float) +
                         (size_t)kBlkEStages * kBlkChunk * sizeof(uint4);
        GB_CUDA(cudaFuncSetAttribute(prBlockedKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b));
        return b;
    }();
    return bytes;
}

// Enqueue one iteration of `variant` on the handle's stream (capturable).
static void enqueueIteration(gb_pr& h, int v, const gb_pr_options& o, PrArgs& a, PrArgs& ag) {
    const uint32_t tg = o.tg;
    cudaStream_t s = h.stream.s;
    const uint32_t gN = gridFor(h.n, 256);
    auto pullGrid = [&](int mode) {
        if (mode == 0) return residentGrid(prPullKernel<0, false>, h.n, tg);
        if (mode == 1) return residentGrid(prPullKernel<1, false>, h.n * 32, tg);
        uint64_t tasks = h.nChunks;  // adaptive: warp tasks
        for (int b = 0; b < h.nBins; ++b) tasks += ((uint64_t)(h.binHi[b] - h.binLo[b]) * h.binG[b] + 31) / 32;
        return residentGrid(prPullKernel<2, false>, tasks * 32, tg);
    };
    const bool inplace = v == GB_PR_PULL_GS || (o.inplace && v != GB_PR_PUSH && v != GB_PR_PULL_F64);
    if (v == GB_PR_PUSH) {
        prPushKernel<<<gridFor(h.n, tg), tg, 0, s>>>(a, h.rowOut.get(), h.colOut.get());
        prPushFinalizeKernel<<<gN, 256, 0, s>>>(a);
    } else if (v == GB_PR_PULL_F64) {
        prPullF64Kernel<<<gridFor(h.n * 32, tg), tg, 0, s>>>(a);
    } else if (v == GB_PR_PULL_BLOCKED) {
        BlkArgs b{reinterpret_cast<const uint4*>(h.blkEdges.get()), h.blkOff.get(), h.blkHubs.get(), h.nRowBlocks,
                  h.rowsPer, h.nParts, h.nBlkHubs, 1ull << 22};
        const uint32_t grid = (uint32_t)std::min<uint64_t>({(uint64_t)deviceSmCount(), (uint64_t)kMaxGrid,
                                                            (uint64_t)std::max(h.nRowBlocks, h.nBlkHubs)});
        prBlockedKernel<<<std::max(grid, 1u), kBlkThreads, blkSmemBytes(), s>>>(a, b);
    } else if (!inplace) {
        if (v == GB_PR_PULL_SCALAR) prPullKernel<0, false><<<pullGrid(0), tg, 0, s>>>(a);
        else if (v == GB_PR_PULL_VECTOR) prPullKernel<1, false><<<pullGrid(1), tg, 0, s>>>(a);
        else prPullKernel<2, false><<<pullGrid(2), tg, 0, s>>>(ag);
    } else {
        const bool colored = v == GB_PR_PULL_GS && h.gsColored;
        PrArgs& w = (colored || v == GB_PR_PULL_ADAPTIVE) ? ag : a;
        gsContribKernel<<<gN, 256, 0, s>>>(w);
        if (v == GB_PR_PULL_GS) {
            if (colored) {
                // one in-place sweep per colour set, in set order: the set's
                // split hubs and degree classes in one task-space launch
                for (const auto& L : h.gsSetLayout) {
                    PrArgs ws = w;
                    ws.chunks = h.gsHubChunks.get() + L.chunk0;
                    ws.nChunks = L.chunk1 - L.chunk0;
                    ws.hubFirst = h.gsHubFirst.get();
                    ws.hubDone = h.gsHubDone.get();
                    ws.hubPart = h.gsHubPart.get();
                    ws.chunkBase = L.chunk0;
                    ws.nBins = L.nBins;
                    uint64_t tasks = ws.nChunks;
                    for (int b = 0; b < 8; ++b) {
                        ws.binLo[b] = L.lo[b];
                        ws.binHi[b] = L.hi[b];
                        ws.binG[b] = L.g[b];
                        if (b < L.nBins) tasks += ((uint64_t)(L.hi[b] - L.lo[b]) * L.g[b] + 31) / 32;
                    }
                    prPullKernel<2, true><<<residentGrid(prPullKernel<2, true>, tasks * 32, tg), tg, 0, s>>>(ws);
                }
            } else {
                PrArgs wa = w;
                if (h.gsChunks) {
                    wa.chunks = h.gsHubChunks.get();
                    wa.hubFirst = h.gsHubFirst.get();
                    wa.hubDone = h.gsHubDone.get();
                    wa.hubPart = h.gsHubPart.get();
                    wa.nChunks = h.gsChunks;
                    gsHubKernel<<<gridFor((uint64_t)h.gsChunks * 32, tg), tg, 0, s>>>(wa);
                }
                // The main list runs as kGsNatSlices consecutive launches in
                // list order, so every slice reads the finished values of
                // all earlier ones.  One launch of the whole list puts every
                // vertex of a small graph into a single wave whose reads of
                // one another are a random mix of old and new values; its
                // per-sweep change then understates the remaining error
                // (rmat12, K = 0: top-1000 relative error up to 1.1e-3 when
                // stopped at L1 change 2.5e-7, 30-36 sweeps; in slices the
                // same stop gives about 3e-4 in about 21 sweeps).
                const uint32_t slices = h.gsNatA >= kGsNatSlices * 32u ? kGsNatSlices : 1u;
                for (uint32_t k = 0; k < slices; ++k) {
                    const uint32_t lo = (uint32_t)((uint64_t)h.gsNatA * k / slices);
                    const uint32_t hi = (uint32_t)((uint64_t)h.gsNatA * (k + 1) / slices);
                    wa.list = h.gsNat.get() + lo;
                    gsSweepListKernel<<<gridFor((uint64_t)(hi - lo) * 32, tg), tg, 0, s>>>(wa, hi - lo);
                }
                if (h.gsNatB > 0) {
                    wa.list = h.gsNat.get() + h.gsNatA;
                    gsSweepListKernel<<<gridFor((uint64_t)h.gsNatB * 32, tg), tg, 0, s>>>(wa, h.gsNatB);
                }
            }
        } else if (v == GB_PR_PULL_SCALAR) {
            prPullKernel<0, true><<<pullGrid(0), tg, 0, s>>>(w);
        } else if (v == GB_PR_PULL_VECTOR) {
            prPullKernel<1, true><<<pullGrid(1), tg, 0, s>>>(w);
        } else {
            prPullKernel<2, true><<<pullGrid(2), tg, 0, s>>>(w);
        }
        prSumKernel<<<gN, 256, 0, s>>>(w);
        prScaleKernel<<<gN, 256, 0, s>>>(w);
    }
    GB_LAUNCH_CHECK();
}

gb_pr_result gb_pr::run(int v, const gb_pr_options& o) {
    if (o.tg < 32 || o.tg > 1024 || o.tg % 32)
        throw Error(GB_ERR_ARG, "threadgroup size must be a multiple of 32 in [32, 1024]");
    if (v < GB_PR_PUSH || v > GB_PR_PULL_BLOCKED) throw Error(GB_ERR_ARG, "unknown GPU PageRank variant");
    if (v == GB_PR_PUSH && !hasOut) throw Error(GB_ERR_ARG, "gpu_push needs the out-CSR");
    if (v != GB_PR_PUSH && !hasIn) throw Error(GB_ERR_ARG, "pull variants need the in-CSR");
    if (o.iters < 0) throw Error(GB_ERR_ARG, "iters must be >= 0");
    if (v == GB_PR_PULL_ADAPTIVE) prepareAdaptive(o.small_max, o.large_min);
    if (v == GB_PR_PULL_GS && !gsReady) prepareGS(2);
    if (v == GB_PR_PULL_BLOCKED) {
        prepareBlocked();
        (void)blkSmemBytes();  // raise the shared-memory limit before any capture
    }
    gb_pr_result res{};
    res.last_delta = -1;
    res.last_max_rel = -1;
    gsLastRun = v == GB_PR_PULL_GS && gsColored;
    lastVariant = v;
    if (n == 0) return res;
    const void* before[6] = {r64[0].get(), r64[1].get(), contrib64[0].get(), contrib64[1].get(), acc.get(),
                             accLo.get()};
    if (v == GB_PR_PULL_F64) {
        for (auto& b : r64) b.ensure(n);
        for (auto& b : contrib64) b.ensure(n);
    }
    if (v == GB_PR_PUSH) {
        acc.ensure(n);
        accLo.ensure(n);
    }
    const void* after[6] = {r64[0].get(), r64[1].get(), contrib64[0].get(), contrib64[1].get(), acc.get(),
                            accLo.get()};
    if (std::memcmp(before, after, sizeof before) != 0) invalidateGraphs();
    const bool tolMode = o.tol > 0;
    GbPrControl c{};
    c.cap = o.iters;
    c.stopped = o.iters == 0;
    c.withDelta = tolMode ? 1 : 0;
    c.best = 1e300;
    c.tol = o.tol;
    c.tolRel = o.tol_rel;
    PrArgs a = makeArgs(*this, false);
    a.damping = o.damping;
    a.base = (1.0f - o.damping) / (float)n;
    a.invN = 1.0f / (float)n;
    // The FP64 variant uses the decimal value the float option was written as
    // (0.85f -> 0.85), as the double-precision CPU reference does.
    {
        char buf[32];
        std::snprintf(buf, sizeof buf, "%.7g", (double)o.damping);
        a.damping64 = std::strtod(buf, nullptr);
    }
    a.base64 = (1.0 - a.damping64) / (double)n;
    a.invN64 = 1.0 / (double)n;
    PrArgs ag = a;
    if (v == GB_PR_PULL_ADAPTIVE) {  // hub-first relabeled layout
        ag.rp = rowA.get();
        ag.ci = colA.get();
        ag.outdeg = outdegA.get();
        ag.chunks = hubChunks.get();
        ag.hubFirst = hubFirst.get();
        ag.hubDone = hubDone.get();
        ag.hubPart = hubPart.get();
        ag.nChunks = nChunks;
        ag.nBins = nBins;
        for (int b = 0; b < 8; ++b) {
            ag.binLo[b] = binLo[b];
            ag.binHi[b] = binHi[b];
            ag.binG[b] = binG[b];
        }
    } else if (gsColored && gsReady) {
        ag.rp = rowGS.get();
        ag.ci = colGS.get();
        ag.outdeg = outdegGS.get();
    }
    const bool relabel = (v == GB_PR_PULL_GS && gsColored) || v == GB_PR_PULL_ADAPTIVE;
    GB_CUDA(cudaEventRecord(ev.a, stream.s));
    GB_CUDA(cudaMemcpyAsync(ctl.get(), &c, sizeof c, cudaMemcpyHostToDevice, stream.s));
    if (v == GB_PR_PUSH) {
        GB_CUDA(cudaMemsetAsync(acc.get(), 0, n * 4, stream.s));
        GB_CUDA(cudaMemsetAsync(accLo.get(), 0, n * 4, stream.s));
    }
    {
        PrArgs ai = relabel ? ag : a;
        if (v == GB_PR_PULL_F64) prInit64Kernel<<<gridFor(n, 256), 256, 0, stream.s>>>(ai);
        else prInitKernel<<<gridFor(n, 256), 256, 0, stream.s>>>(ai);
        GB_LAUNCH_CHECK();
    }
    // Iteration batches as CUDA graphs (cached per variant / shape).
    const int batch = tolMode ? kGraphBatch : std::max(1, o.iters);
    auto key = std::make_tuple(v, batch, (int)o.tg, (int)(o.inplace != 0), relabel ? 1 : 0, (int)binSmall,
                               (int)binLarge);
    cudaGraphExec_t exec = nullptr;
    auto it = graphs.find(key);
    if (it != graphs.end()) {
        exec = it->second;
    } else {
        cudaGraph_t g;
        GB_CUDA(cudaStreamBeginCapture(stream.s, cudaStreamCaptureModeThreadLocal));
        try {
            for (int i = 0; i < batch; ++i) enqueueIteration(*this, v, o, a, ag);
        } catch (...) {
            cudaStreamEndCapture(stream.s, &g);
            throw;
        }
        GB_CUDA(cudaStreamEndCapture(stream.s, &g));
        GB_CUDA(cudaGraphInstantiate(&exec, g, 0));
        cudaGraphDestroy(g);
        graphs[key] = exec;
    }
    GbPrControl hc{};
    for (int launched = 0;;) {
        GB_CUDA(cudaGraphLaunch(exec, stream.s));
        launched += batch;
        if (!tolMode) break;
        GB_CUDA(cudaMemcpyAsync(&hc, ctl.get(), sizeof hc, cudaMemcpyDeviceToHost, stream.s));
        GB_CUDA(cudaStreamSynchronize(stream.s));
        if (hc.stopped || launched >= o.iters) break;
    }
    GB_CUDA(cudaEventRecord(ev.b, stream.s));
    GB_CUDA(cudaMemcpyAsync(&hc, ctl.get(), sizeof hc, cudaMemcpyDeviceToHost, stream.s));
    GB_CUDA(cudaStreamSynchronize(stream.s));
    res.gpu_ms = ev.ms();
    if (hc.error) throw Error(GB_ERR_TIMEOUT, "PageRank: a device wait for a staging copy exceeded its limit");
    res.iters = hc.iters;
    res.floor_stop = hc.floorStop;
    if (tolMode) {
        res.last_delta = hc.lastDelta;
        res.last_max_rel = hc.lastMaxRel;
    }
    return res;
}

void gb_pr::ranks(float* out) {
    if (lastVariant < 0) throw Error(GB_ERR_STATE, "ranks() before run()");
    if (lastVariant == GB_PR_PULL_F64) throw Error(GB_ERR_STATE, "last run was FP64: use the double ranks");
    GbPrControl hc{};
    GB_CUDA(cudaMemcpy(&hc, ctl.get(), sizeof hc, cudaMemcpyDeviceToHost));
    const std::vector<uint32_t>* map = lastVariant == GB_PR_PULL_ADAPTIVE ? &permA : gsLastRun ? &gsNewId : nullptr;
    if (!map) {
        GB_CUDA(cudaMemcpy(out, r[hc.cur].get(), n * 4, cudaMemcpyDeviceToHost));
        return;
    }
    std::vector<float> tmp(n);  // relabeled layout: back to the caller's ids
    GB_CUDA(cudaMemcpy(tmp.data(), r[hc.cur].get(), n * 4, cudaMemcpyDeviceToHost));
    const uint32_t* m = map->data();
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < (int64_t)n; ++v) out[v] = tmp[m[v]];
}

void gb_pr::ranks64(double* out) {
    if (lastVariant != GB_PR_PULL_F64) throw Error(GB_ERR_STATE, "no FP64 run to read");
    GbPrControl hc{};
    GB_CUDA(cudaMemcpy(&hc, ctl.get(), sizeof hc, cudaMemcpyDeviceToHost));
    GB_CUDA(cudaMemcpy(out, r64[hc.cur].get(), n * 8, cudaMemcpyDeviceToHost));
}
