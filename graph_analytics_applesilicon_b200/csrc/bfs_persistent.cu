// bfs_persistent.cu -- single-source BFS with every level in one cooperative
// launch (gpu_do_persistent; `hybrid` maps here).
//
// Replaces the reference's per-level command buffer + host wait
// (src/metal/bfs_gpu.mm:83-104, ~0.1-0.2 ms per level) and the CPU half of its
// hybrid (bfs_gpu.mm:307-325): the blocks of a co-resident grid run a level,
// meet at a bounded grid barrier, read the level's counters from device
// memory and all take the same next-level decision (alpha/beta rule, the
// learned selector, or a forced strategy) without a host round trip.
//
// Device state (n vertices, W = ceil(n/32) words):
//   dist u32[n]; visited bitmap u32[W]; frontier bitmaps bm[3] u32[W]
//   (level L reads bm[L%3], writes bm[(L+1)%3], clears bm[(L+2)%3]);
//   frontier queue q[2] = (vertex, adjacency start, degree) u32[n] each;
//   hub list hub[2] = (vertex, start, exclusive offset in the hubs' edge space)
//   for vertices of degree >= hub_min, whose edges are split across blocks;
//   counters ctr[3] (level L writes ctr[L%3], zeroes ctr[(L+1)%3]).
// Top-down claims a vertex with atomicOr on its visited bit (an L2-resident
// word instead of a 32-bit CAS on dist); bottom-up writes only bitmaps.
#include <algorithm>
#include <cstring>

#include "bfs.hpp"
#include "bfs_device.cuh"

namespace gb {
namespace {

constexpr unsigned long long kHubShift = 40;
constexpr unsigned long long kHubMask = (1ull << kHubShift) - 1;
constexpr uint32_t kTraceCap = 1u << 16;
constexpr uint64_t kEnqueueEdges = 1ull << 18;  // top-down levels with this many edges build no queue

enum { S_LEVEL, S_BOTTOMUP, S_SCOUT, S_TOCHECK, S_UNEXPLORED, S_REACHED, S_QVALID, S_LAST, S_COUNT };

struct PArgs {
    const uint32_t* __restrict__ row_ptr;
    const uint32_t* __restrict__ col_idx;
    uint32_t* dist;
    uint32_t* qv[2];
    uint32_t* qs[2];
    uint32_t* qd[2];
    uint32_t* hv[2];
    uint32_t* hs[2];
    unsigned long long* ho[2];
    uint32_t* bm[3];
    uint32_t* visited;
    const uint32_t* iso;  // bit per vertex of degree 0, or null
    GbPCounters* ctr;
    unsigned* ctl;  // [0] barrier word, [1] error flag, [2] levels run
    gb_level* trace;
    const float* sel;
    double* state;
    uint64_t n, m;
    uint32_t words, source, hubMin, traceCap;
    double alpha, beta;
    float selMargin;  // learned selector: log2 margin for leaving the rule's direction
    int selector, force;
    unsigned long long spinLimit;
    uint32_t startLevel, maxLevels;
};

__device__ __forceinline__ unsigned long long ldv(const unsigned long long* p) {
    return *reinterpret_cast<const volatile unsigned long long*>(p);
}
__device__ __forceinline__ unsigned ldv(const unsigned* p) { return *reinterpret_cast<const volatile unsigned*>(p); }

// Per-thread accumulators of one level, flushed once per block.
struct Acc {
    unsigned long long found = 0, deg = 0, exam = 0;
};

// Append a claimed u (all 32 lanes call together) to the next frontier:
// depth, bitmap bit and, when enq, a queue entry (degree < hub_min) or hub
// entry.  Without enq the next level, if top-down, rebuilds its queue from
// the bitmap (one block-aggregated append per block and round instead of one
// atomic per warp here).
__device__ __forceinline__ void appendClaimed(const PArgs& a, bool claimed, uint32_t u, uint32_t st, uint32_t en,
                                              uint32_t level, GbPCounters* cur, uint32_t* bmNext, uint32_t nq,
                                              Acc& acc, bool enq) {
    const uint32_t w = u >> 5, bit = 1u << (u & 31);
    if (!__any_sync(kFull, claimed)) return;
    const uint32_t d = claimed ? en - st : 0u;
    if (claimed) {
        a.dist[u] = level + 1;
        atomicOr(&bmNext[w], bit);
        acc.found++;
        acc.deg += d;
    }
    if (!enq) return;
    const bool hub = claimed && d >= a.hubMin;
    const bool q = claimed && !hub;
    if (__any_sync(kFull, q)) {
        uint32_t pos = warpAppend(q, &cur->qtail);
        if (q) {
            a.qv[nq][pos] = u;
            a.qs[nq][pos] = st;
            a.qd[nq][pos] = d;
        }
    }
    if (hub) {
        unsigned long long old = atomicAdd(&cur->hubPack, (1ull << kHubShift) | d);
        uint32_t i = (uint32_t)(old >> kHubShift);
        a.hv[nq][i] = u;
        a.hs[nq][i] = st;
        a.ho[nq][i] = old & kHubMask;
    }
}

// Claim K vertices per lane for level+1 and append the claimed ones (all 32
// lanes call together).  The K claims are issued stage by stage -- visited
// words (large levels read them first to spare atomics on visited
// neighbours), row bounds and atomicOr claims -- so their round trips overlap
// rather than run one claim after another.
template <int K>
__device__ __forceinline__ void discoverN(const PArgs& a, const bool* has, const uint32_t* u, uint32_t level,
                                          GbPCounters* cur, uint32_t* bmNext, uint32_t nq, Acc& acc, bool precheck,
                                          bool enq) {
    bool cand[K];
    uint32_t st[K], en[K], old[K];
#pragma unroll
    for (int k = 0; k < K; ++k) cand[k] = has[k];
    if (precheck) {
        uint32_t vw[K];
#pragma unroll
        for (int k = 0; k < K; ++k) vw[k] = cand[k] ? a.visited[u[k] >> 5] : 0u;
#pragma unroll
        for (int k = 0; k < K; ++k) cand[k] = cand[k] && !(vw[k] & (1u << (u[k] & 31)));
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
        st[k] = cand[k] ? a.row_ptr[u[k]] : 0u;
        en[k] = cand[k] ? a.row_ptr[u[k] + 1] : 0u;
        old[k] = cand[k] ? atomicOr(&a.visited[u[k] >> 5], 1u << (u[k] & 31)) : ~0u;
    }
#pragma unroll
    for (int k = 0; k < K; ++k)
        appendClaimed(a, !(old[k] & (1u << (u[k] & 31))), u[k], st[k], en[k], level, cur, bmNext, nq, acc, enq);
}

template <int NT>
struct Smem {
    uint32_t scan[NT / 32 + 1];
    uint32_t off[NT];
    uint32_t st[NT];
    float sel[kSelParams];
    unsigned long long acc[3];
    unsigned long long cnt[4];  // level counters after a barrier: found, nextEdges, qtail, hubPack
    uint32_t range[2];
    unsigned item;
    int strat;
    uint32_t base;
    int ok;
};

// Grid barrier after which every thread of the block sees counters *c in
// sm.cnt: thread 0 reads them once for its block, so a level costs one L2
// request per block on the counters' line rather than one per warp.
template <int NT>
__device__ __forceinline__ bool barrierWithCounters(const PArgs& a, Smem<NT>& sm, const GbPCounters* c) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const bool ok = gridArriveWait(&a.ctl[0], &a.ctl[1], a.spinLimit, gridDim.x);
        sm.ok = ok;
        if (ok) {
            sm.cnt[0] = ldv(&c->found);
            sm.cnt[1] = ldv(&c->nextEdges);
            sm.cnt[2] = ldv(&c->qtail);
            sm.cnt[3] = ldv(&c->hubPack);
        }
    }
    __syncthreads();
    return sm.ok != 0;
}

// Edge-balanced expansion of one tile of NT queue entries: the entries'
// degrees are scanned in shared memory and every thread takes EPT edges per
// round (thread t: edges base + k*NT + t), owner found by a shared-memory
// binary search over the staged offsets.  The block expands part `part` of
// `parts` equal slices of the tile's edges (a tile of high-degree entries is
// split over several blocks; each scans the tile's degrees itself).
template <int NT, int EPT>
__device__ void tdTile(const PArgs& a, Smem<NT>& sm, uint32_t item, uint32_t S, uint32_t qc, uint32_t level,
                       GbPCounters* cur, uint32_t* bmNext, Acc& acc, bool pre, bool enq, uint32_t part,
                       uint32_t parts) {
    const uint32_t idx = item * NT + threadIdx.x;
    uint32_t st = 0, d = 0;
    if (idx < S) {
        st = a.qs[qc][idx];
        d = a.qd[qc][idx];
    }
    uint32_t tot;
    const uint32_t off = blockScan<NT>(d, &tot, sm.scan);
    sm.off[threadIdx.x] = off;
    sm.st[threadIdx.x] = st;
    __syncthreads();
    const uint32_t cnt = min((uint32_t)NT, S - item * NT);
    const uint32_t lo = (uint32_t)((uint64_t)tot * part / parts), hi = (uint32_t)((uint64_t)tot * (part + 1) / parts);
    for (uint32_t base = lo; base < hi; base += NT * EPT) {
        uint32_t u[EPT];
        bool has[EPT];
#pragma unroll
        for (int k = 0; k < EPT; ++k) {
            const uint32_t e = base + k * NT + threadIdx.x;
            has[k] = e < hi;
            u[k] = 0;
            if (has[k]) {
                const uint32_t o = ownerOf(sm.off, 0u, cnt - 1, e);
                u[k] = a.col_idx[sm.st[o] + (e - sm.off[o])];
            }
        }
        discoverN<EPT>(a, has, u, level, cur, bmNext, qc ^ 1u, acc, pre, enq);
    }
    __syncthreads();
}

// Top-down over the queue in groups of G lanes per entry (G = 4..32, a power
// of two of at least twice the level's mean degree; G = 32 is warp per
// vertex, the degree-binned form): a warp takes 32/G consecutive entries, and
// each group strides its vertex's adjacency list.  Low-degree frontiers (road
// graphs, degree ~4, G = 8) thus use a quarter of the warps, so a quarter of
// the queue appends, and most vertices still finish in one round.
__device__ __forceinline__ void tdGroups(const PArgs& a, uint32_t S, unsigned G, uint32_t qc, uint32_t level,
                                         GbPCounters* cur, uint32_t* bmNext, Acc& acc, bool pre, bool enq) {
    const unsigned lane = laneId(), per = 32u / G;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t base = warp * per; base < S; base += nwarps * per) {  // warp-uniform
        const uint64_t idx = base + lane / G;
        const bool has = idx < S;
        const uint32_t st = has ? a.qs[qc][idx] : 0u, d = has ? a.qd[qc][idx] : 0u;
        const uint32_t maxd = __reduce_max_sync(kFull, d);
        for (uint32_t e0 = 0; e0 < maxd; e0 += 2 * G) {  // two rounds per step: their claims overlap
            const uint32_t e = e0 + (lane & (G - 1));
            const bool he[2] = {e < d, e + G < d};
            const uint32_t u[2] = {he[0] ? a.col_idx[st + e] : 0u, he[1] ? a.col_idx[st + e + G] : 0u};
            discoverN<2>(a, he, u, level, cur, bmNext, qc ^ 1u, acc, pre, enq);
        }
    }
}

// One chunk of the hubs' concatenated edge space, split over the block:
// kHubEdges edges per thread in one round (kHubEdges NT edges per chunk), so
// a thread's column reads, visited reads and claims are in flight together
// and a large hub level takes few dependent rounds per block.
constexpr int kHubEdges = 4;

template <int NT>
__device__ void tdHubChunk(const PArgs& a, Smem<NT>& sm, uint64_t e0, uint64_t e1, uint32_t H, uint32_t qc,
                           uint32_t level, GbPCounters* cur, uint32_t* bmNext, Acc& acc, bool pre, bool enq) {
    const unsigned long long* ho = a.ho[qc];
    if (threadIdx.x < 64) {  // the chunk's first and last owners: warp 0 and warp 1 side by side
        const unsigned long long key = threadIdx.x < 32 ? e0 : e1 - 1;
        const uint32_t o = warpOwnerOf(ho, 0u, H - 1, key);
        if ((threadIdx.x & 31u) == 0) sm.range[threadIdx.x >> 5] = o;
    }
    __syncthreads();
    const uint32_t lo = sm.range[0], hi = sm.range[1];
    for (uint64_t base = e0; base < e1; base += kHubEdges * NT) {
        uint32_t u[kHubEdges];
        bool has[kHubEdges];
#pragma unroll
        for (int k = 0; k < kHubEdges; ++k) {
            const uint64_t e = base + k * NT + threadIdx.x;
            has[k] = e < e1;
            u[k] = 0;
            if (has[k]) {
                const uint32_t o = ownerOf(ho, lo, hi, (unsigned long long)e);
                u[k] = a.col_idx[a.hs[qc][o] + (uint32_t)(e - ho[o])];
            }
        }
        discoverN<kHubEdges>(a, has, u, level, cur, bmNext, qc ^ 1u, acc, pre, enq);
    }
    __syncthreads();
}

// Bottom-up: warp per visited-bitmap word; each unvisited lane scans its list
// for the first neighbour in the frontier bitmap (early exit).  The found
// lanes form the next frontier word (__ballot_sync); the owning warp writes
// it and the visited word with plain stores.
// The rest of one vertex's bottom-up scan after its first entry missed: the
// first parent in the frontier, scanning in list order from i; aligned groups
// of 4 entries are loaded at once and their 4 frontier words fetched
// together, so a step costs two dependent loads for 4 entries.  Returns one
// past the first hit, or e when there is none (found tells which).
__device__ __forceinline__ uint32_t buScanFrom(const PArgs& a, const uint32_t* front, uint32_t i, uint32_t e,
                                               bool& found) {
    for (; i < e && (i & 3u); ++i) {
        const uint32_t u = a.col_idx[i];
        if ((front[u >> 5] >> (u & 31)) & 1u) {
            found = true;
            return i + 1;
        }
    }
    for (; i + 4 <= e; i += 4) {
        const uint4 q = *reinterpret_cast<const uint4*>(a.col_idx + i);
        const uint32_t f0 = front[q.x >> 5], f1 = front[q.y >> 5], f2 = front[q.z >> 5], f3 = front[q.w >> 5];
        const unsigned hits = ((f0 >> (q.x & 31)) & 1u) | (((f1 >> (q.y & 31)) & 1u) << 1) |
                              (((f2 >> (q.z & 31)) & 1u) << 2) | (((f3 >> (q.w & 31)) & 1u) << 3);
        if (hits) {
            found = true;
            return i + __ffs(hits);
        }
    }
    for (; i < e; ++i) {
        const uint32_t u = a.col_idx[i];
        if ((front[u >> 5] >> (u & 31)) & 1u) {
            found = true;
            return i + 1;
        }
    }
    return e;
}

// Bottom-up level: each unvisited vertex looks for its first parent in the
// frontier bitmap.  A warp takes kBuWords bitmap words (32 vertices each, a
// lane per vertex) per round and issues their loads stage by stage -- visited
// words, then row bounds, then first entries, then frontier bits -- so the
// four dependent loads of the words overlap instead of running one word
// after another; a vertex whose first entry is not a parent (rare once lists
// are hub-first) continues with buScanFrom.
#ifndef GB_BU_WORDS
#define GB_BU_WORDS 4
#endif
constexpr int kBuWords = GB_BU_WORDS;

__device__ void buLevel(const PArgs& a, uint32_t level, Acc& acc) {
    const uint32_t* front = a.bm[level % 3];
    uint32_t* next = a.bm[(level + 1) % 3];
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const unsigned lane = laneId();
    for (uint64_t w0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w0 < a.words;
         w0 += nwarps * kBuWords) {
        uint32_t vw[kBuWords], b[kBuWords], e[kBuWords], u[kBuWords];
        bool need[kBuWords], found[kBuWords];
#pragma unroll
        for (int k = 0; k < kBuWords; ++k) {
            const uint64_t w = w0 + (uint64_t)k * nwarps;
            vw[k] = w < a.words ? a.visited[w] : kFull;
            need[k] = !((vw[k] >> lane) & 1u);
            found[k] = false;
        }
#pragma unroll
        for (int k = 0; k < kBuWords; ++k) {
            const uint32_t v = (uint32_t)((w0 + (uint64_t)k * nwarps) * 32 + lane);
            b[k] = need[k] ? a.row_ptr[v] : 0u;
            e[k] = need[k] ? a.row_ptr[v + 1] : 0u;
        }
#pragma unroll
        for (int k = 0; k < kBuWords; ++k) u[k] = b[k] < e[k] ? a.col_idx[b[k]] : 0u;
#pragma unroll
        for (int k = 0; k < kBuWords; ++k) {
            if (b[k] < e[k] && ((front[u[k] >> 5] >> (u[k] & 31)) & 1u)) {
                found[k] = true;
                acc.exam += 1;
            }
        }
#pragma unroll
        for (int k = 0; k < kBuWords; ++k) {
            if (need[k] && !found[k]) acc.exam += (b[k] < e[k] ? buScanFrom(a, front, b[k] + 1, e[k], found[k]) : e[k]) - b[k];
            const unsigned F = __ballot_sync(kFull, found[k]);
            const uint64_t w = w0 + (uint64_t)k * nwarps;
            if (found[k]) {
                a.dist[w * 32 + lane] = level + 1;
                acc.deg += e[k] - b[k];
                acc.found++;
            }
            if (lane == 0 && F) {
                next[w] = F;
                a.visited[w] = vw[k] | F;
            }
        }
    }
}

// Frontier bitmap -> queue + hub list (only after a bottom-up level, when the
// next level runs top-down).  Per block-round of NT words: per-thread counts,
// a block scan, one atomic for the block's queue range.
template <int NT>
__device__ void bitmapToQueue(const PArgs& a, Smem<NT>& sm, uint32_t level, GbPCounters* prev) {
    const uint32_t* bm = a.bm[level % 3];
    const uint32_t qc = level & 1u;
    for (uint64_t t0 = (uint64_t)blockIdx.x * NT; t0 < a.words; t0 += (uint64_t)gridDim.x * NT) {
        const uint64_t w = t0 + threadIdx.x;
        const uint32_t word = w < a.words ? bm[w] : 0u;
        uint32_t c = 0;
        for (uint32_t x = word; x; x &= x - 1) {
            const uint32_t v = (uint32_t)(w * 32 + __ffs(x) - 1);
            const uint32_t st = a.row_ptr[v], d = a.row_ptr[v + 1] - st;
            if (d >= a.hubMin) {
                unsigned long long old = atomicAdd(&prev->hubPack, (1ull << kHubShift) | d);
                uint32_t i = (uint32_t)(old >> kHubShift);
                a.hv[qc][i] = v;
                a.hs[qc][i] = st;
                a.ho[qc][i] = old & kHubMask;
            } else {
                ++c;
            }
        }
        uint32_t tot;
        uint32_t pos = blockScan<NT>(c, &tot, sm.scan);
        if (threadIdx.x == 0) sm.base = tot ? atomicAdd(&prev->qtail, tot) : 0u;
        __syncthreads();
        pos += sm.base;
        for (uint32_t x = word; x; x &= x - 1) {
            const uint32_t v = (uint32_t)(w * 32 + __ffs(x) - 1);
            const uint32_t st = a.row_ptr[v], d = a.row_ptr[v + 1] - st;
            if (d < a.hubMin) {
                a.qv[qc][pos] = v;
                a.qs[qc][pos] = st;
                a.qd[qc][pos] = d;
                ++pos;
            }
        }
        __syncthreads();
    }
}

template <int NT>
__global__ void __launch_bounds__(NT, 1024 / NT) persistentBfsKernel(PArgs a) {
    __shared__ Smem<NT> sm;
    const unsigned tid = threadIdx.x;
    const uint64_t gtid = (uint64_t)blockIdx.x * NT + tid, gthreads = (uint64_t)gridDim.x * NT;
    unsigned* bar = &a.ctl[0];
    unsigned* err = &a.ctl[1];
    const bool learned = a.selector == GB_SELECT_LEARNED && a.sel != nullptr;
    // the selector's parameters arrive in shared memory while the prologue
    // runs; the wait sits before the prologue's grid barrier (whose block
    // barrier makes them visible to every warp)
    if (learned) selectorStageAsync(sm.sel, a.sel, tid, NT);

    uint32_t level;
    bool bottomUp, qValid;
    uint64_t scout, toCheck, unexplored, reached;
    int lastStrat;
    if (a.startLevel == 0) {
        // One pass writes the initial state with the source already placed
        // (depth 0, visited, frontier bit), so a single grid barrier ends the
        // prologue.  bm[2] needs no clearing: level 0 clears it.  The depth
        // array was set to infinity by a memset before the launch (the copy
        // engine's fill is faster than the kernel's stores).
        const uint32_t src = a.source;
        const uint32_t st = a.row_ptr[src], d = a.row_ptr[src + 1] - st;
        if (gtid == 0) a.dist[src] = 0;  // the rest is already infinity (memset before the launch)
        for (uint64_t w = gtid; w < a.words; w += gthreads) {
            uint32_t pad = 0;
            if (w == a.words - 1 && (a.n & 31)) pad = ~((1u << (a.n & 31)) - 1u);  // bits past n read as visited
            const uint32_t srcBit = w == (src >> 5) ? 1u << (src & 31) : 0u;
            // vertices of degree 0 start as visited: no edge reaches them (their
            // depth stays infinity from the memset), and a bottom-up round then
            // skips a bitmap word as soon as its other vertices are reached
            a.visited[w] = pad | srcBit | (a.iso ? a.iso[w] : 0u);
            a.bm[0][w] = srcBit;
            a.bm[1][w] = 0;
        }
        if (gtid == 0) {
            for (int s = 0; s < 3; ++s) a.ctr[s] = GbPCounters{};
            GbPCounters& c = a.ctr[2];
            c.found = 1;
            c.nextEdges = d;
            if (d >= a.hubMin) {
                a.hv[0][0] = src;
                a.hs[0][0] = st;
                a.ho[0][0] = 0;
                c.hubPack = (1ull << kHubShift) | d;
            } else {
                a.qv[0][0] = src;
                a.qs[0][0] = st;
                a.qd[0][0] = d;
                c.qtail = 1;
            }
        }
        if (learned) selectorStageWait();
        if (!gridBarrier(bar, err, a.spinLimit)) return;
        level = 0;
        bottomUp = false;
        qValid = true;
        scout = d;
        toCheck = a.m;
        unexplored = a.m - d;
        reached = 1;
        lastStrat = -1;
    } else {
        level = (uint32_t)a.state[S_LEVEL];
        bottomUp = a.state[S_BOTTOMUP] != 0;
        scout = (uint64_t)a.state[S_SCOUT];
        toCheck = (uint64_t)a.state[S_TOCHECK];
        unexplored = (uint64_t)a.state[S_UNEXPLORED];
        reached = (uint64_t)a.state[S_REACHED];
        qValid = a.state[S_QVALID] != 0;
        lastStrat = (int)a.state[S_LAST];
        if (learned) selectorStageWait();
        if (!gridBarrier(bar, err, a.spinLimit)) return;
    }
    const uint32_t endLevel = a.maxLevels ? a.startLevel + a.maxLevels : 0xFFFFFFFFu;
    uint64_t tPrev = globaltimer();
    int selLast = -1;  // last evaluated learned decision and the frontier it was made for
    bool selLastBU = false;
    float selLastF = 0.0f, selLastE = 0.0f;
    // The previous level's counters, read once after each barrier and carried
    // into the next level in registers.
    uint64_t nextSize, nextEdgesC, nextQ;
    unsigned long long nextHub;
    {
        const GbPCounters* p0 = &a.ctr[(level + 2) % 3];
        nextSize = ldv(&p0->found);
        nextEdgesC = ldv(&p0->nextEdges);
        nextQ = ldv(&p0->qtail);
        nextHub = ldv(&p0->hubPack);
    }

    for (;;) {
        GbPCounters* prev = &a.ctr[(level + 2) % 3];
        GbPCounters* cur = &a.ctr[level % 3];
        const uint64_t size = nextSize, fedges = nextEdgesC;
        if (size == 0 || level >= endLevel) break;

        // alpha/beta rule (src/cpu/bfs_cpu.cpp:247-279): always evaluated, it
        // is the fallback and the judge of the learned choice.
        if (!bottomUp && (double)scout > (double)toCheck / a.alpha) bottomUp = true;
        if (!bottomUp) toCheck -= min(toCheck, scout);
        const int ruleStrat = bottomUp ? GB_STRAT_BU : GB_STRAT_TD_EPT2;
        int strat = a.force >= 0 ? a.force : ruleStrat;
        // Warp 0 evaluates the learned selector while the other warps do the
        // level's bookkeeping; one block barrier covers both.  A level whose
        // frontier differs from the last evaluated one by less than 0.25 in
        // log2 of both its vertex and edge counts, in the same rule
        // direction, reuses that decision (every block sees the same
        // counters, so all blocks reuse alike): long runs of similar levels
        // (a road graph's 1,800) then skip the evaluation.
        // A frontier of at most 32 vertices runs the rule's top-down (its hubs
        // are split by edges): every strategy costs about the same there, so
        // the selector's evaluation would only add to the level.  The MLP is
        // evaluated only on levels the rule runs top-down (it picks the
        // top-down strategy and may go bottom-up early, within the trust
        // region); a bottom-up phase and its end follow the rule, where the
        // MLP never departed from it on the benchmark graphs and its
        // evaluation cost about 1 us per level.
        bool useSel = a.force < 0 && learned && !bottomUp && size > 32;
        if (useSel) {
            const float lf = log2f(1.0f + (float)size), le = log2f(1.0f + (float)fedges);
            if (selLast >= 0 && bottomUp == selLastBU && fabsf(lf - selLastF) < 0.25f && fabsf(le - selLastE) < 0.25f) {
                strat = selLast;
                useSel = false;
            } else {
                selLastF = lf;
                selLastE = le;
                selLastBU = bottomUp;
            }
        }
        if (useSel && tid < 32) {
            float f[kSelFeatures];
            selectorFeatures((double)size, (double)fedges, (double)unexplored, (double)(a.n - reached), (double)a.n,
                             (double)a.m, (double)level, f);
            // trust region: a top-down level may go bottom-up only when its
            // edges are within 4x of the rule's threshold (toCheck / alpha);
            // far below it bottom-up would scan every unvisited vertex for a
            // small frontier
            const bool mayGoBU = (double)scout * 4.0 > (double)toCheck / a.alpha;
            int s = selectorChoose(sm.sel, f, tid, bottomUp, a.selMargin, mayGoBU);
            if (tid == 0) sm.strat = s;
        }
        if (tid == 0) sm.acc[0] = sm.acc[1] = sm.acc[2] = 0;
        if (gtid == 0) {
            if (a.trace && level > 0 && level - 1 < a.traceCap && lastStrat == GB_STRAT_BU)
                a.trace[level - 1].edges = ldv(&prev->examined);
            a.ctr[(level + 1) % 3] = GbPCounters{};
        }
        uint32_t* clearBm = a.bm[(level + 2) % 3];
        for (uint64_t w = gtid; w < a.words; w += gthreads) clearBm[w] = 0;
        __syncthreads();
        if (useSel) {
            if (sm.strat >= 0) strat = sm.strat;
            selLast = sm.strat;
        }
        if (gtid == 0 && a.trace && level < a.traceCap) {
            gb_level r;
            r.level = level;
            r.direction = strat == GB_STRAT_BU ? 'B' : 'T';
            r.device = 'G';
            r.strategy = (uint8_t)strat;
            r.pad = (uint8_t)ruleStrat;
            r.frontier = size;
            r.edges = fedges;
            r.time_ms = 0;
            a.trace[level] = r;
        }

        Acc acc;
        if (strat == GB_STRAT_BU) {
            buLevel(a, level, acc);
        } else {
            uint32_t S = (uint32_t)nextQ;
            unsigned long long hp = nextHub;
            if (!qValid) {
                bitmapToQueue<NT>(a, sm, level, prev);
                if (!barrierWithCounters<NT>(a, sm, prev)) return;
                S = (uint32_t)sm.cnt[2];
                hp = sm.cnt[3];
            }
            const uint32_t qc = level & 1u;
            const uint32_t H = (uint32_t)(hp >> kHubShift);
            const uint64_t HE = hp & kHubMask;
            // a level with many edges to expand skips the queue appends: its
            // successor is most often bottom-up (no queue), and a top-down one
            // rebuilds the queue from the bitmap
            const bool enq = fedges < kEnqueueEdges;
            // warp per vertex: a static warp-strided loop over the queue (no
            // tickets, no block barriers); edge-balanced tiles: block tickets
            const bool warpMode = strat == GB_STRAT_TD_WARP;
            if (warpMode) {
                const uint64_t qEdges = fedges > HE ? fedges - HE : 0;  // the queue entries' edges
                // group of at least twice the mean degree: most vertices take one round
                const uint64_t want = S ? 2 * ((qEdges + S - 1) / S) : 1;
                const unsigned G = want <= 4 ? 4u : want <= 8 ? 8u : want <= 16 ? 16u : 32u;
                tdGroups(a, S, G, qc, level, cur, a.bm[(level + 1) % 3], acc, fedges >= 65536, enq);
            }
            const uint32_t nt = warpMode ? 0u : (S + NT - 1) / NT;
            // fewer tiles than half the blocks (a small queue, often of
            // high-degree entries): every tile is split by edge range into
            // parts of at least 8 NT edges, so its edges spread over the grid
            // instead of running on nt blocks while the rest wait
            uint32_t parts = 1;
            if (nt && nt * 2 <= gridDim.x) {
                const uint64_t perPart = (fedges > HE ? fedges - HE : 0) / nt / (8ull * NT);
                const uint64_t cap = gridDim.x / nt;
                parts = perPart < 1 ? 1u : (uint32_t)(perPart < cap ? perPart : cap);
            }
            const uint32_t nti = nt * parts;
            const uint64_t HC = (uint64_t)NT * kHubEdges;
            const bool pre = fedges >= 65536;
            const uint32_t nh = (uint32_t)((HE + HC - 1) / HC);
            uint32_t* bmNext = a.bm[(level + 1) % 3];
            // block b takes item b first; further items come from a ticket
            // (none when the first items cover the level), which thread 0
            // requests while the block still works on the current item
            const bool oneRound = nti + nh <= gridDim.x;
            uint32_t nextItem = blockIdx.x;
            for (;;) {
                if (tid == 0) {
                    sm.item = nextItem;
                    nextItem = (oneRound || nextItem >= nti + nh) ? ~0u : gridDim.x + atomicAdd(&cur->work, 1u);
                }
                __syncthreads();
                const uint32_t item = sm.item;
                __syncthreads();
                if (item >= nti + nh) break;
                if (item < nti) {
                    const uint32_t tile = item / parts, part = item - tile * parts;
                    switch (strat) {
                        case GB_STRAT_TD_EPT1:
                            tdTile<NT, 1>(a, sm, tile, S, qc, level, cur, bmNext, acc, pre, enq, part, parts);
                            break;
                        case GB_STRAT_TD_EPT4:
                            tdTile<NT, 4>(a, sm, tile, S, qc, level, cur, bmNext, acc, pre, enq, part, parts);
                            break;
                        default: tdTile<NT, 2>(a, sm, tile, S, qc, level, cur, bmNext, acc, pre, enq, part, parts); break;
                    }
                } else {
                    const uint64_t e0 = (uint64_t)(item - nti) * HC;
                    tdHubChunk<NT>(a, sm, e0, min(e0 + HC, HE), H, qc, level, cur, bmNext, acc, pre, enq);
                }
            }
        }
        // one atomic per block and counter
        unsigned long long f = warpSum(acc.found), dg = warpSum(acc.deg), ex = warpSum(acc.exam);
        if (laneId() == 0) {
            if (f) atomicAdd(&sm.acc[0], f);
            if (dg) atomicAdd(&sm.acc[1], dg);
            if (ex) atomicAdd(&sm.acc[2], ex);
        }
        __syncthreads();
        if (tid == 0) {
            if (sm.acc[0]) atomicAdd(&cur->found, sm.acc[0]);
            if (sm.acc[1]) atomicAdd(&cur->nextEdges, sm.acc[1]);
            if (sm.acc[2]) atomicAdd(&cur->examined, sm.acc[2]);
        }
        if (!barrierWithCounters<NT>(a, sm, cur)) return;
        if (gtid == 0) {
            const uint64_t t = globaltimer();
            if (a.trace && level < a.traceCap) a.trace[level].time_ms = (double)(t - tPrev) * 1e-6;
            tPrev = t;
        }
        const uint64_t found = sm.cnt[0], nextE = sm.cnt[1];
        nextSize = found;
        nextEdgesC = nextE;
        nextQ = sm.cnt[2];
        nextHub = sm.cnt[3];
        reached += found;
        unexplored -= min(unexplored, nextE);
        if (bottomUp) {
            if (!(found >= size || (double)found > (double)a.n / a.beta)) {
                bottomUp = false;
                scout = 1;
            }
        } else {
            scout = nextE;
        }
        qValid = strat != GB_STRAT_BU && fedges < kEnqueueEdges;
        lastStrat = strat;
        ++level;
    }
    if (gtid == 0) {
        if (a.trace && level > 0 && level - 1 < a.traceCap && lastStrat == GB_STRAT_BU)
            a.trace[level - 1].edges = ldv(&a.ctr[(level + 2) % 3].examined);
        a.ctl[2] = level;
        a.state[S_LEVEL] = level;
        a.state[S_BOTTOMUP] = bottomUp;
        a.state[S_SCOUT] = (double)scout;
        a.state[S_TOCHECK] = (double)toCheck;
        a.state[S_UNEXPLORED] = (double)unexplored;
        a.state[S_REACHED] = (double)reached;
        a.state[S_QVALID] = qValid;
        a.state[S_LAST] = lastStrat;
    }
}

// Bit v of word v / 32: vertex v has no adjacency entries (row_ptr[v] ==
// row_ptr[v + 1]); bits past n are 0.
__global__ void isolatedBitmapKernel(const uint32_t* __restrict__ row_ptr, uint64_t n, uint32_t words,
                                     uint32_t* out) {
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < words;
         w += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t bits = 0;
        const uint64_t v0 = w * 32;
        const uint32_t cnt = (uint32_t)(n - v0 < 32 ? n - v0 : 32);
        uint32_t prev = row_ptr[v0];
        for (uint32_t i = 0; i < cnt; ++i) {
            const uint32_t next = row_ptr[v0 + i + 1];
            if (next == prev) bits |= 1u << i;
            prev = next;
        }
        out[w] = bits;
    }
}

template <int NT>
void launchPersistent(PArgs& a, int grid, cudaStream_t st) {
    void* args[] = {&a};
    GB_CUDA(cudaLaunchCooperativeKernel((void*)persistentBfsKernel<NT>, dim3(grid), dim3(NT), args, 0, st));
}

PArgs makeArgs(gb_bfs& h, const gb_bfs_options& o, uint32_t src) {
    PArgs a{};
    a.row_ptr = h.rowPtr.get();
    a.col_idx = h.colIdx.get();
    a.dist = h.dist.get();
    for (int i = 0; i < 2; ++i) {
        a.qv[i] = h.pq[i][0].get();
        a.qs[i] = h.pq[i][1].get();
        a.qd[i] = h.pq[i][2].get();
        a.hv[i] = h.phub[i][0].get();
        a.hs[i] = h.phub[i][1].get();
        a.ho[i] = h.phubOff[i].get();
    }
    for (int i = 0; i < 3; ++i) a.bm[i] = h.pbm[i].get();
    a.visited = h.pvisited.get();
    a.iso = h.pIso.get();
    a.ctr = h.pctr.get();
    a.ctl = h.pctl.get();
    a.trace = h.ptrace.get();
    a.traceCap = kTraceCap;
    a.sel = h.selLoaded[0] ? h.selParams[0].get() : nullptr;
    a.state = h.pstate.get();
    a.n = h.n;
    a.m = h.m;
    a.words = (uint32_t)((h.n + 31) / 32);
    a.source = src;
    a.hubMin = std::max<uint32_t>(o.hub_min, 32);
    a.alpha = o.alpha;
    a.selMargin = o.sel_margin;
    a.beta = o.beta;
    a.selector = (int)o.selector;
    a.force = o.force_strategy;
    a.spinLimit = o.spin_limit ? o.spin_limit : (1ull << 24);
    a.startLevel = 0;
    a.maxLevels = 0;
    return a;
}

void launchFor(gb_bfs& h, PArgs& a, int grid = 0, cudaStream_t st = nullptr) {
    if (!grid) grid = h.pGrid;
    if (!st) st = h.stream.s;
    if (h.pBlock == 256) launchPersistent<256>(a, grid, st);
    else launchPersistent<512>(a, grid, st);
}

// The state of in-flight slot `slot` (> 0) in place of slot 0's.
void useSlot(gb_bfs& h, PArgs& a, int slot) {
    gb_bfs::PSlot& p = h.pSlot[slot - 1];
    for (int i = 0; i < 2; ++i) {
        a.qv[i] = p.q[i][0].get();
        a.qs[i] = p.q[i][1].get();
        a.qd[i] = p.q[i][2].get();
        a.hv[i] = p.hub[i][0].get();
        a.hs[i] = p.hub[i][1].get();
        a.ho[i] = p.hubOff[i].get();
    }
    for (int i = 0; i < 3; ++i) a.bm[i] = p.bm[i].get();
    a.visited = p.visited.get();
    a.ctr = p.ctr.get();
    a.trace = p.trace.get();
    a.state = p.state.get();
}

}  // namespace
}  // namespace gb

using namespace gb;

void gb_bfs::ensurePersistent(const gb_bfs_options& o) {
    const int block = o.block ? (int)o.block : 512;
    pWant = (int)o.grid_blocks;
    const uint64_t hubCap = std::min<uint64_t>(n, m / 32 + 1);
    for (int i = 0; i < 2; ++i) {
        for (int j = 0; j < 3; ++j) pq[i][j].ensure(n);
        for (int j = 0; j < 2; ++j) phub[i][j].ensure(hubCap);
        phubOff[i].ensure(hubCap);
    }
    const uint64_t words = (n + 31) / 32;
    for (auto& b : pbm) b.ensure(words);
    pvisited.ensure(words);
    if (!pIsoReady) {  // degrees never change for a handle (hub-first only reorders lists)
        pIso.ensure(words);
        isolatedBitmapKernel<<<(uint32_t)std::min<uint64_t>((words + 255) / 256, 4096), 256, 0, stream.s>>>(
            rowPtr.get(), n, (uint32_t)words, pIso.get());
        GB_LAUNCH_CHECK();
        pIsoReady = true;
    }
    pctr.ensure(3);
    pctl.ensure(4);
    ptrace.ensure(kTraceCap);
    pstate.ensure(S_COUNT);
    for (uint32_t k = 1; k < std::max<uint32_t>(1, o.in_flight); ++k) {
        PSlot& p = pSlot[k - 1];
        for (int i = 0; i < 2; ++i) {
            for (int j = 0; j < 3; ++j) p.q[i][j].ensure(n);
            for (int j = 0; j < 2; ++j) p.hub[i][j].ensure(hubCap);
            p.hubOff[i].ensure(hubCap);
        }
        for (auto& b : p.bm) b.ensure(words);
        p.visited.ensure(words);
        p.ctr.ensure(3);
        p.trace.ensure(kTraceCap);
        p.state.ensure(S_COUNT);
    }
    if (pBlock != block) {
        int perSm = 0;
        if (block == 256)
            GB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, persistentBfsKernel<256>, 256, 0));
        else
            GB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, persistentBfsKernel<512>, 512, 0));
        if (perSm < 1) throw Error(GB_ERR_CUDA, "persistent BFS kernel cannot be resident");
        pMax = perSm * deviceSmCount();
        pBlock = block;
    }
    pGrid = pWant > 0 ? std::min(pWant, pMax) : pMax;
}

void gb_bfs::runPersistent(uint32_t src, const gb_bfs_options& o, std::vector<gb_level>* tr) {
    validateOptions(o);
    ensurePersistent(o);
    PArgs a = makeArgs(*this, o, src);
    if (o.selector == GB_SELECT_LEARNED && !selLoaded[0])
        throw Error(GB_ERR_STATE, "learned selector requested but no parameters are loaded");
    GB_CUDA(cudaMemsetAsync(pctl.get(), 0, 4 * sizeof(unsigned), stream.s));
    GB_CUDA(cudaEventRecord(ev.a, stream.s));
    GB_CUDA(cudaMemsetAsync(dist.get(), 0xFF, n * 4, stream.s));  // every depth infinity (0xFFFFFFFF)
    launchFor(*this, a);
    GB_CUDA(cudaEventRecord(ev.b, stream.s));
    unsigned ctl[4];
    GB_CUDA(cudaMemcpyAsync(ctl, pctl.get(), sizeof ctl, cudaMemcpyDeviceToHost, stream.s));
    GB_CUDA(cudaStreamSynchronize(stream.s));
    lastGpuMs = ev.ms();
    lastLevels = ctl[2];
    if (ctl[1]) throw Error(GB_ERR_TIMEOUT, "persistent BFS: grid barrier wait exceeded its spin limit");
    if (tr) {
        const uint32_t k = std::min<uint32_t>(ctl[2], kTraceCap);
        std::vector<gb_level> t(k);
        if (k) GB_CUDA(cudaMemcpy(t.data(), ptrace.get(), k * sizeof(gb_level), cudaMemcpyDeviceToHost));
        for (auto& r : t) r.pad = 0;
        tr->insert(tr->end(), t.begin(), t.end());
    }
}

// Several sources in one call.  K = in_flight traversals run at once:
// traversal i runs on stream i % K (stream 0 is the handle's) with that
// slot's state, on a cooperative grid of grid_blocks blocks (0: the resident
// blocks / K), writing depth buffer i % B (B = K + 2: dist, then mDist[]) and
// its own four control words (all zeroed by one memset).  The traversals of
// one stream follow one another with no host round trip, and the K streams
// run side by side: a traversal's levels wait on dependent loads and its grid
// barrier, so K of them on a share of the SMs each overlap those waits.  A
// depth buffer is refilled only after its previous traversal (and, with a host
// output, that one's pack and copy) are done: the stream that reuses it waits
// on the buffer's events.  With a host output, traversal i's depths are
// packed on its stream right behind it (the width predicted from the most
// levels seen so far; a depth that does not fit raises the overflow flag),
// copied to pinned memory on the copy stream, and widened by host threads
// while the next traversals run.  The host finishes source i before it queues
// traversal i + B, the next user of buffer i % B, so an overflowing source can
// still be copied whole from its depth buffer.
void gb_bfs::runPersistentMany(const uint32_t* src, uint32_t count, uint32_t* out, uint64_t stride,
                               const gb_bfs_options& o, float* msOut, uint32_t* levelsOut) {
    validateOptions(o);
    ensurePersistent(o);
    if (o.selector == GB_SELECT_LEARNED && !selLoaded[0])
        throw Error(GB_ERR_STATE, "learned selector requested but no parameters are loaded");
    if (count == 0) return;
    const uint32_t K = std::max<uint32_t>(1, o.in_flight), B = K + 2;
    int grid = pGrid;
    if (K > 1) {
        const int share = pMax / (int)K;
        if (share < 1) throw Error(GB_ERR_ARG, "in_flight exceeds the resident blocks of the persistent kernel");
        grid = pWant > 0 ? std::min(pWant, share) : share;
    }
    for (uint32_t b = 1; b < B; ++b) mDist[b - 1].ensure(n + 4);
    if (out)
        for (uint32_t b = 0; b < B; ++b) {  // sized for the widest packed form up front
            mPackDev[b].ensure(2 * n + 16);
            mPackHost[b].ensure(2 * n + 16);
        }
    mCtl.ensure((size_t)count * 4);
    mCtlHost.ensure((size_t)count * 4);
    mFlag.ensure(kManySlots);
    mFlagHost.ensure(count);
    while (mEv.size() < 2 * (size_t)count) {
        cudaEvent_t e;
        GB_CUDA(cudaEventCreate(&e));
        mEv.push_back(e);
    }
    // per buffer: packed, copied, released; then the start event and one end event per stream
    while (mSlotEv.size() < 3 * (size_t)kManySlots + 1 + kMaxInFlight) {
        cudaEvent_t e;
        GB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        mSlotEv.push_back(e);
    }
    uint32_t* bufs[kManySlots];
    bufs[0] = dist.get();
    for (uint32_t b = 1; b < B; ++b) bufs[b] = mDist[b - 1].get();
    cudaStream_t streams[kMaxInFlight];
    streams[0] = stream.s;
    for (uint32_t k = 1; k < K; ++k) {
        if (!pStream[k - 1]) pStream[k - 1] = std::make_unique<gb::Stream>();
        streams[k] = pStream[k - 1]->s;
    }
    cudaEvent_t startEv = mSlotEv[3 * kManySlots];
    std::vector<int> fmt(count, -1);
    // packed width: from the most levels among this call's finished sources,
    // else the handle's last run, else one byte per depth
    uint32_t maxSeen = 0;
    bool anySeen = false;
    const bool timed = msOut != nullptr;
    cudaStream_t cs = copyStream.s;

    GB_CUDA(cudaMemsetAsync(mCtl.get(), 0, (size_t)count * 4 * sizeof(unsigned), stream.s));
    // the other streams start after the work queued before this call on the handle's stream
    GB_CUDA(cudaEventRecord(startEv, stream.s));
    for (uint32_t k = 1; k < K; ++k) GB_CUDA(cudaStreamWaitEvent(streams[k], startEv, 0));
    auto enqueue = [&](uint32_t i) {
        const uint32_t k = i % K, b = i % B;
        cudaStream_t st = streams[k];
        PArgs a = makeArgs(*this, o, src[i]);
        if (k) useSlot(*this, a, (int)k);
        a.dist = bufs[b];
        a.ctl = mCtl.get() + 4 * (size_t)i;
        cudaEvent_t packed = mSlotEv[b], copied = mSlotEv[kManySlots + b], released = mSlotEv[2 * kManySlots + b];
        if (i >= B) {  // buffer b's previous traversal (and its pack and copy) first
            GB_CUDA(cudaStreamWaitEvent(st, released, 0));
            if (out) GB_CUDA(cudaStreamWaitEvent(st, copied, 0));
        }
        if (timed || i + 1 == count) GB_CUDA(cudaEventRecord(mEv[2 * i], st));
        GB_CUDA(cudaMemsetAsync(bufs[b], 0xFF, n * 4, st));  // every depth infinity
        launchFor(*this, a, grid, st);
        if (timed || i + 1 == count) GB_CUDA(cudaEventRecord(mEv[2 * i + 1], st));
        if (!out) {
            GB_CUDA(cudaEventRecord(released, st));
            return;
        }
        fmt[i] = packFormat(n, anySeen ? maxSeen : lastLevels ? lastLevels : 254);
        if (fmt[i] >= 0) {
            GB_CUDA(cudaMemsetAsync(mFlag.get() + b, 0, sizeof(unsigned), st));
            enqueuePack(fmt[i], bufs[b], n, mPackDev[b].get(), mFlag.get() + b, st);
        }
        GB_CUDA(cudaEventRecord(packed, st));
        GB_CUDA(cudaEventRecord(released, st));
        GB_CUDA(cudaStreamWaitEvent(cs, packed, 0));
        if (fmt[i] >= 0) {
            GB_CUDA(cudaMemcpyAsync(mPackHost[b].p, mPackDev[b].get(), packedBytes(fmt[i], n),
                                    cudaMemcpyDeviceToHost, cs));
            GB_CUDA(cudaMemcpyAsync(mFlagHost.p + i, mFlag.get() + b, sizeof(unsigned), cudaMemcpyDeviceToHost, cs));
        }
        GB_CUDA(cudaMemcpyAsync(mCtlHost.p + 4 * (size_t)i, mCtl.get() + 4 * (size_t)i, 4 * sizeof(unsigned),
                                cudaMemcpyDeviceToHost, cs));
        GB_CUDA(cudaEventRecord(copied, cs));
    };
    auto joinStreams = [&]() {  // the handle's stream covers every stream's work
        for (uint32_t k = 1; k < K; ++k) {
            cudaEvent_t endEv = mSlotEv[3 * kManySlots + 1 + k];
            GB_CUDA(cudaEventRecord(endEv, streams[k]));
            GB_CUDA(cudaStreamWaitEvent(stream.s, endEv, 0));
        }
    };
    auto timeout = [&]() {
        for (uint32_t k = 0; k < K; ++k) cudaStreamSynchronize(streams[k]);
        cudaStreamSynchronize(cs);
        return Error(GB_ERR_TIMEOUT, "persistent BFS: grid barrier wait exceeded its spin limit");
    };

    uint32_t queued = 0;
    if (!out) {
        for (; queued < count; ++queued) enqueue(queued);
        joinStreams();
        GB_CUDA(cudaMemcpyAsync(mCtlHost.p, mCtl.get(), (size_t)count * 4 * sizeof(unsigned),
                                cudaMemcpyDeviceToHost, stream.s));
    } else {
        for (uint32_t i = 0; i < count; ++i) {
            for (; queued < count && queued < i + B; ++queued) enqueue(queued);
            const uint32_t b = i % B;
            GB_CUDA(cudaEventSynchronize(mSlotEv[kManySlots + b]));
            const unsigned* c = mCtlHost.p + 4 * (size_t)i;
            if (c[1]) throw timeout();
            maxSeen = std::max(maxSeen, c[2]);
            anySeen = true;
            uint32_t* dst = out + (uint64_t)i * stride;
            if (fmt[i] >= 0 && mFlagHost.p[i] == 0) {
                widenPacked(fmt[i], mPackHost[b].p, n, dst);
            } else {  // too many levels for the predicted width: the buffer is still intact
                GB_CUDA(cudaMemcpyAsync(dst, bufs[b], n * 4, cudaMemcpyDeviceToHost, cs));
                GB_CUDA(cudaStreamSynchronize(cs));
            }
        }
        joinStreams();
    }
    for (uint32_t k = 0; k < K; ++k) GB_CUDA(cudaStreamSynchronize(streams[k]));
    GB_CUDA(cudaStreamSynchronize(cs));
    for (uint32_t i = 0; i < count; ++i)
        if (mCtlHost.p[4 * (size_t)i + 1]) throw timeout();
    for (uint32_t i = 0; i < count; ++i) {
        if (levelsOut) levelsOut[i] = mCtlHost.p[4 * (size_t)i + 2];
        if (timed) GB_CUDA(cudaEventElapsedTime(&msOut[i], mEv[2 * i], mEv[2 * i + 1]));
    }
    float last = 0;
    GB_CUDA(cudaEventElapsedTime(&last, mEv[2 * (count - 1)], mEv[2 * (count - 1) + 1]));
    lastGpuMs = last;
    lastLevels = mCtlHost.p[4 * (size_t)(count - 1) + 2];
    const uint32_t lastBuf = (count - 1) % B;
    if (lastBuf) dist.swap(mDist[lastBuf - 1]);  // dist holds the last source's depths
}

// Selector training data.  A level's vertex set does not depend on the
// strategy that ran the earlier levels, so running the whole BFS once per
// strategy (forced at every level, alpha/beta rule off) gives every level's
// device time under every strategy, measured in a running traversal (warm
// caches, the real barrier and counter traffic) rather than in a one-level
// launch.  The features come from the top-down run's trace, whose per-level
// edge count is the frontier's degree sum, exactly as the kernel sees it.
size_t gb_bfs::profileLevels(uint32_t src, const gb_bfs_options& o0, int repeats, float* feats, float* times,
                             size_t cap) {
    gb_bfs_options o = o0;
    o.selector = GB_SELECT_RULE;
    std::vector<std::vector<gb_level>> per(GB_NUM_STRATS);
    for (int s = 0; s < GB_NUM_STRATS; ++s) {
        o.force_strategy = s;
        for (int r = 0; r <= repeats; ++r) {  // run 0 warms up
            std::vector<gb_level> tr;
            runPersistent(src, o, &tr);
            if (r == 0) continue;
            if (per[s].empty()) {
                per[s] = tr;
            } else {
                for (size_t i = 0; i < std::min(tr.size(), per[s].size()); ++i)
                    per[s][i].time_ms = std::min(per[s][i].time_ms, tr[i].time_ms);
            }
        }
        if (per[s].size() != per[0].size()) throw Error(GB_ERR_STATE, "level count differs between strategies");
    }
    const std::vector<gb_level>& td = per[GB_STRAT_TD_EPT2];
    double reached = 0, seenEdges = 0;
    size_t rows = 0;
    for (size_t L = 0; L < td.size() && rows < cap; ++L, ++rows) {
        const double frontier = (double)td[L].frontier, fedges = (double)td[L].edges;
        reached += frontier;
        seenEdges += fedges;
        selectorFeatures(frontier, fedges, std::max(0.0, (double)m - seenEdges), std::max(0.0, (double)n - reached),
                         (double)n, (double)m, (double)L, feats + rows * kSelFeatures);
        for (int s = 0; s < GB_NUM_STRATS; ++s) times[rows * GB_NUM_STRATS + s] = (float)(per[s][L].time_ms * 1e3);
    }
    return rows;
}
