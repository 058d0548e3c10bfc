// bfs_batch.cu -- up to 64 BFS sources in one persistent cooperative launch.
//
// Replaces the reference's one-source-at-a-time loop (src/bench/main.cpp:324-364).
// Bit i of a vertex's 64-bit masks stands for source i:
//   seen[v]    sources that have reached v;
//   fr[2][v]   sources whose frontier v is on at the current / next level;
//   nx[v]      bits pushed to v during a top-down level (zero between levels).
// Active vertices (fr != 0) are kept in a queue (vertex, adjacency start,
// degree) and a hub list for degree >= hub_min, as in the single-source kernel.
// A level runs top-down (push: bits = fr[u] & ~seen[v], atomicOr into nx[v];
// the first pusher of v appends it to a candidate list; after a grid barrier
// the candidates' new bits are folded into seen / fr / depths) or bottom-up
// (pull: every vertex still missing sources ORs its neighbours' frontier masks
// until it has them all).  The direction rule of cpu::bfsDO
// (src/cpu/bfs_cpu.cpp:227-283) runs on the batch's counters (active vertices
// and their edges), or the learned selector picks; depths are the same either
// way.  Depths: dist[i*n + v]; unreached entries are written once at the end.
#include <algorithm>
#include <cstring>

#include "bfs.hpp"
#include "bfs_device.cuh"

namespace gb {
namespace {

constexpr unsigned long long kHubShift = 40;
constexpr unsigned long long kHubMask = (1ull << kHubShift) - 1;
constexpr uint32_t kTraceCap = 1u << 16;
#ifndef GB_BATCH_BU_SERIAL
#define GB_BATCH_BU_SERIAL 64
#endif
#ifndef GB_BATCH_BU_COOP
#define GB_BATCH_BU_COOP 64
#endif
#ifndef GB_BATCH_BU_BLOCK
#define GB_BATCH_BU_BLOCK 256
#endif
// bottom-up list scans: serial per thread for the first kBatchBuSerial entries,
// then a rest of kBatchBuCoop entries or more by the warp, kBatchBuBlock or
// more by the block
constexpr uint32_t kBatchBuSerial = GB_BATCH_BU_SERIAL;
constexpr uint32_t kBatchBuCoop = GB_BATCH_BU_COOP;
constexpr uint32_t kBatchBuBlock = GB_BATCH_BU_BLOCK;
#ifndef GB_BATCH_BU_UNROLL
#define GB_BATCH_BU_UNROLL 8
#endif
constexpr int kBuUnroll = GB_BATCH_BU_UNROLL;  // entries per thread per cooperative step

struct BCounters {
    unsigned acnt;                 // next active queue entries
    unsigned ccnt;                 // top-down candidates
    unsigned work[2];              // work tickets: expansion, finalisation
    unsigned long long hubPack;    // next active hubs: (count << 40) | degree sum
    unsigned long long aedges;     // degree sum of the next active vertices
    unsigned long long found;      // next active vertices
    unsigned long long bits;       // newly set (vertex, source) pairs
    unsigned long long fullEdges;  // degree sum of vertices that became fully seen
    unsigned long long fullCount;
    unsigned long long examined;
    unsigned dcnt;                 // bottom-up: lists whose rest is deferred to a whole block
};

struct BArgs {
    const uint32_t* __restrict__ row_ptr;
    const uint32_t* __restrict__ col_idx;
    unsigned long long* seen;
    unsigned long long* fr[2];
    unsigned long long* nx;
    uint32_t* qv[2];
    uint32_t* qs[2];
    uint32_t* qd[2];
    uint32_t* hv[2];
    uint32_t* hs[2];
    unsigned long long* ho[2];
    uint32_t* cq;
    uint2* dq;  // bottom-up: (vertex, resume position) of the deferred rests
    uint32_t* dist;
    const uint32_t* sources;
    BCounters* ctr;
    unsigned* ctl;
    gb_level* trace;
    const float* sel;
    uint64_t n, m;
    unsigned long long all;
    int k;
    uint32_t hubMin, traceCap;
    double alpha, beta;
    float selMargin;  // learned selector: log2 margin for leaving the rule's direction
    int selector, force;
    unsigned long long spinLimit;
};

__device__ __forceinline__ unsigned long long ldv64(const unsigned long long* p) {
    return *reinterpret_cast<const volatile unsigned long long*>(p);
}
__device__ __forceinline__ unsigned ldv32(const unsigned* p) { return *reinterpret_cast<const volatile unsigned*>(p); }

__device__ __forceinline__ unsigned long long warpOr64(unsigned long long x) {
    unsigned lo = __reduce_or_sync(kFull, (unsigned)x), hi = __reduce_or_sync(kFull, (unsigned)(x >> 32));
    return ((unsigned long long)hi << 32) | lo;
}

struct BAcc {
    unsigned long long found = 0, aedges = 0, bits = 0, fullEdges = 0, fullCount = 0, exam = 0;
};

template <int NT>
struct BSmem {
    uint32_t scan[NT / 32 + 1];
    uint32_t off[NT];
    uint32_t st[NT];
    unsigned long long f[NT];
    float sel[kSelParams];
    unsigned long long acc[6];
    unsigned long long cnt[7];  // counters after a barrier (see batchBarrier)
    uint32_t range[2];
    unsigned item;
    int strat;
    uint32_t base;
    int ok;
    unsigned bor[2];  // bottom-up deferred rests: OR of the frontier masks found (lo, hi)
    uint32_t dn;      // ... and their count
};

// Grid barrier after which every thread of the block sees counters *c in
// sm.cnt (found, aedges, fullEdges, fullCount, acnt, hubPack, ccnt), read
// once per block by thread 0 instead of once per warp.
template <int NT>
__device__ __forceinline__ bool batchBarrier(const BArgs& a, BSmem<NT>& sm, const BCounters* c) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const bool ok = gridArriveWait(&a.ctl[0], &a.ctl[1], a.spinLimit, gridDim.x);
        sm.ok = ok;
        if (ok) {
            sm.cnt[0] = ldv64(&c->found);
            sm.cnt[1] = ldv64(&c->aedges);
            sm.cnt[2] = ldv64(&c->fullEdges);
            sm.cnt[3] = ldv64(&c->fullCount);
            sm.cnt[4] = ldv32(&c->acnt);
            sm.cnt[5] = ldv64(&c->hubPack);
            sm.cnt[6] = ldv32(&c->ccnt);
        }
    }
    __syncthreads();
    return sm.ok != 0;
}

// Write depth `level` for the sources in b (lanes of a warp call together;
// consecutive vertices give coalesced stores per source).
__device__ __forceinline__ void writeDepths(const BArgs& a, uint64_t v, unsigned long long b, uint32_t value) {
    unsigned long long any = warpOr64(b);
    while (any) {
        const int s = __ffsll((long long)any) - 1;
        any &= any - 1;
        if ((b >> s) & 1ull) a.dist[(uint64_t)s * a.n + v] = value;
    }
}

// Block-aggregated append of vertex v (with its adjacency start and degree)
// to the next active queue or hub list.  All threads of the block call it.
template <int NT>
__device__ __forceinline__ void appendActive(const BArgs& a, BSmem<NT>& sm, bool want, uint32_t v, uint32_t st,
                                             uint32_t d, uint32_t nq, BCounters* cur) {
    const bool hub = want && d >= a.hubMin;
    const bool q = want && !hub;
    uint32_t tot;
    const uint32_t pos = blockScan<NT>(q ? 1u : 0u, &tot, sm.scan);
    if (threadIdx.x == 0) sm.base = tot ? atomicAdd(&cur->acnt, tot) : 0u;
    __syncthreads();
    if (q) {
        const uint32_t p = sm.base + pos;
        a.qv[nq][p] = v;
        a.qs[nq][p] = st;
        a.qd[nq][p] = d;
    }
    if (hub) {
        const unsigned long long old = atomicAdd(&cur->hubPack, (1ull << kHubShift) | d);
        const uint32_t i = (uint32_t)(old >> kHubShift);
        a.hv[nq][i] = v;
        a.hs[nq][i] = st;
        a.ho[nq][i] = old & kHubMask;
    }
    __syncthreads();
}

// Warp-aggregated form of appendActive (every lane of the warp calls it): no
// block barrier, so the warps of a block need not wait for one another.
__device__ __forceinline__ void warpAppendActive(const BArgs& a, bool want, uint32_t v, uint32_t st, uint32_t d,
                                                 uint32_t nq, BCounters* cur) {
    const bool hub = want && d >= a.hubMin;
    const bool q = want && !hub;
    if (__any_sync(kFull, q)) {
        const uint32_t p = warpAppend(q, &cur->acnt);
        if (q) {
            a.qv[nq][p] = v;
            a.qs[nq][p] = st;
            a.qd[nq][p] = d;
        }
    }
    if (hub) {
        const unsigned long long old = atomicAdd(&cur->hubPack, (1ull << kHubShift) | d);
        const uint32_t i = (uint32_t)(old >> kHubShift);
        a.hv[nq][i] = v;
        a.hs[nq][i] = st;
        a.ho[nq][i] = old & kHubMask;
    }
}

// Fold new bits b into v (owner thread only): seen, next frontier, depths
// (by the caller, warp-wide), counters.
__device__ __forceinline__ void foldBits(const BArgs& a, uint64_t v, unsigned long long old,
                                         unsigned long long b, uint32_t d, BAcc& acc) {
    a.seen[v] = old | b;
    acc.found++;
    acc.aedges += d;
    acc.bits += __popcll(b);
    if ((old | b) == a.all) {
        acc.fullEdges += d;
        acc.fullCount++;
    }
}

// Top-down push of one tile of NT active entries (edge-balanced, as the
// single-source kernel): the entry's frontier mask minus the target's seen
// mask is ORed into nx[target]; the first pusher records a candidate.  The
// block pushes part `part` of `parts` equal slices of the tile's edges.
template <int NT, int EPT>
__device__ void pushTile(const BArgs& a, BSmem<NT>& sm, uint32_t item, uint32_t S, uint32_t qc, BCounters* cur,
                         uint32_t part, uint32_t parts) {
    const uint32_t idx = item * NT + threadIdx.x;
    uint32_t st = 0, d = 0;
    unsigned long long f = 0;
    if (idx < S) {
        st = a.qs[qc][idx];
        d = a.qd[qc][idx];
        f = a.fr[qc][a.qv[qc][idx]];
    }
    uint32_t tot;
    const uint32_t off = blockScan<NT>(d, &tot, sm.scan);
    sm.off[threadIdx.x] = off;
    sm.st[threadIdx.x] = st;
    sm.f[threadIdx.x] = f;
    __syncthreads();
    const uint32_t cnt = min((uint32_t)NT, S - item * NT);
    const uint32_t lo = (uint32_t)((uint64_t)tot * part / parts), hi = (uint32_t)((uint64_t)tot * (part + 1) / parts);
    for (uint32_t base = lo; base < hi; base += NT * EPT) {
        uint32_t u[EPT];
        unsigned long long fu[EPT];
#pragma unroll
        for (int k = 0; k < EPT; ++k) {
            const uint32_t e = base + k * NT + threadIdx.x;
            u[k] = 0;
            fu[k] = 0;
            if (e < hi) {
                const uint32_t o = ownerOf(sm.off, 0u, cnt - 1, e);
                u[k] = a.col_idx[sm.st[o] + (e - sm.off[o])];
                fu[k] = sm.f[o];
            }
        }
        // the EPT pushes issued stage by stage (seen masks, then the ORs), so
        // their round trips overlap
        unsigned long long bits[EPT], old[EPT];
#pragma unroll
        for (int k = 0; k < EPT; ++k) bits[k] = fu[k] ? (fu[k] & ~a.seen[u[k]]) : 0ull;
#pragma unroll
        for (int k = 0; k < EPT; ++k) old[k] = bits[k] ? atomicOr(&a.nx[u[k]], bits[k]) : 1ull;
#pragma unroll
        for (int k = 0; k < EPT; ++k) {
            const bool cand = old[k] == 0ull;
            if (__any_sync(kFull, cand)) {
                const uint32_t pos = warpAppend(cand, &cur->ccnt);
                if (cand) a.cq[pos] = u[k];
            }
        }
    }
    __syncthreads();
}

template <int NT>
__device__ void pushWarpItem(const BArgs& a, uint32_t item, uint32_t S, uint32_t qc, BCounters* cur) {
    const uint32_t idx = item * (NT / 32) + (threadIdx.x >> 5);
    if (idx >= S) return;  // warp-uniform
    const uint32_t st = a.qs[qc][idx], d = a.qd[qc][idx];
    const unsigned long long f = a.fr[qc][a.qv[qc][idx]];
    for (uint32_t base = 0; base < d; base += 64) {  // two rounds per step: their pushes overlap
        const uint32_t e0 = base + laneId(), e1 = e0 + 32;
        const uint32_t u0 = e0 < d ? a.col_idx[st + e0] : 0u, u1 = e1 < d ? a.col_idx[st + e1] : 0u;
        const unsigned long long b0 = e0 < d ? f & ~a.seen[u0] : 0ull, b1 = e1 < d ? f & ~a.seen[u1] : 0ull;
        const unsigned long long o0 = b0 ? atomicOr(&a.nx[u0], b0) : 1ull, o1 = b1 ? atomicOr(&a.nx[u1], b1) : 1ull;
        const bool c0 = o0 == 0ull, c1 = o1 == 0ull;
        if (__any_sync(kFull, c0 || c1)) {
            const uint32_t p0 = warpAppend(c0, &cur->ccnt);
            if (c0) a.cq[p0] = u0;
            const uint32_t p1 = warpAppend(c1, &cur->ccnt);
            if (c1) a.cq[p1] = u1;
        }
    }
}

template <int NT>
__device__ void pushHubChunk(const BArgs& a, BSmem<NT>& sm, uint64_t e0, uint64_t e1, uint32_t H, uint32_t qc,
                             BCounters* cur) {
    const unsigned long long* ho = a.ho[qc];
    if (threadIdx.x < 64) {  // the chunk's first and last owners: warp 0 and warp 1 side by side
        const unsigned long long key = threadIdx.x < 32 ? e0 : e1 - 1;
        const uint32_t o = warpOwnerOf(ho, 0u, H - 1, key);
        if ((threadIdx.x & 31u) == 0) sm.range[threadIdx.x >> 5] = o;
    }
    __syncthreads();
    const uint32_t lo = sm.range[0], hi = sm.range[1];
    for (uint64_t base = e0; base < e1; base += NT) {
        const uint64_t e = base + threadIdx.x;
        bool cand = false;
        uint32_t u = 0;
        if (e < e1) {
            const uint32_t o = ownerOf(ho, lo, hi, (unsigned long long)e);
            u = a.col_idx[a.hs[qc][o] + (uint32_t)(e - ho[o])];
            const unsigned long long bits = a.fr[qc][a.hv[qc][o]] & ~a.seen[u];
            if (bits) cand = atomicOr(&a.nx[u], bits) == 0ull;
        }
        if (__any_sync(kFull, cand)) {
            const uint32_t pos = warpAppend(cand, &cur->ccnt);
            if (cand) a.cq[pos] = u;
        }
    }
    __syncthreads();
}

template <int NT>
__global__ void __launch_bounds__(NT, 1024 / NT) batchBfsKernel(BArgs a) {
    __shared__ BSmem<NT> sm;
    const unsigned tid = threadIdx.x;
    const uint64_t gtid = (uint64_t)blockIdx.x * NT + tid, gthreads = (uint64_t)gridDim.x * NT;
    unsigned* bar = &a.ctl[0];
    unsigned* err = &a.ctl[1];
    const bool learned = a.selector == GB_SELECT_LEARNED && a.sel != nullptr;
    if (learned)
        selectorStage(sm.sel, a.sel, tid, NT);

    // prologue: masks zeroed, counters zeroed, then the sources
    for (uint64_t v = gtid; v < a.n; v += gthreads) {
        a.seen[v] = 0;
        a.fr[0][v] = 0;
        a.fr[1][v] = 0;
        a.nx[v] = 0;
    }
    if (gtid == 0)
        for (int s = 0; s < 4; ++s) a.ctr[s] = BCounters{};
    if (!gridBarrier(bar, err, a.spinLimit)) return;
    if (blockIdx.x == 0 && tid < (unsigned)a.k) {
        const uint32_t v = a.sources[tid];
        const unsigned long long bit = 1ull << tid;
        const unsigned long long old = atomicOr(&a.fr[0][v], bit);
        atomicOr(&a.seen[v], bit);
        a.dist[(uint64_t)tid * a.n + v] = 0;
        BCounters* c = &a.ctr[3];
        atomicAdd(&c->bits, 1ull);
        if (old == 0) {  // first source at v: v becomes active
            const uint32_t st = a.row_ptr[v], d = a.row_ptr[v + 1] - st;
            atomicAdd(&c->found, 1ull);
            atomicAdd(&c->aedges, (unsigned long long)d);
            if (d >= a.hubMin) {
                const unsigned long long o = atomicAdd(&c->hubPack, (1ull << kHubShift) | d);
                const uint32_t i = (uint32_t)(o >> kHubShift);
                a.hv[0][i] = v;
                a.hs[0][i] = st;
                a.ho[0][i] = o & kHubMask;
            } else {
                const uint32_t p = atomicAdd(&c->acnt, 1u);
                a.qv[0][p] = v;
                a.qs[0][p] = st;
                a.qd[0][p] = d;
            }
        }
    }
    if (!batchBarrier<NT>(a, sm, &a.ctr[3])) return;

    uint32_t level = 0;
    bool bottomUp = false;
    uint64_t scout = sm.cnt[1], toCheck = a.m, fullEdges = 0, fullCount = 0;
    int lastStrat = -1;
    uint64_t tPrev = globaltimer();
    // The last two levels' outputs, carried in registers: (size, fedges,
    // qCount, qHub) of level-1 and (q2Count, q2Hub) of level-2.
    uint64_t size = sm.cnt[0], fedges = sm.cnt[1];
    uint32_t qCount = (uint32_t)sm.cnt[4], q2Count = 0;
    unsigned long long qHub = sm.cnt[5], q2Hub = 0;
    for (;;) {
        BCounters* prev = &a.ctr[(level + 3) & 3];
        BCounters* cur = &a.ctr[level & 3];
        if (size == 0) break;
        if (!bottomUp && (double)scout > (double)toCheck / a.alpha) bottomUp = true;
        if (!bottomUp) toCheck -= min(toCheck, scout);
        const int ruleStrat = bottomUp ? GB_STRAT_BU : GB_STRAT_TD_EPT2;
        int strat = ruleStrat;
        if (a.force >= 0) {
            strat = a.force;
        } else if (learned) {
            if (tid < 32) {
                float f[kSelFeatures];
                selectorFeatures((double)size, (double)fedges, (double)(a.m > fullEdges ? a.m - fullEdges : 0),
                                 (double)(a.n - fullCount), (double)a.n, (double)a.m, (double)level, f);
                // trust region: bottom-up only within 4x of the rule's threshold
                const bool mayGoBU = (double)scout * 4.0 > (double)toCheck / a.alpha;
                const int s = selectorChoose(sm.sel, f, tid, bottomUp, a.selMargin, mayGoBU);
                if (tid == 0) sm.strat = s;
            }
            __syncthreads();
            if (sm.strat >= 0) strat = sm.strat;
        }
        if (gtid == 0) {
            if (a.trace && level > 0 && level - 1 < a.traceCap && lastStrat == GB_STRAT_BU)
                a.trace[level - 1].edges = ldv64(&prev->examined);
            if (a.trace && level < a.traceCap) {
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
            a.ctr[(level + 1) & 3] = BCounters{};
        }
        if (tid == 0)
            for (int i = 0; i < 6; ++i) sm.acc[i] = 0;
        __syncthreads();
        const uint32_t qc = level & 1u, nq = qc ^ 1u;
        BAcc acc;
        if (strat == GB_STRAT_BU) {
            const unsigned long long* fc = a.fr[qc];
            for (uint64_t base = (uint64_t)blockIdx.x * NT; base < a.n; base += gthreads) {
                const uint64_t v = base + tid;
                unsigned long long b = 0, old = 0, need = 0;
                uint32_t st = 0, d = 0;
                if (v < a.n) {
                    old = a.seen[v];
                    need = a.all & ~old;
                    st = a.row_ptr[v];
                    d = a.row_ptr[v + 1] - st;
                }
                // Each thread ORs its vertex's neighbours' frontier masks until
                // every missing source is covered (most lists stop early), for
                // at most kBatchBuSerial entries; aligned groups of 4 entries
                // are loaded at once with their 4 masks.  What is left of a
                // list then goes to the whole warp (kBatchBuCoop or more
                // entries left: the warp takes such lists one after another,
                // 32 kBuUnroll entries per step) or, from kBatchBuBlock entries
                // left, to a whole block after this loop; shorter rests finish
                // serially.  One long list scanned by one thread would hold its
                // warp and the level; the loop has no block barrier, so the
                // warps of a block do not wait for one another.
                unsigned long long got = 0;
                uint32_t i = st;
                const uint32_t e = st + d;
                auto scanTo = [&](uint32_t lim) {
                    for (; i < lim && (i & 3u) && (got & need) != need; ++i) got |= fc[a.col_idx[i]];
                    for (; i + 4 <= lim && (got & need) != need; i += 4) {
                        const uint4 q = *reinterpret_cast<const uint4*>(a.col_idx + i);
                        got |= fc[q.x] | fc[q.y] | fc[q.z] | fc[q.w];
                    }
                    for (; i < lim && (got & need) != need; ++i) got |= fc[a.col_idx[i]];
                };
                if (need) scanTo(st + min(d, kBatchBuSerial));
                const uint32_t rest = (need && (got & need) != need) ? e - i : 0u;
                const bool huge = rest >= kBatchBuBlock;
                const bool coop = !huge && rest >= kBatchBuCoop;
                if (rest && !huge && !coop) scanTo(e);
                const unsigned long long want = need & ~got;  // still missing after the serial part
                for (unsigned hm = __ballot_sync(kFull, coop); hm; hm &= hm - 1) {
                    const int l = __ffs(hm) - 1;
                    const uint32_t hs = __shfl_sync(kFull, i, l), hd = __shfl_sync(kFull, e, l) - hs;
                    const unsigned long long hn = __shfl_sync(kFull, want, l);
                    unsigned long long g2 = 0;
                    uint32_t off = 0;
                    while (off < hd) {
                        unsigned long long g = 0;
#pragma unroll
                        for (int q = 0; q < kBuUnroll; ++q) {
                            const uint32_t j = off + laneId() + 32u * q;
                            if (j < hd) g |= fc[a.col_idx[hs + j]];
                        }
                        g2 |= warpOr64(g);
                        off += 32u * kBuUnroll;
                        if ((g2 & hn) == hn) break;
                    }
                    if (laneId() == (unsigned)l) {
                        got |= g2;
                        i += min(off, hd);
                    }
                }
                // rests of kBatchBuBlock or more entries: deferred to the phase
                // below (the masks found so far wait in nx, zero in bottom-up levels)
                if (huge) a.nx[v] = got;
                if (__any_sync(kFull, huge)) {
                    const uint32_t p = warpAppend(huge, &cur->dcnt);
                    if (huge) a.dq[p] = make_uint2((uint32_t)v, i);
                }
                if (v < a.n && !huge) {
                    if (need) {
                        acc.exam += i - st;
                        b = got & need;
                    }
                    a.fr[nq][v] = b;  // dense: also clears the level-before-last frontier
                    if (b) foldBits(a, v, old, b, d, acc);
                }
                writeDepths(a, v, b, level + 1);
                warpAppendActive(a, b != 0, (uint32_t)v, st, d, nq, cur);
            }
            // the deferred rests, one at a time per block, taken by ticket over
            // the whole grid (kBuUnroll NT entries per step, the block's OR of
            // masks in shared memory, stopping once every missing source is found)
            if (!batchBarrier<NT>(a, sm, cur)) return;
            if (tid == 0) sm.dn = ldv32(&cur->dcnt);
            __syncthreads();
            const uint32_t D = sm.dn;
            for (bool first = true;; first = false) {
                if (tid == 0) sm.item = first ? blockIdx.x : gridDim.x + atomicAdd(&cur->work[0], 1u);
                __syncthreads();
                const uint32_t item = sm.item;
                if (item >= D) break;  // block-uniform
                const uint2 ent = a.dq[item];
                const uint32_t v = ent.x, st = a.row_ptr[v], e = a.row_ptr[v + 1];
                const unsigned long long old = a.seen[v], need = a.all & ~old, got0 = a.nx[v];
                const unsigned long long hn = need & ~got0;
                if (tid == 0) {
                    sm.bor[0] = 0;
                    sm.bor[1] = 0;
                }
                __syncthreads();
                const uint32_t hd = e - ent.y;
                unsigned long long g2 = 0;
                uint32_t off = 0;
                while (off < hd) {
                    unsigned long long g = 0;
#pragma unroll
                    for (int q = 0; q < kBuUnroll; ++q) {
                        const uint32_t j = off + tid + (uint32_t)NT * q;
                        if (j < hd) g |= fc[a.col_idx[ent.y + j]];
                    }
                    g = warpOr64(g);
                    if (laneId() == 0 && g) {
                        atomicOr(&sm.bor[0], (unsigned)g);
                        atomicOr(&sm.bor[1], (unsigned)(g >> 32));
                    }
                    __syncthreads();
                    g2 = ((unsigned long long)sm.bor[1] << 32) | sm.bor[0];
                    off += (uint32_t)kBuUnroll * NT;
                    if ((g2 & hn) == hn) break;  // block-uniform: all read bor between barriers
                    __syncthreads();
                }
                if (tid == 0) {
                    const unsigned long long b = (got0 | g2) & need;
                    const uint32_t d = e - st;
                    acc.exam += (ent.y - st) + min(off, hd);
                    a.nx[v] = 0;
                    a.fr[nq][v] = b;
                    if (b) {
                        foldBits(a, v, old, b, d, acc);
                        for (unsigned long long bb = b; bb; bb &= bb - 1)
                            a.dist[(uint64_t)(__ffsll((long long)bb) - 1) * a.n + v] = level + 1;
                        if (d >= a.hubMin) {
                            const unsigned long long hp = atomicAdd(&cur->hubPack, (1ull << kHubShift) | d);
                            const uint32_t hi = (uint32_t)(hp >> kHubShift);
                            a.hv[nq][hi] = v;
                            a.hs[nq][hi] = st;
                            a.ho[nq][hi] = hp & kHubMask;
                        } else {
                            const uint32_t p = atomicAdd(&cur->acnt, 1u);
                            a.qv[nq][p] = v;
                            a.qs[nq][p] = st;
                            a.qd[nq][p] = d;
                        }
                    }
                }
                __syncthreads();  // sm.bor and sm.item are reused by the next list
            }
        } else {
            // phase A: clear the previous level's frontier entries of fr[nq]
            // (its active list is still intact), then push.
            {
                const uint32_t P = q2Count;
                for (uint64_t i = gtid; i < P; i += gthreads) a.fr[nq][a.qv[nq][i]] = 0;
                const uint32_t PH = (uint32_t)(q2Hub >> kHubShift);
                for (uint64_t i = gtid; i < PH; i += gthreads) a.fr[nq][a.hv[nq][i]] = 0;
            }
            const uint32_t S = qCount;
            const unsigned long long hp = qHub;
            const uint32_t H = (uint32_t)(hp >> kHubShift);
            const uint64_t HE = hp & kHubMask;
            const uint32_t per = strat == GB_STRAT_TD_WARP ? NT / 32 : NT;
            const uint32_t nt = (S + per - 1) / per;
            // fewer edge-balanced tiles than half the blocks: each is split by
            // edge range into parts of at least 8 NT edges (as the
            // single-source kernel)
            uint32_t parts = 1;
            if (strat != GB_STRAT_TD_WARP && nt && nt * 2 <= gridDim.x) {
                const uint64_t perPart = (fedges > HE ? fedges - HE : 0) / nt / (8ull * NT);
                const uint64_t cap = gridDim.x / nt;
                parts = perPart < 1 ? 1u : (uint32_t)(perPart < cap ? perPart : cap);
            }
            const uint32_t nti = nt * parts;
            const uint64_t HC = (uint64_t)NT * 4;
            const uint32_t nh = (uint32_t)((HE + HC - 1) / HC);
            for (bool first = true;; first = false) {  // block b takes item b first
                if (tid == 0) sm.item = first ? blockIdx.x : gridDim.x + atomicAdd(&cur->work[0], 1u);
                __syncthreads();
                const uint32_t item = sm.item;
                __syncthreads();
                if (item >= nti + nh) break;
                if (item < nti) {
                    const uint32_t tile = item / parts, part = item - tile * parts;
                    switch (strat) {
                        case GB_STRAT_TD_EPT1: pushTile<NT, 1>(a, sm, tile, S, qc, cur, part, parts); break;
                        case GB_STRAT_TD_EPT4: pushTile<NT, 4>(a, sm, tile, S, qc, cur, part, parts); break;
                        case GB_STRAT_TD_WARP: pushWarpItem<NT>(a, item, S, qc, cur); break;
                        default: pushTile<NT, 2>(a, sm, tile, S, qc, cur, part, parts); break;
                    }
                } else {
                    const uint64_t e0 = (uint64_t)(item - nti) * HC;
                    pushHubChunk<NT>(a, sm, e0, min(e0 + HC, HE), H, qc, cur);
                }
            }
            if (!batchBarrier<NT>(a, sm, cur)) return;
            // phase B: fold the candidates' pushed bits
            const uint32_t C = (uint32_t)sm.cnt[6];
            for (uint64_t base = (uint64_t)blockIdx.x * NT; base < C; base += gthreads) {
                const uint64_t i = base + tid;
                unsigned long long b = 0;
                uint32_t v = 0, st = 0, d = 0;
                if (i < C) {
                    v = a.cq[i];
                    const unsigned long long old = a.seen[v];
                    b = a.nx[v] & ~old;
                    a.nx[v] = 0;
                    if (b) {
                        st = a.row_ptr[v];
                        d = a.row_ptr[v + 1] - st;
                        a.fr[nq][v] = b;
                        foldBits(a, v, old, b, d, acc);
                        unsigned long long bb = b;
                        while (bb) {
                            const int s = __ffsll((long long)bb) - 1;
                            bb &= bb - 1;
                            a.dist[(uint64_t)s * a.n + v] = level + 1;
                        }
                    }
                }
                appendActive<NT>(a, sm, b != 0, v, st, d, nq, cur);
            }
        }
        // counters: one atomic per block and counter
        unsigned long long vals[6] = {acc.found, acc.aedges, acc.bits, acc.fullEdges, acc.fullCount, acc.exam};
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            const unsigned long long x = warpSum(vals[i]);
            if (laneId() == 0 && x) atomicAdd(&sm.acc[i], x);
        }
        __syncthreads();
        if (tid == 0) {
            if (sm.acc[0]) atomicAdd(&cur->found, sm.acc[0]);
            if (sm.acc[1]) atomicAdd(&cur->aedges, sm.acc[1]);
            if (sm.acc[2]) atomicAdd(&cur->bits, sm.acc[2]);
            if (sm.acc[3]) atomicAdd(&cur->fullEdges, sm.acc[3]);
            if (sm.acc[4]) atomicAdd(&cur->fullCount, sm.acc[4]);
            if (sm.acc[5]) atomicAdd(&cur->examined, sm.acc[5]);
        }
        if (!batchBarrier<NT>(a, sm, cur)) return;
        if (gtid == 0) {
            const uint64_t t = globaltimer();
            if (a.trace && level < a.traceCap) a.trace[level].time_ms = (double)(t - tPrev) * 1e-6;
            tPrev = t;
        }
        const uint64_t found = sm.cnt[0], nextE = sm.cnt[1];
        fullEdges += sm.cnt[2];
        fullCount += sm.cnt[3];
        q2Count = qCount;
        q2Hub = qHub;
        qCount = (uint32_t)sm.cnt[4];
        qHub = sm.cnt[5];
        if (bottomUp) {
            if (!(found >= size || (double)found > (double)a.n / a.beta)) {
                bottomUp = false;
                scout = 1;
            }
        } else {
            scout = nextE;
        }
        size = found;
        fedges = nextE;
        lastStrat = strat;
        ++level;
    }
    // epilogue: depths of the (vertex, source) pairs never reached
    for (uint64_t base = (uint64_t)blockIdx.x * NT; base < a.n; base += gthreads) {
        const uint64_t v = base + tid;
        const unsigned long long miss = v < a.n ? (a.all & ~a.seen[v]) : 0ull;
        writeDepths(a, v, miss, kInf);
    }
    if (gtid == 0) {
        if (a.trace && level > 0 && level - 1 < a.traceCap && lastStrat == GB_STRAT_BU)
            a.trace[level - 1].edges = ldv64(&a.ctr[(level + 3) & 3].examined);
        a.ctl[2] = level;
    }
}

}  // namespace
}  // namespace gb

using namespace gb;

void gb_bfs::ensureBatch(const gb_bfs_options& o, int k) {
    const int block = o.block ? (int)o.block : 512;
    const uint64_t hubCap = std::min<uint64_t>(n, m / 32 + 1);
    bSeen.ensure(n);
    bNext.ensure(n);
    for (int i = 0; i < 2; ++i) {
        bFront[i].ensure(n);
        bActive[i].ensure(3 * n);  // vertex | start | degree
        bHubV[i].ensure(2 * hubCap);  // vertex | start
        bHubOff[i].ensure(hubCap);
    }
    bCand.ensure(n);
    bDefer.ensure(n);
    bDist.ensure((uint64_t)k * n + 4);
    pctl.ensure(4);
    ptrace.ensure(kTraceCap);
    if (bBlock != block) {
        int perSm = 0;
        if (block == 256)
            GB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, batchBfsKernel<256>, 256, 0));
        else
            GB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, batchBfsKernel<512>, 512, 0));
        if (perSm < 1) throw Error(GB_ERR_CUDA, "batched BFS kernel cannot be resident");
        bMax = perSm * deviceSmCount();
        bBlock = block;
    }
    bGrid = o.grid_blocks > 0 ? std::min<int>((int)o.grid_blocks, bMax) : bMax;
}

// gb_bfs_run_many for the batched kernel: one launch per group of up to 64
// sources, then every row of the group returned to the host as the single-
// source path does (packed to the width the batch's level count allows,
// copied on the copy stream, widened by host threads) through a ring of
// kRowRing buffers, so row j + 1's pack and copy overlap row j's widening.
// The pack kernel checks every depth against the width; a row that does not
// fit is copied whole.  gpu_ms[i]: the group's launch time shared evenly over
// its sources; levels[i]: the group's level count.  Without out the last
// source's depths are left in the handle's depth buffer.
void gb_bfs::runBatchMany(const uint32_t* src, uint32_t count, uint32_t* out, uint64_t stride,
                          const gb_bfs_options& o, float* msOut, uint32_t* levelsOut) {
    constexpr uint32_t kRowRing = 4;
    static_assert(kRowRing <= kManySlots, "row ring exceeds the handle's pack buffers");
    validateOptions(o);
    if (count == 0) return;
    if (out)
        for (uint32_t b = 0; b < kRowRing; ++b) {
            mPackDev[b].ensure(2 * n + 16);
            mPackHost[b].ensure(2 * n + 16);
        }
    mFlag.ensure(kManySlots);
    mFlagHost.ensure(64);
    while (mSlotEv.size() < 3 * (size_t)kManySlots + 1 + kMaxInFlight) {
        cudaEvent_t e;
        GB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        mSlotEv.push_back(e);
    }
    cudaStream_t cs = copyStream.s;
    for (uint32_t g0 = 0; g0 < count; g0 += 64) {
        const uint32_t k = std::min<uint32_t>(64, count - g0);
        runBatch(src + g0, (int)k, o, nullptr);  // returns with the launch finished
        for (uint32_t j = 0; j < k; ++j) {
            if (msOut) msOut[g0 + j] = (float)(lastGpuMs / k);
            if (levelsOut) levelsOut[g0 + j] = lastLevels;
        }
        if (!out) {
            if (g0 + k == count)
                GB_CUDA(cudaMemcpyAsync(dist.get(), bDist.get() + (uint64_t)(k - 1) * n, n * 4,
                                        cudaMemcpyDeviceToDevice, stream.s));
            continue;
        }
        const int fmt = packFormat(n, lastLevels);
        if (fmt < 0) {
            for (uint32_t j = 0; j < k; ++j)
                GB_CUDA(cudaMemcpyAsync(out + (uint64_t)(g0 + j) * stride, bDist.get() + (uint64_t)j * n, n * 4,
                                        cudaMemcpyDeviceToHost, stream.s));
            GB_CUDA(cudaStreamSynchronize(stream.s));
            continue;
        }
        auto enqueue = [&](uint32_t j) {
            const uint32_t b = j % kRowRing;
            cudaEvent_t packed = mSlotEv[b], copied = mSlotEv[kManySlots + b];
            GB_CUDA(cudaMemsetAsync(mFlag.get() + b, 0, sizeof(unsigned), stream.s));
            enqueuePack(fmt, bDist.get() + (uint64_t)j * n, n, mPackDev[b].get(), mFlag.get() + b, stream.s);
            GB_CUDA(cudaEventRecord(packed, stream.s));
            GB_CUDA(cudaStreamWaitEvent(cs, packed, 0));
            GB_CUDA(cudaMemcpyAsync(mPackHost[b].p, mPackDev[b].get(), packedBytes(fmt, n), cudaMemcpyDeviceToHost,
                                    cs));
            GB_CUDA(cudaMemcpyAsync(mFlagHost.p + j, mFlag.get() + b, sizeof(unsigned), cudaMemcpyDeviceToHost, cs));
            GB_CUDA(cudaEventRecord(copied, cs));
        };
        // buffer b is packed again only after the host has widened its last
        // row (the host enqueues row j + kRowRing after widening row j)
        uint32_t queued = 0;
        for (; queued < k && queued < kRowRing; ++queued) enqueue(queued);
        for (uint32_t j = 0; j < k; ++j) {
            const uint32_t b = j % kRowRing;
            GB_CUDA(cudaEventSynchronize(mSlotEv[kManySlots + b]));
            uint32_t* dst = out + (uint64_t)(g0 + j) * stride;
            if (mFlagHost.p[j] == 0) {
                widenPacked(fmt, mPackHost[b].p, n, dst);
            } else {  // a depth did not fit the width: the row is still intact on the device
                GB_CUDA(cudaMemcpyAsync(dst, bDist.get() + (uint64_t)j * n, n * 4, cudaMemcpyDeviceToHost, cs));
                GB_CUDA(cudaStreamSynchronize(cs));
            }
            if (queued < k) enqueue(queued++);
        }
    }
    GB_CUDA(cudaStreamSynchronize(stream.s));
    GB_CUDA(cudaStreamSynchronize(cs));
}

void gb_bfs::runBatch(const uint32_t* src, int k, const gb_bfs_options& o, std::vector<gb_level>* tr) {
    validateOptions(o);
    if (k < 1 || k > 64) throw Error(GB_ERR_ARG, "batched BFS takes 1 to 64 sources");
    for (int i = 0; i < k; ++i)
        if (src[i] >= n) throw Error(GB_ERR_ARG, "source out of range");
    if (o.selector == GB_SELECT_LEARNED && !selLoaded[1])
        throw Error(GB_ERR_STATE, "learned batched selector requested but no parameters are loaded");
    ensureBatch(o, k);
    DevBuf<BCounters> ctr;
    ctr.ensure(4);
    DevBuf<uint32_t> dsrc;
    dsrc.ensure(64);
    hstage.ensure(64);
    std::memcpy(hstage.p, src, k * 4);
    GB_CUDA(cudaMemcpyAsync(dsrc.get(), hstage.p, k * 4, cudaMemcpyHostToDevice, stream.s));
    BArgs a{};
    a.row_ptr = rowPtr.get();
    a.col_idx = colIdx.get();
    a.seen = bSeen.get();
    a.nx = bNext.get();
    for (int i = 0; i < 2; ++i) {
        a.fr[i] = bFront[i].get();
        a.qv[i] = bActive[i].get();
        a.qs[i] = bActive[i].get() + n;
        a.qd[i] = bActive[i].get() + 2 * n;
        const uint64_t hubCap = std::min<uint64_t>(n, m / 32 + 1);
        a.hv[i] = bHubV[i].get();
        a.hs[i] = bHubV[i].get() + hubCap;
        a.ho[i] = bHubOff[i].get();
    }
    a.cq = bCand.get();
    a.dq = bDefer.get();
    a.dist = bDist.get();
    a.sources = dsrc.get();
    a.ctr = ctr.get();
    a.ctl = pctl.get();
    a.trace = ptrace.get();
    a.sel = selLoaded[1] ? selParams[1].get() : nullptr;
    a.n = n;
    a.m = m;
    a.all = k == 64 ? ~0ull : ((1ull << k) - 1);
    a.k = k;
    a.hubMin = std::max<uint32_t>(o.hub_min, 32);
    a.traceCap = kTraceCap;
    a.alpha = o.alpha;
    a.selMargin = o.sel_margin;
    a.beta = o.beta;
    a.selector = (int)o.selector;
    a.force = o.force_strategy;
    a.spinLimit = o.spin_limit ? o.spin_limit : (1ull << 24);
    GB_CUDA(cudaMemsetAsync(pctl.get(), 0, 4 * sizeof(unsigned), stream.s));
    GB_CUDA(cudaEventRecord(ev.a, stream.s));
    void* args[] = {&a};
    if (bBlock == 256)
        GB_CUDA(cudaLaunchCooperativeKernel((void*)batchBfsKernel<256>, dim3(bGrid), dim3(256), args, 0, stream.s));
    else
        GB_CUDA(cudaLaunchCooperativeKernel((void*)batchBfsKernel<512>, dim3(bGrid), dim3(512), args, 0, stream.s));
    GB_CUDA(cudaEventRecord(ev.b, stream.s));
    unsigned ctl[4];
    GB_CUDA(cudaMemcpyAsync(ctl, pctl.get(), sizeof ctl, cudaMemcpyDeviceToHost, stream.s));
    GB_CUDA(cudaStreamSynchronize(stream.s));
    lastGpuMs = ev.ms();
    lastLevels = ctl[2];
    if (ctl[1]) throw Error(GB_ERR_TIMEOUT, "batched BFS: grid barrier wait exceeded its spin limit");
    if (tr) {
        const uint32_t kk = std::min<uint32_t>(ctl[2], kTraceCap);
        std::vector<gb_level> t(kk);
        if (kk) GB_CUDA(cudaMemcpy(t.data(), ptrace.get(), kk * sizeof(gb_level), cudaMemcpyDeviceToHost));
        for (auto& r : t) r.pad = 0;
        tr->insert(tr->end(), t.begin(), t.end());
    }
}
