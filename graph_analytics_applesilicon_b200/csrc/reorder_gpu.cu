// reorder_gpu.cu -- vertex orderings on the GPU: the reference's
// reorder::compute "degree" and "rcm" (src/graph/reorder.cpp:27-100), with
// the same permutations, byte for byte.
//
// degree: one sort of (degree-descending, id) keys.
//
// rcm: the reference runs, per connected component, a Cuthill-McKee
// breadth-first pass from the component's first vertex in (degree, id) order,
// takes the first lowest-degree vertex of that pass's last level as the start
// of a second pass, appends the second pass's order, and reverses everything.
// In its breadth-first pass a vertex w of the next level is appended under the
// first vertex u of the current level (in level order) that sees it, and u's
// newly seen neighbours are appended sorted by (degree, id).  So the next
// level is the set of unvisited neighbours sorted by (position of the first
// parent, degree, id).  Here every component runs at once, level by level:
//   claim   atomicMin(claim[w], position of u) over the edges of the level;
//           the first claimer appends w to the next level (unordered);
//   order   one 64-bit key per new vertex, (claim << b) | rankDI[w], where
//           rankDI is w's rank in the global (degree, id) order; sorting the
//           keys gives the reference's level order, and because the level
//           list is grouped by component (components in the order of their
//           first vertex, by induction from level 0), so is the next one.
// Pass 1 records each vertex's level and visit index; per component the start
// of pass 2 is min (degree, visit index) over its last level.  Pass 2 records
// the visit order; a final stable sort of the visit order by component rank
// gives the concatenation of the components' orders, which is reversed into
// perm.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "bfs_device.cuh"
#include "capi_util.hpp"
#include "graph_prep.cuh"

namespace gb {
namespace {

constexpr uint32_t kNone = 0xFFFFFFFFu;

__global__ void degreeKeysKernel(const uint32_t* rp, uint64_t n, int b, bool descending, unsigned long long* keys) {
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t d = rp[v + 1] - rp[v];
        keys[v] = ((unsigned long long)(descending ? kNone - d : d) << b) | v;
    }
}

// order[i] = id of sorted key i; rank[order[i]] = i (rank may be null);
// perm[order[i]] = i (perm may be null).
__global__ void keysToOrderKernel(const unsigned long long* keys, uint64_t n, int b, uint32_t* order, uint32_t* rank,
                                  uint32_t* perm) {
    const unsigned long long mask = (1ull << b) - 1ull;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = (uint32_t)(keys[i] & mask);
        if (order) order[i] = v;
        if (rank) rank[v] = (uint32_t)i;
        if (perm) perm[v] = (uint32_t)i;
    }
}

// trig[root] = min rankDI over the component (trig preset to kNone).
__global__ void compTriggerKernel(uint64_t n, const uint32_t* parent, const uint32_t* rankDI, uint32_t* trig) {
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
        atomicMin(&trig[parent[v]], rankDI[v]);
}

// flag[rank of each component's first vertex] = 1 (flag zeroed).
__global__ void trigFlagKernel(uint64_t n, const uint32_t* parent, const uint32_t* trig, uint32_t* flag) {
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
        if (parent[v] == v) flag[trig[v]] = 1u;
}

// Level 0 of pass 1: the components' first vertices in component order.
__global__ void level0Kernel(uint64_t n, const uint32_t* flag, const uint32_t* crankOfRank, const uint32_t* byDegree,
                             uint32_t* cur) {
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (uint64_t)gridDim.x * blockDim.x)
        if (flag[r]) cur[crankOfRank[r]] = byDegree[r];
}

// Marks the level-0 vertices (component c's vertex is cur[c]).
__global__ void startLevelKernel(const uint32_t* cur, uint32_t C, uint8_t* vis, uint32_t* crank, uint32_t* lvl,
                                 uint32_t* vidx, uint32_t* visit) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < C; c += gridDim.x * blockDim.x) {
        const uint32_t w = cur[c];
        vis[w] = 1;
        crank[w] = c;
        if (lvl) lvl[w] = 0;
        vidx[w] = c;
        visit[c] = w;
    }
}

// A warp per vertex of the current level: claim its unvisited neighbours.
__global__ void claimKernel(const uint32_t* cur, uint32_t S, const uint32_t* rp, const uint32_t* ci,
                            const uint8_t* vis, uint32_t* claim, uint32_t* next, uint32_t* count) {
    const unsigned lane = threadIdx.x & 31;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < S; i += nw) {
        const uint32_t u = cur[i];
        for (uint32_t e = rp[u] + lane; e < rp[u + 1]; e += 32) {
            const uint32_t w = ci[e];
            if (vis[w]) continue;
            if (atomicMin(&claim[w], i) == kNone) next[atomicAdd(count, 1u)] = w;
        }
    }
}

// Keys of the new level; marks it visited and gives it its component and level.
__global__ void levelKeysKernel(const uint32_t* next, uint32_t K, const uint32_t* claim, const uint32_t* rankDI,
                                const uint32_t* cur, int b, uint8_t* vis, uint32_t* crank, uint32_t* lvl,
                                uint32_t level, unsigned long long* keys) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < K; j += gridDim.x * blockDim.x) {
        const uint32_t w = next[j], c = claim[w];
        keys[j] = ((unsigned long long)c << b) | rankDI[w];
        vis[w] = 1;
        crank[w] = crank[cur[c]];
        if (lvl) lvl[w] = level;
    }
}

// Sorted keys -> the ordered level, appended to the visit order.
__global__ void levelDecodeKernel(const unsigned long long* keys, uint32_t K, int b, const uint32_t* byDegree,
                                  uint32_t* next, uint32_t* visit, uint32_t offset, uint32_t* vidx) {
    const unsigned long long mask = (1ull << b) - 1ull;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < K; j += gridDim.x * blockDim.x) {
        const uint32_t w = byDegree[(uint32_t)(keys[j] & mask)];
        next[j] = w;
        visit[offset + j] = w;
        vidx[w] = offset + j;
    }
}

__global__ void lastLevelKernel(uint64_t n, const uint32_t* crank, const uint32_t* lvl, uint32_t* last) {
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
        atomicMax(&last[crank[v]], lvl[v]);
}

// best[c] = min (degree << 32 | visit index) over c's last level (best preset to ~0).
__global__ void startPickKernel(uint64_t n, const uint32_t* rp, const uint32_t* crank, const uint32_t* lvl,
                                const uint32_t* last, const uint32_t* vidx, unsigned long long* best) {
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t c = crank[v];
        if (lvl[v] != last[c]) continue;
        atomicMin(&best[c], ((unsigned long long)(rp[v + 1] - rp[v]) << 32) | vidx[v]);
    }
}

__global__ void startListKernel(const unsigned long long* best, uint32_t C, const uint32_t* visit1, uint32_t* cur) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < C; c += gridDim.x * blockDim.x)
        cur[c] = visit1[(uint32_t)(best[c] & 0xFFFFFFFFull)];
}

// keys[i] = (component rank of the i-th visited vertex << b) | i.
__global__ void finalKeysKernel(const uint32_t* visit, uint64_t n, const uint32_t* crank, int b,
                                unsigned long long* keys) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        keys[i] = ((unsigned long long)crank[visit[i]] << b) | i;
}

// perm[visit[i of sorted key j]] = n - 1 - j (the reversal).
__global__ void finalPermKernel(const unsigned long long* keys, uint64_t n, int b, const uint32_t* visit,
                                uint32_t* perm) {
    const unsigned long long mask = (1ull << b) - 1ull;
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x)
        perm[visit[(uint32_t)(keys[j] & mask)]] = (uint32_t)(n - 1 - j);
}

// Levels of at most kSmallCap vertices run many at a time in one block
// (graphs of long, narrow traversals such as road grids have thousands of
// them), with no host round trip in between and the level's working arrays in
// shared memory.  Per level: one claim sweep balanced over the level's edges;
// then the new vertices are counted per parent, scattered to their parent's
// segment (an exclusive scan of the counts) and each segment is sorted by
// (degree, id) rank with an insertion sort -- segments are a vertex's newly
// seen neighbours, a handful in such graphs.  A level whose largest segment
// exceeds kSegmentSort is sorted whole by a bitonic network instead.
constexpr int kSmallThreads = 1024;
constexpr uint32_t kSmallCap = 4096;
constexpr uint32_t kPerThread = kSmallCap / kSmallThreads;  // level entries per thread
constexpr uint32_t kSegmentSort = 32;
constexpr uint32_t kSmallLevelsPerLaunch = 1u << 14;  // bounds one launch's duration
constexpr size_t kSmallSmem = 6 * kSmallCap * sizeof(uint32_t);
enum : uint32_t { kSmallDone = 1, kSmallBig = 2, kSmallBad = 3, kSmallMore = 4 };

struct SmallState {
    uint32_t S, K, level, status;
    unsigned long long offset;
};

// The level vertex owning edge e of the level: the last i with pre[i] <= e.
__device__ __forceinline__ uint32_t edgeOwner(const uint32_t* pre, uint32_t S, uint32_t e) {
    uint32_t lo = 0, hi = S - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= e) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// cur (size st->S) holds the current level in order; next receives the
// claimed vertices of the following level.  Stops when a pass ends (status
// done), when a level has more than kSmallCap vertices (status big: next
// holds its K claimed vertices, not yet keyed; the host continues from there)
// or after kSmallLevelsPerLaunch levels (status more: relaunch).
__global__ void __launch_bounds__(kSmallThreads) smallLevelsKernel(
    uint32_t* cur, uint32_t* next, const uint32_t* rp, const uint32_t* ci, uint8_t* vis, uint32_t* claim,
    const uint32_t* rankDI, const uint32_t* byDegree, uint32_t* crank, uint32_t* lvl, uint32_t* vidx, uint32_t* visit,
    int b, uint64_t n, SmallState* st) {
    extern __shared__ __align__(16) uint32_t smem[];
    uint32_t* pre = smem;                      // degree prefix of the level
    uint32_t* row = pre + kSmallCap;           // rp[] of the level's vertices
    uint32_t* curS = row + kSmallCap;          // the level, in order
    uint32_t* cnt = curS + kSmallCap;          // children per parent
    uint32_t* off = cnt + kSmallCap;           // segment cursor per parent
    uint32_t* vals = off + kSmallCap;          // ranks, scattered by parent
    unsigned long long* keys = reinterpret_cast<unsigned long long*>(cnt);  // bitonic path (cnt + off)
    __shared__ uint32_t scan[kSmallThreads / 32 + 1];
    __shared__ uint32_t count, maxSeg;
    const unsigned tid = threadIdx.x;
    const unsigned long long mask = (1ull << b) - 1ull;
    uint32_t S = st->S, level = st->level;
    unsigned long long offset = st->offset;
    for (uint32_t j = tid; j < S; j += kSmallThreads) curS[j] = cur[j];
    auto stop = [&](uint32_t status, uint32_t K) {
        if (tid == 0) {
            st->S = S;
            st->K = K;
            st->level = level;
            st->offset = offset;
            st->status = status;
        }
    };
    __syncthreads();
    for (uint32_t done = 0;; ++done) {
        if (done == kSmallLevelsPerLaunch) {
            for (uint32_t j = tid; j < S; j += kSmallThreads) cur[j] = curS[j];  // relaunched from cur
            stop(kSmallMore, 0);
            return;
        }
        // degree prefix and row starts of the level (kPerThread vertices per thread)
        uint32_t d[kPerThread], sum = 0;
#pragma unroll
        for (uint32_t q = 0; q < kPerThread; ++q) {
            const uint32_t i = tid * kPerThread + q;
            d[q] = 0;
            if (i < S) {
                const uint32_t u = curS[i], r0 = rp[u];
                row[i] = r0;
                d[q] = rp[u + 1] - r0;
            }
            sum += d[q];
        }
        if (tid == 0) {
            count = 0;
            maxSeg = 0;
        }
        uint32_t E;
        uint32_t run = blockScan<kSmallThreads>(sum, &E, scan);
#pragma unroll
        for (uint32_t q = 0; q < kPerThread; ++q) {
            const uint32_t i = tid * kPerThread + q;
            if (i < S) {
                pre[i] = run;
                cnt[i] = 0;
            }
            run += d[q];
        }
        __syncthreads();
        // claim sweep
        for (uint32_t e = tid; e < E; e += kSmallThreads) {
            const uint32_t i = edgeOwner(pre, S, e);
            const uint32_t w = ci[row[i] + (e - pre[i])];
            if (vis[w]) continue;
            if (atomicMin(&claim[w], i) == kNone) next[atomicAdd(&count, 1u)] = w;
        }
        __syncthreads();
        const uint32_t K = count;
        if (K == 0 || K > kSmallCap || offset + K > n) {
            for (uint32_t j = tid; j < S; j += kSmallThreads) cur[j] = curS[j];  // the host continues from cur
            stop(K == 0 ? kSmallDone : (offset + K > n ? kSmallBad : kSmallBig), K);
            return;
        }
        // each new vertex: its parent (final claim; ld.cg past L1), its rank;
        // it joins the visited set and inherits its parent's component
        uint32_t pc[kPerThread], pr[kPerThread];
#pragma unroll
        for (uint32_t q = 0; q < kPerThread; ++q) {
            const uint32_t j = tid + q * kSmallThreads;
            if (j < K) {
                const uint32_t w = next[j], c = __ldcg(&claim[w]);
                pc[q] = c;
                pr[q] = rankDI[w];
                vis[w] = 1;
                crank[w] = crank[curS[c]];
                if (lvl) lvl[w] = level;
                atomicAdd(&cnt[c], 1u);
            }
        }
        __syncthreads();
        // segment starts: exclusive scan of the per-parent counts
        uint32_t c4[kPerThread], csum = 0, cmax = 0;
#pragma unroll
        for (uint32_t q = 0; q < kPerThread; ++q) {
            const uint32_t i = tid * kPerThread + q;
            c4[q] = i < S ? cnt[i] : 0u;
            csum += c4[q];
            cmax = max(cmax, c4[q]);
        }
        if (cmax) atomicMax(&maxSeg, cmax);
        uint32_t total;
        uint32_t at = blockScan<kSmallThreads>(csum, &total, scan);
#pragma unroll
        for (uint32_t q = 0; q < kPerThread; ++q) {
            const uint32_t i = tid * kPerThread + q;
            if (i < S) off[i] = at;
            at += c4[q];
        }
        __syncthreads();
        if (maxSeg <= kSegmentSort) {
#pragma unroll
            for (uint32_t q = 0; q < kPerThread; ++q) {
                const uint32_t j = tid + q * kSmallThreads;
                if (j < K) vals[atomicAdd(&off[pc[q]], 1u)] = pr[q];
            }
            __syncthreads();
            // off[i] is now the end of segment i; insertion-sort each segment
#pragma unroll
            for (uint32_t q = 0; q < kPerThread; ++q) {
                const uint32_t i = tid * kPerThread + q;
                if (i >= S) continue;
                const uint32_t hi = off[i], lo = hi - cnt[i];
                for (uint32_t x = lo + 1; x < hi; ++x) {
                    const uint32_t v = vals[x];
                    uint32_t y = x;
                    for (; y > lo && vals[y - 1] > v; --y) vals[y] = vals[y - 1];
                    vals[y] = v;
                }
            }
            __syncthreads();
            for (uint32_t j = tid; j < K; j += kSmallThreads) {
                const uint32_t w = byDegree[vals[j]];
                curS[j] = w;
                visit[offset + j] = w;
                vidx[w] = (uint32_t)(offset + j);
            }
        } else {
            // keys (parent, rank), padded to a power of two; bitonic network
            uint32_t P = 2;
            while (P < K) P <<= 1;
#pragma unroll
            for (uint32_t q = 0; q < kPerThread; ++q) {
                const uint32_t j = tid + q * kSmallThreads;
                if (j < P) keys[j] = j < K ? (((unsigned long long)pc[q] << b) | pr[q]) : ~0ull;
            }
            __syncthreads();
            for (uint32_t k = 2; k <= P; k <<= 1)
                for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                    for (uint32_t t = tid; t < P / 2; t += kSmallThreads) {
                        const uint32_t i = (t / j) * 2 * j + (t % j), x = i + j;
                        const unsigned long long a = keys[i], c = keys[x];
                        if ((a > c) == ((i & k) == 0)) {
                            keys[i] = c;
                            keys[x] = a;
                        }
                    }
                    __syncthreads();
                }
            for (uint32_t j = tid; j < K; j += kSmallThreads) {
                const uint32_t w = byDegree[(uint32_t)(keys[j] & mask)];
                curS[j] = w;
                visit[offset + j] = w;
                vidx[w] = (uint32_t)(offset + j);
            }
        }
        __syncthreads();
        offset += K;
        S = K;
        ++level;
    }
}

struct Rcm {
    uint64_t n;
    int b;
    cudaStream_t st;
    const uint32_t *rp, *ci;
    ScanScratch sc;
    DevBuf<uint32_t> byDegree, rankDI, claim, crank, lvl, vidx, visit1, visit2, cur, next, count, counts;
    DevBuf<uint8_t> vis;
    DevBuf<unsigned long long> keys, tmp;
    DevBuf<SmallState> small;

    // One Cuthill-McKee pass over every component from the C vertices in
    // cur (component order); visit gets the order, lvl (if given) the level.
    void pass(uint32_t C, uint32_t* visit, uint32_t* lvlOut) {
        GB_CUDA(cudaMemsetAsync(vis.get(), 0, n, st));
        GB_CUDA(cudaMemsetAsync(claim.get(), 0xFF, n * 4, st));
        startLevelKernel<<<prepGrid(C, 256), 256, 0, st>>>(cur.get(), C, vis.get(), crank.get(), lvlOut, vidx.get(),
                                                           visit);
        GB_LAUNCH_CHECK();
        uint32_t S = C, level = 1;
        uint64_t offset = C;
        uint32_t* a = cur.get();
        uint32_t* z = next.get();
        while (S > 0) {
            uint32_t K = 0;
            if (S <= kSmallCap) {  // run levels in one block until one is large or the pass ends
                SmallState h{S, 0, level, 0, offset};
                GB_CUDA(cudaMemcpyAsync(small.get(), &h, sizeof h, cudaMemcpyHostToDevice, st));
                smallLevelsKernel<<<1, kSmallThreads, kSmallSmem, st>>>(a, z, rp, ci, vis.get(), claim.get(),
                                                                        rankDI.get(),
                                                               byDegree.get(), crank.get(), lvlOut, vidx.get(), visit,
                                                               b, n, small.get());
                GB_LAUNCH_CHECK();
                GB_CUDA(cudaMemcpyAsync(&h, small.get(), sizeof h, cudaMemcpyDeviceToHost, st));
                GB_CUDA(cudaStreamSynchronize(st));
                if (h.status == kSmallBad) throw Error(GB_ERR_STATE, "rcm: visited more vertices than the graph has");
                S = h.S;
                level = h.level;
                offset = h.offset;
                if (h.status == kSmallDone) break;
                if (h.status == kSmallMore) continue;
                K = h.K;  // a large level: its vertices are claimed and listed in z
            } else {
                GB_CUDA(cudaMemsetAsync(count.get(), 0, 4, st));
                claimKernel<<<prepGrid((uint64_t)S * 32, 256), 256, 0, st>>>(a, S, rp, ci, vis.get(), claim.get(),
                                                                             z, count.get());
                GB_LAUNCH_CHECK();
                GB_CUDA(cudaMemcpyAsync(&K, count.get(), 4, cudaMemcpyDeviceToHost, st));
                GB_CUDA(cudaStreamSynchronize(st));
                if (K == 0) break;
            }
            if (offset + K > n) throw Error(GB_ERR_STATE, "rcm: visited more vertices than the graph has");
            const int cb = keyBits(S);
            levelKeysKernel<<<prepGrid(K, 256), 256, 0, st>>>(z, K, claim.get(), rankDI.get(), a, b, vis.get(),
                                                              crank.get(), lvlOut, level, keys.get());
            GB_LAUNCH_CHECK();
            radixSortKeys(keys, tmp, K, cb + b, sc, st, &counts);
            levelDecodeKernel<<<prepGrid(K, 256), 256, 0, st>>>(keys.get(), K, b, byDegree.get(), z, visit,
                                                                (uint32_t)offset, vidx.get());
            GB_LAUNCH_CHECK();
            offset += K;
            S = K;
            ++level;
            std::swap(a, z);
        }
        if (offset != n) throw Error(GB_ERR_STATE, "rcm: a pass did not visit every vertex");
    }
};

// perm[old] = new for "degree" (descending degree, ties by id).
void degreeOrder(const gb_csr* g, uint32_t* permHost) {
    Stream st;
    ScanScratch sc;
    DevBuf<uint32_t> rp, ci, perm;
    uploadCheckedCsr(g, rp, ci, st.s);
    const uint64_t n = g->n;
    const int b = keyBits(n);
    DevBuf<unsigned long long> keys, tmp;
    keys.ensure(n);
    perm.ensure(n);
    degreeKeysKernel<<<prepGrid(n, 256), 256, 0, st.s>>>(rp.get(), n, b, true, keys.get());
    GB_LAUNCH_CHECK();
    radixSortKeys(keys, tmp, n, 32 + b, sc, st.s);
    keysToOrderKernel<<<prepGrid(n, 256), 256, 0, st.s>>>(keys.get(), n, b, nullptr, nullptr, perm.get());
    GB_LAUNCH_CHECK();
    GB_CUDA(cudaMemcpyAsync(permHost, perm.get(), n * 4, cudaMemcpyDeviceToHost, st.s));
    GB_CUDA(cudaStreamSynchronize(st.s));
}

void rcmOrder(const gb_csr* g, uint32_t* permHost) {
    Stream st;
    DevBuf<uint32_t> drp, dci;
    uploadCheckedCsr(g, drp, dci, st.s);
    Rcm R;
    R.n = g->n;
    R.b = keyBits(g->n);
    R.st = st.s;
    R.rp = drp.get();
    R.ci = dci.get();
    const uint64_t n = R.n;
    const int b = R.b;
    for (DevBuf<uint32_t>* a : {&R.byDegree, &R.rankDI, &R.claim, &R.crank, &R.lvl, &R.vidx, &R.visit1, &R.visit2})
        a->ensure(n);
    R.cur.ensure(n);
    R.next.ensure(n);
    GB_CUDA(cudaFuncSetAttribute(smallLevelsKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmallSmem));
    R.count.ensure(1);
    R.small.ensure(1);
    R.vis.ensure(n);
    R.keys.ensure(n);
    // the global (degree, id) order and each vertex's rank in it
    degreeKeysKernel<<<prepGrid(n, 256), 256, 0, st.s>>>(R.rp, n, b, false, R.keys.get());
    GB_LAUNCH_CHECK();
    radixSortKeys(R.keys, R.tmp, n, 32 + b, R.sc, st.s, &R.counts);
    keysToOrderKernel<<<prepGrid(n, 256), 256, 0, st.s>>>(R.keys.get(), n, b, R.byDegree.get(), R.rankDI.get(),
                                                          nullptr);
    GB_LAUNCH_CHECK();
    // components, ordered by their first vertex in (degree, id) order
    {
        DevBuf<uint32_t> parent, trig, flag, total;
        parent.ensure(n);
        trig.ensure(n);
        flag.ensure(n + 1);
        total.ensure(1);
        connectedComponents(R.rp, R.ci, n, parent.get(), st.s);
        GB_CUDA(cudaMemsetAsync(trig.get(), 0xFF, n * 4, st.s));
        GB_CUDA(cudaMemsetAsync(flag.get(), 0, (n + 1) * 4, st.s));
        compTriggerKernel<<<prepGrid(n, 256), 256, 0, st.s>>>(n, parent.get(), R.rankDI.get(), trig.get());
        trigFlagKernel<<<prepGrid(n, 256), 256, 0, st.s>>>(n, parent.get(), trig.get(), flag.get());
        GB_LAUNCH_CHECK();
        scanExclusive(flag.get(), trig.get(), n, total.get(), R.sc, st.s);  // trig now: component rank by rank
        uint32_t C = 0;
        GB_CUDA(cudaMemcpyAsync(&C, total.get(), 4, cudaMemcpyDeviceToHost, st.s));
        level0Kernel<<<prepGrid(n, 256), 256, 0, st.s>>>(n, flag.get(), trig.get(), R.byDegree.get(), R.cur.get());
        GB_LAUNCH_CHECK();
        GB_CUDA(cudaStreamSynchronize(st.s));
        // pass 1 (probe) -> the start of each component's pass 2
        R.pass(C, R.visit1.get(), R.lvl.get());
        DevBuf<uint32_t> last;
        DevBuf<unsigned long long> best;
        last.ensure(C);
        best.ensure(C);
        GB_CUDA(cudaMemsetAsync(last.get(), 0, (uint64_t)C * 4, st.s));
        GB_CUDA(cudaMemsetAsync(best.get(), 0xFF, (uint64_t)C * 8, st.s));
        lastLevelKernel<<<prepGrid(n, 256), 256, 0, st.s>>>(n, R.crank.get(), R.lvl.get(), last.get());
        startPickKernel<<<prepGrid(n, 256), 256, 0, st.s>>>(n, R.rp, R.crank.get(), R.lvl.get(), last.get(),
                                                            R.vidx.get(), best.get());
        startListKernel<<<prepGrid(C, 256), 256, 0, st.s>>>(best.get(), C, R.visit1.get(), R.cur.get());
        GB_LAUNCH_CHECK();
        // pass 2, then the components' orders concatenated and reversed
        R.pass(C, R.visit2.get(), nullptr);
        const int cb = keyBits(C);
        finalKeysKernel<<<prepGrid(n, 256), 256, 0, st.s>>>(R.visit2.get(), n, R.crank.get(), b, R.keys.get());
        GB_LAUNCH_CHECK();
        radixSortKeys(R.keys, R.tmp, n, cb + b, R.sc, st.s, &R.counts);
        finalPermKernel<<<prepGrid(n, 256), 256, 0, st.s>>>(R.keys.get(), n, b, R.visit2.get(), R.next.get());
        GB_LAUNCH_CHECK();
    }
    GB_CUDA(cudaMemcpyAsync(permHost, R.next.get(), n * 4, cudaMemcpyDeviceToHost, st.s));
    GB_CUDA(cudaStreamSynchronize(st.s));
}

// key[i] = (row << b) | rank[ci[i]] for every entry (a warp per row).
__global__ void rowRankKeysKernel(const uint32_t* rp, const uint32_t* ci, uint64_t n, int b, const uint32_t* rank,
                                  unsigned long long* keys) {
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    for (uint64_t v = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += nw)
        for (uint32_t i = rp[v] + lane; i < rp[v + 1]; i += 32) keys[i] = (v << b) | rank[ci[i]];
}

__global__ void rowRankDecodeKernel(const unsigned long long* keys, uint64_t m, int b, const uint32_t* order,
                                    uint32_t* ci) {
    const unsigned long long mask = (1ull << b) - 1ull;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x)
        ci[i] = order[(uint32_t)(keys[i] & mask)];
}

}  // namespace

void hubFirstAdjacency(const uint32_t* rp, uint32_t* ci, uint64_t n, uint64_t m, cudaStream_t st) {
    if (m < 2) return;
    const int b = keyBits(n);
    ScanScratch sc;
    DevBuf<uint32_t> order, rank, counts;
    DevBuf<unsigned long long> keys, tmp;
    order.ensure(n);
    rank.ensure(n);
    keys.ensure(std::max<uint64_t>(n, m));
    degreeKeysKernel<<<prepGrid(n, 256), 256, 0, st>>>(rp, n, b, true, keys.get());
    GB_LAUNCH_CHECK();
    radixSortKeys(keys, tmp, n, 32 + b, sc, st, &counts);
    keysToOrderKernel<<<prepGrid(n, 256), 256, 0, st>>>(keys.get(), n, b, order.get(), rank.get(), nullptr);
    GB_LAUNCH_CHECK();
    rowRankKeysKernel<<<prepGrid(n * 32, 256), 256, 0, st>>>(rp, ci, n, b, rank.get(), keys.get());
    GB_LAUNCH_CHECK();
    radixSortKeys(keys, tmp, m, 2 * b, sc, st, &counts);
    rowRankDecodeKernel<<<prepGrid(m, 256), 256, 0, st>>>(keys.get(), m, b, order.get(), ci);
    GB_LAUNCH_CHECK();
    GB_CUDA(cudaStreamSynchronize(st));
}

}  // namespace gb

using namespace gb;

extern "C" {

int gb_csr_hub_first_gpu(const gb_csr* g, gb_csr* out) {
    return guard([&] {
        GB_REQUIRE(g && out, "null argument");
        Stream st;
        DevBuf<uint32_t> rp, ci;
        uploadCheckedCsr(g, rp, ci, st.s);
        hubFirstAdjacency(rp.get(), ci.get(), g->n, g->m, st.s);
        uint32_t* hrp = static_cast<uint32_t*>(std::malloc((g->n + 1) * 4));
        uint32_t* hci = static_cast<uint32_t*>(std::malloc(std::max<uint64_t>(g->m, 1) * 4));
        if (!hrp || !hci) {
            std::free(hrp);
            std::free(hci);
            throw Error(GB_ERR_OOM, "host allocation failed");
        }
        std::memcpy(hrp, g->row_ptr, (g->n + 1) * 4);
        if (g->m) GB_CUDA(cudaMemcpy(hci, ci.get(), g->m * 4, cudaMemcpyDeviceToHost));
        out->n = g->n;
        out->m = g->m;
        out->flags = g->flags & ~2u;  // rows are no longer sorted by id
        out->row_ptr = hrp;
        out->col_idx = hci;
    });
}

int gb_reorder_gpu(const gb_csr* g, const char* ordering, uint64_t seed, uint32_t* perm) {
    return guard([&] {
        GB_REQUIRE(g && ordering && (perm || g->n == 0), "null argument");
        const std::string o = ordering;
        if (o == "original" || o == "random" || g->n == 0) {
            const int rc = gb_reorder(g, ordering, seed, perm);  // host: identity / seeded Fisher-Yates
            if (rc != GB_OK) throw Error((gb_status)rc, gb_last_error());
            return;
        }
        GB_REQUIRE(!(g->flags & 1u), "gb_reorder_gpu: orderings are computed on a symmetric graph");
        if (o == "degree") degreeOrder(g, perm);
        else if (o == "rcm") rcmOrder(g, perm);
        else throw Error(GB_ERR_ARG, "unknown ordering '" + o + "' (original|random|degree|rcm)");
    });
}

}  // extern "C"
