// bfs_levels.cu -- the host-driven BFS forms: one launch sequence and one host
// synchronisation per level, as the reference's GpuBfs::run* loops
// (src/metal/bfs_gpu.mm:115-429).  They are the "plain" forms the persistent
// kernel is measured against, and the drop-in for gpu_vertex / gpu_naive /
// gpu_binned / gpu_edge / gpu_do.
//
// Kernels are new sm_100a code: warp-aggregated queue appends (__ballot_sync
// + one atomic per warp), CAS claims on dist, shared-memory staging of the
// scanned frontier degrees in the edge-balanced expansion, and bitmap
// frontiers with __ballot_sync word assembly in the bottom-up step.
#include <algorithm>
#include <chrono>

#include "bfs.hpp"

namespace gb {

uint32_t checkTg(uint32_t tg) {
    if (tg < 32 || tg > 1024 || tg % 32 != 0)
        throw Error(GB_ERR_ARG, "threadgroup size must be a multiple of 32 in [32, 1024]");
    return tg;
}

void validateOptions(const gb_bfs_options& o) {
    checkTg(o.tg);
    if (o.ept == 0) throw Error(GB_ERR_ARG, "ept must be >= 1");
    if (o.ept > 64) throw Error(GB_ERR_ARG, "ept must be <= 64");
    if (!(o.alpha > 0) || !(o.beta > 0)) throw Error(GB_ERR_ARG, "alpha and beta must be > 0");
    if (o.force_strategy >= GB_NUM_STRATS) throw Error(GB_ERR_ARG, "force_strategy out of range");
    if (o.block != 0 && o.block != 256 && o.block != 512)
        throw Error(GB_ERR_ARG, "persistent block size must be 256 or 512");
    if (o.selector > GB_SELECT_LEARNED) throw Error(GB_ERR_ARG, "unknown selector");
    if (o.in_flight > (uint32_t)kMaxInFlight)
        throw Error(GB_ERR_ARG, "in_flight must be at most " + std::to_string(kMaxInFlight));
}

namespace {

using Stats = GbLevelStats;

__device__ __forceinline__ bool claimDist(uint32_t* dist, uint32_t u, uint32_t value) {
    // Plain load first: skips the atomic for already-visited vertices.
    if (*reinterpret_cast<volatile uint32_t*>(&dist[u]) != kInf) return false;
    return atomicCAS(&dist[u], kInf, value) == kInf;
}

__device__ __forceinline__ void addStats(Stats* s, unsigned long long frontier, unsigned long long edges,
                                         unsigned long long nextEdges) {
    frontier = warpSum(frontier);
    edges = warpSum(edges);
    nextEdges = warpSum(nextEdges);
    if (laneId() == 0) {
        if (frontier) atomicAdd(&s->frontier, frontier);
        if (edges) atomicAdd(&s->edges, edges);
        if (nextEdges) atomicAdd(&s->nextEdges, nextEdges);
    }
}

__global__ void initDistKernel(uint32_t* dist, uint64_t n, uint32_t source) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t n4 = n / 4;
    uint4* d4 = reinterpret_cast<uint4*>(dist);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride)
        d4[i] = make_uint4(kInf, kInf, kInf, kInf);
    for (uint64_t i = n4 * 4 + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) dist[i] = kInf;
}

__global__ void setSourceKernel(uint32_t* dist, uint32_t source) { dist[source] = 0; }

// gpu_vertex: thread per vertex every level; plain stores (all writers store
// level + 1, readers only test for "unreached"), so `found` may overcount and
// is used only as "something changed" (src/shaders/bfs.metal:45-54).
__global__ void vertexLevelKernel(const uint32_t* row_ptr, const uint32_t* col_idx, uint32_t* dist, uint64_t n,
                                  uint32_t level, Stats* s) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    unsigned long long frontier = 0, edges = 0, found = 0;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        uint64_t v = base + threadIdx.x;
        if (v < n && dist[v] == level) {
            uint32_t b = row_ptr[v], e = row_ptr[v + 1];
            frontier++;
            edges += e - b;
            for (uint32_t i = b; i < e; ++i) {
                uint32_t u = col_idx[i];
                if (dist[u] == kInf) {
                    dist[u] = level + 1;
                    found++;
                }
            }
        }
    }
    found = warpSum(found);
    if (laneId() == 0 && found) atomicAdd(&s->found, (unsigned)min(found, 0xFFFFFFFFull));
    addStats(s, frontier, edges, 0);
}

// gpu_naive: thread per frontier vertex, CAS claim, one atomic append per claim.
__global__ void naiveLevelKernel(const uint32_t* row_ptr, const uint32_t* col_idx, uint32_t* dist, Stats* s,
                                 const uint32_t* queue, uint32_t* next, uint32_t size, uint32_t level) {
    unsigned long long frontier = 0, edges = 0;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < size) {
        uint32_t v = queue[i], b = row_ptr[v], e = row_ptr[v + 1];
        frontier = 1;
        edges = e - b;
        for (uint32_t k = b; k < e; ++k) {
            uint32_t u = col_idx[k];
            if (claimDist(dist, u, level + 1)) next[atomicAdd(&s->found, 1u)] = u;
        }
    }
    addStats(s, frontier, edges, 0);
}

// ----------------------------------------------------------- gpu_binned

struct BinArgs {
    const uint32_t* row_ptr;
    const uint32_t* col_idx;
    uint32_t* dist;
    Stats* s;
    const uint32_t* queue;
    uint32_t* q[3];
    uint32_t size, level, smallMax, largeMin;
};

// Discovery: claim u and append it to the next-level queue of its degree bin.
// Called by all 32 lanes together.
__device__ __forceinline__ void binVisit(const BinArgs& a, bool has, uint32_t e) {
    uint32_t u = has ? a.col_idx[e] : 0u;
    bool claimed = has && claimDist(a.dist, u, a.level + 1);
    if (!__any_sync(kFull, claimed)) return;
    uint32_t udeg = claimed ? a.row_ptr[u + 1] - a.row_ptr[u] : 0u;
    uint32_t bin = udeg < a.smallMax ? 0u : (udeg < a.largeMin ? 1u : 2u);
#pragma unroll
    for (int b = 0; b < 3; ++b) {
        bool want = claimed && bin == (uint32_t)b;
        if (!__any_sync(kFull, want)) continue;
        uint32_t pos = warpAppend(want, &a.s->bin[b]);
        if (want) a.q[b][pos] = u;
    }
    unsigned long long ne = warpSum((unsigned long long)udeg);
    if (laneId() == 0 && ne) atomicAdd(&a.s->nextEdges, ne);
}

// Small bin: the warp expands its 32 short lists together: lane j takes edge
// j of the lists' concatenation; the owner lane is found by a shuffle binary
// search over the lanes' exclusive degree prefix.
__global__ void binnedSmallKernel(BinArgs a) {
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned lane = laneId();
    bool active = gid < a.size;
    uint32_t v = active ? a.queue[gid] : 0u;
    uint32_t begin = active ? a.row_ptr[v] : 0u;
    uint32_t deg = active ? a.row_ptr[v + 1] - begin : 0u;
    uint32_t incl = deg;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(kFull, incl, o);
        if ((int)lane >= o) incl += y;
    }
    uint32_t pre = incl - deg, total = __shfl_sync(kFull, incl, 31);
    for (uint32_t base = 0; base < total; base += 32) {
        uint32_t j = base + lane;
        uint32_t owner = 0;
#pragma unroll
        for (uint32_t step = 16; step > 0; step >>= 1) {
            uint32_t cand = owner + step;
            if (__shfl_sync(kFull, pre, cand) <= j) owner = cand;
        }
        uint32_t ob = __shfl_sync(kFull, begin, owner), op = __shfl_sync(kFull, pre, owner);
        binVisit(a, j < total, ob + (j - op));
    }
}

// Medium bin: warp per vertex, lanes stride the list (coalesced col_idx).
__global__ void binnedMediumKernel(BinArgs a) {
    const uint32_t vi = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    if (vi >= a.size) return;  // uniform per warp
    uint32_t v = a.queue[vi], b = a.row_ptr[v], e = a.row_ptr[v + 1];
    for (uint32_t base = b; base < e; base += 32) binVisit(a, base + laneId() < e, base + laneId());
}

// Large bin: block per vertex.
__global__ void binnedLargeKernel(BinArgs a) {
    if (blockIdx.x >= a.size) return;
    uint32_t v = a.queue[blockIdx.x], b = a.row_ptr[v], e = a.row_ptr[v + 1];
    for (uint32_t base = b; base < e; base += blockDim.x) binVisit(a, base + threadIdx.x < e, base + threadIdx.x);
}

// ------------------------------------------------------------- gpu_edge

constexpr uint32_t kStageCap = 2048;

__device__ __forceinline__ uint32_t findOwner(const uint32_t* off, uint32_t lo, uint32_t hi, uint32_t e) {
    while (lo < hi) {  // largest i in [lo, hi] with off[i] <= e
        uint32_t mid = (lo + hi + 1) >> 1;
        if (off[mid] <= e) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Edge-balanced expansion: block b owns edges [b*chunk, (b+1)*chunk) of the
// level (chunk = blockDim * ept); thread t takes edges t, t+blockDim, ... so a
// warp reads 32 consecutive edges per round.  Thread 0 finds the chunk's
// owner range once; the range's scanned offsets and adjacency starts are
// staged in shared memory so every per-edge owner search runs there.
__global__ void edgeExpandKernel(const uint32_t* row_ptr, const uint32_t* col_idx, uint32_t* dist, Stats* s,
                                 const uint32_t* queue, const uint32_t* offsets, uint32_t* nextQ, uint32_t* nextDeg,
                                 uint32_t size, uint32_t total, uint32_t level, uint32_t ept) {
    __shared__ uint32_t sOff[kStageCap], sStart[kStageCap];
    __shared__ uint32_t sRange[2];
    const uint32_t chunk = blockDim.x * ept;
    const uint32_t c0 = blockIdx.x * chunk;
    const uint32_t c1 = min(c0 + chunk, total);
    if (threadIdx.x == 0) {
        uint32_t lo = findOwner(offsets, 0, size - 1, c0);
        sRange[0] = lo;
        sRange[1] = findOwner(offsets, lo, size - 1, c1 - 1);
    }
    __syncthreads();
    const uint32_t lo = sRange[0], hi = sRange[1], cnt = hi - lo + 1;
    const bool staged = cnt <= kStageCap;
    if (staged)
        for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x) {
            sOff[i] = offsets[lo + i];
            sStart[i] = row_ptr[queue[lo + i]];
        }
    __syncthreads();
    for (uint32_t k = 0; k < ept; ++k) {  // block-uniform rounds: appends stay convergent
        uint32_t e = c0 + k * blockDim.x + threadIdx.x;
        bool has = e < c1;
        uint32_t u = 0;
        if (has) {
            if (staged) {
                uint32_t i = findOwner(sOff, 0, cnt - 1, e);
                u = col_idx[sStart[i] + (e - sOff[i])];
            } else {
                uint32_t i = findOwner(offsets, lo, hi, e);
                u = col_idx[row_ptr[queue[i]] + (e - offsets[i])];
            }
        }
        bool claimed = has && claimDist(dist, u, level + 1);
        if (!__any_sync(kFull, claimed)) continue;
        uint32_t udeg = claimed ? row_ptr[u + 1] - row_ptr[u] : 0u;
        uint32_t pos = warpAppend(claimed, &s->found);
        if (claimed) {
            nextQ[pos] = u;
            nextDeg[pos] = udeg;
        }
        unsigned long long ne = warpSum((unsigned long long)udeg);
        if (laneId() == 0 && ne) atomicAdd(&s->nextEdges, ne);
    }
}

// ------------------------------------------------------------- bottom-up

// Thread per vertex: an unreached vertex scans its list for the first parent
// in the frontier bitmap (early exit).  The 32 lanes of a warp are one bitmap
// word of the next frontier, assembled with __ballot_sync and stored by lane
// 0, so every word of `next` is written and needs no clearing.
__global__ void bottomUpKernel(const uint32_t* row_ptr, const uint32_t* col_idx, uint32_t* dist,
                               const uint32_t* front, uint32_t* next, Stats* s, uint64_t n, uint32_t level) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    unsigned long long foundC = 0, examined = 0, ndeg = 0;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        const uint64_t v = base + threadIdx.x;
        bool found = false;
        if (v < n && dist[v] == kInf) {
            uint32_t b = row_ptr[v], e = row_ptr[v + 1];
            for (uint32_t i = b; i < e; ++i) {
                ++examined;
                uint32_t u = col_idx[i];
                if ((front[u >> 5] >> (u & 31)) & 1u) {
                    found = true;
                    break;
                }
            }
            if (found) {
                dist[v] = level + 1;
                ndeg += e - b;
                ++foundC;
            }
        }
        unsigned word = __ballot_sync(kFull, found);
        if (laneId() == 0 && v < n) next[v >> 5] = word;
    }
    foundC = warpSum(foundC);
    if (laneId() == 0 && foundC) atomicAdd(&s->found, (unsigned)foundC);
    addStats(s, 0, examined, ndeg);
}

uint32_t gridCap(uint64_t work, uint32_t threads) {
    uint64_t b = (work + threads - 1) / threads;
    uint64_t cap = (uint64_t)deviceSmCount() * (2048 / threads) * 4;
    return (uint32_t)std::max<uint64_t>(1, std::min(b, cap));
}

double msSince(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace
}  // namespace gb

using namespace gb;

void gb_bfs::initDist(uint32_t src) {
    initDistKernel<<<gridCap(n / 4 + 1, 256), 256, 0, stream.s>>>(dist.get(), n, src);
    setSourceKernel<<<1, 1, 0, stream.s>>>(dist.get(), src);
    GB_LAUNCH_CHECK();
}

void gb_bfs::beginLevel() {
    GB_CUDA(cudaMemsetAsync(stats.get(), 0, sizeof(GbLevelStats), stream.s));
}

void gb_bfs::endLevel() {
    GB_CUDA(cudaMemcpyAsync(hstats.p, stats.get(), sizeof(GbLevelStats), cudaMemcpyDeviceToHost, stream.s));
    GB_CUDA(cudaEventRecord(ev.b, stream.s));
    GB_CUDA(cudaStreamSynchronize(stream.s));
    lastGpuMs += ev.ms();
    ++lastLevels;
}

void gb_bfs::ensureEdgeBuffers() {
    qA.ensure(n);
    qB.ensure(n);
    degA.ensure(n);
    degB.ensure(n);
}

void gb_bfs::runVertex(uint32_t src, const gb_bfs_options& o, std::vector<gb_level>* tr) {
    const uint32_t tg = checkTg(o.tg);
    lastGpuMs = 0;
    lastLevels = 0;
    for (uint32_t level = 0;; ++level) {
        auto t0 = std::chrono::steady_clock::now();
        GB_CUDA(cudaEventRecord(ev.a, stream.s));
        beginLevel();
        if (level == 0) initDist(src);
        vertexLevelKernel<<<gridCap(n, tg), tg, 0, stream.s>>>(rowPtr.get(), colIdx.get(), dist.get(), n, level,
                                                               stats.get());
        GB_LAUNCH_CHECK();
        endLevel();
        const GbLevelStats& s = *hstats.p;
        if (tr) tr->push_back({level, 'T', 'G', 0, 0, s.frontier, s.edges, msSince(t0)});
        if (s.found == 0) break;
    }
}

void gb_bfs::runNaive(uint32_t src, const gb_bfs_options& o, std::vector<gb_level>* tr) {
    const uint32_t tg = checkTg(o.tg);
    qA.ensure(n);
    qB.ensure(n);
    uint32_t *cur = qA.get(), *next = qB.get();
    hstage.p[0] = src;
    GB_CUDA(cudaMemcpyAsync(cur, hstage.p, 4, cudaMemcpyHostToDevice, stream.s));
    uint32_t size = 1;
    lastGpuMs = 0;
    lastLevels = 0;
    for (uint32_t level = 0; size > 0; ++level) {
        auto t0 = std::chrono::steady_clock::now();
        GB_CUDA(cudaEventRecord(ev.a, stream.s));
        beginLevel();
        if (level == 0) initDist(src);
        naiveLevelKernel<<<divUp(size, tg), tg, 0, stream.s>>>(rowPtr.get(), colIdx.get(), dist.get(), stats.get(),
                                                               cur, next, size, level);
        GB_LAUNCH_CHECK();
        endLevel();
        const GbLevelStats& s = *hstats.p;
        if (tr) tr->push_back({level, 'T', 'G', 0, 0, s.frontier, s.edges, msSince(t0)});
        size = s.found;
        std::swap(cur, next);
    }
}

void gb_bfs::runBinned(uint32_t src, const gb_bfs_options& o, std::vector<gb_level>* tr) {
    const uint32_t tg = checkTg(o.tg);
    for (auto& set : bins)
        for (auto& q : set) q.ensure(n);
    auto bin = [&](uint32_t d) { return d < o.small_max ? 0 : (d < o.large_min ? 1 : 2); };
    uint32_t count[3] = {0, 0, 0};
    const uint32_t srcDeg = degree(src);
    hstage.p[0] = src;
    GB_CUDA(cudaMemcpyAsync(bins[0][bin(srcDeg)].get(), hstage.p, 4, cudaMemcpyHostToDevice, stream.s));
    count[bin(srcDeg)] = 1;
    uint64_t edges = srcDeg;
    int cur = 0;
    lastGpuMs = 0;
    lastLevels = 0;
    for (uint32_t level = 0; count[0] + count[1] + count[2] > 0; ++level) {
        auto t0 = std::chrono::steady_clock::now();
        GB_CUDA(cudaEventRecord(ev.a, stream.s));
        beginLevel();
        if (level == 0) initDist(src);
        BinArgs a{rowPtr.get(), colIdx.get(), dist.get(), stats.get(), nullptr,
                  {bins[cur ^ 1][0].get(), bins[cur ^ 1][1].get(), bins[cur ^ 1][2].get()},
                  0, level, o.small_max, o.large_min};
        for (int b = 0; b < 3; ++b) {
            if (count[b] == 0) continue;
            a.size = count[b];
            a.queue = bins[cur][b].get();
            if (b == 0) binnedSmallKernel<<<divUp(count[b], tg), tg, 0, stream.s>>>(a);
            else if (b == 1) binnedMediumKernel<<<divUp((uint64_t)count[b] * 32, tg), tg, 0, stream.s>>>(a);
            else binnedLargeKernel<<<count[b], tg, 0, stream.s>>>(a);
            GB_LAUNCH_CHECK();
        }
        endLevel();
        const GbLevelStats& s = *hstats.p;
        if (tr) tr->push_back({level, 'T', 'G', 0, 0, (uint64_t)count[0] + count[1] + count[2], edges, msSince(t0)});
        for (int b = 0; b < 3; ++b) count[b] = s.bin[b];
        edges = s.nextEdges;
        cur ^= 1;
    }
}

namespace {
// One gpu_edge level: scan degrees into offsets in place, then expand.
void edgeLevel(gb_bfs& h, uint32_t* q, uint32_t* deg, uint32_t* qNext, uint32_t* degNext, uint32_t size,
               uint64_t total, uint32_t level, uint32_t tg, uint32_t ept) {
    scanExclusive(deg, deg, size, nullptr, h.scan, h.stream.s);
    const uint64_t chunk = (uint64_t)tg * ept;
    edgeExpandKernel<<<divUp(total, chunk), tg, 0, h.stream.s>>>(h.rowPtr.get(), h.colIdx.get(), h.dist.get(),
                                                                 h.stats.get(), q, deg, qNext, degNext, size,
                                                                 (uint32_t)total, level, ept);
    GB_LAUNCH_CHECK();
}
}  // namespace

void gb_bfs::runEdge(uint32_t src, const gb_bfs_options& o, std::vector<gb_level>* tr) {
    const uint32_t tg = checkTg(o.tg);
    if (o.ept == 0) throw Error(GB_ERR_ARG, "ept must be >= 1");
    ensureEdgeBuffers();
    uint32_t *q = qA.get(), *qNext = qB.get(), *deg = degA.get(), *degNext = degB.get();
    hstage.p[0] = src;
    hstage.p[1] = degree(src);
    GB_CUDA(cudaMemcpyAsync(q, hstage.p, 4, cudaMemcpyHostToDevice, stream.s));
    GB_CUDA(cudaMemcpyAsync(deg, hstage.p + 1, 4, cudaMemcpyHostToDevice, stream.s));
    uint32_t size = 1;
    uint64_t total = degree(src);
    lastGpuMs = 0;
    lastLevels = 0;
    for (uint32_t level = 0; size > 0; ++level) {
        auto t0 = std::chrono::steady_clock::now();
        GB_CUDA(cudaEventRecord(ev.a, stream.s));
        beginLevel();
        if (level == 0) initDist(src);
        if (total > 0) edgeLevel(*this, q, deg, qNext, degNext, size, total, level, tg, o.ept);
        endLevel();
        const GbLevelStats& s = *hstats.p;
        if (tr) tr->push_back({level, 'T', 'G', 0, 0, size, total, msSince(t0)});
        size = s.found;
        total = s.nextEdges;
        std::swap(q, qNext);
        std::swap(deg, degNext);
    }
}

// gpu_do: the alpha/beta rule of cpu::bfsDO / GpuBfs::runDirOpt
// (src/cpu/bfs_cpu.cpp:227-283, src/metal/bfs_gpu.mm:326-429), decided on the
// host from the counters read back after every level.
void gb_bfs::runDirOpt(uint32_t src, const gb_bfs_options& o, std::vector<gb_level>* tr) {
    const uint32_t tg = checkTg(o.tg);
    if (o.ept == 0) throw Error(GB_ERR_ARG, "ept must be >= 1");
    ensureEdgeBuffers();
    const uint64_t words = (n + 31) / 32;
    bmFront.ensure(words);
    bmNext.ensure(words);
    uint32_t *q = qA.get(), *qNext = qB.get(), *deg = degA.get(), *degNext = degB.get();
    uint32_t *front = bmFront.get(), *next = bmNext.get();
    hstage.p[0] = src;
    hstage.p[1] = degree(src);
    GB_CUDA(cudaMemcpyAsync(q, hstage.p, 4, cudaMemcpyHostToDevice, stream.s));
    GB_CUDA(cudaMemcpyAsync(deg, hstage.p + 1, 4, cudaMemcpyHostToDevice, stream.s));
    uint64_t size = 1, total = degree(src), scout = total, toCheck = m;
    bool bottomUp = false, toBitmap = false, toQueue = false;
    lastGpuMs = 0;
    lastLevels = 0;
    for (uint32_t level = 0; size > 0; ++level) {
        auto t0 = std::chrono::steady_clock::now();
        if (!bottomUp && (double)scout > (double)toCheck / o.alpha) {
            bottomUp = true;
            toBitmap = true;
        }
        if (!bottomUp) toCheck -= std::min(toCheck, scout);
        GB_CUDA(cudaEventRecord(ev.a, stream.s));
        beginLevel();
        if (level == 0) initDist(src);
        if (bottomUp) {
            if (toBitmap) queueToBitmap(q, size, front, n, stream.s);
            bottomUpKernel<<<gridCap(n, tg), tg, 0, stream.s>>>(rowPtr.get(), colIdx.get(), dist.get(), front, next,
                                                                stats.get(), n, level);
            GB_LAUNCH_CHECK();
        } else {
            if (toQueue) {
                // Bitmap -> queue with the degrees gpu_edge scans; the count
                // lands in stats.bin[0] (unused by this form).
                bitmapToQueue(front, n, q, &stats.get()->bin[0], rowPtr.get(), deg, stream.s);
            }
            if (total > 0) edgeLevel(*this, q, deg, qNext, degNext, (uint32_t)size, total, level, tg, o.ept);
        }
        endLevel();
        const GbLevelStats& s = *hstats.p;
        toBitmap = toQueue = false;
        if (tr)
            tr->push_back({level, bottomUp ? 'B' : 'T', 'G', (uint8_t)(bottomUp ? GB_STRAT_BU : GB_STRAT_TD_EPT2), 0,
                           size, bottomUp ? s.edges : total, msSince(t0)});
        const uint64_t oldSize = size;
        size = s.found;
        total = s.nextEdges;
        if (bottomUp) {
            std::swap(front, next);
            if (!(size >= oldSize || (double)size > (double)n / o.beta)) {
                bottomUp = false;
                toQueue = true;
                scout = 1;
            }
        } else {
            scout = total;
            std::swap(q, qNext);
            std::swap(deg, degNext);
        }
    }
}
