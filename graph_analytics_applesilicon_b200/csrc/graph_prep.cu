// graph_prep.cu -- graph preparation on the GPU: fromEdgeList, transpose,
// symmetrize and permute (the reference's src/graph/csr.cpp:112-163 and
// src/graph/transform.cpp:9-76, which run on the host and dominate the wall
// time of preparing the 234M-edge graphs).
//
// All four reduce to one step: write one 64-bit key (row << b | column) per
// output entry (b = bits of n - 1), sort the keys, optionally drop repeated
// keys and self-loops, and count rows into row_ptr.  Sorting (row, column)
// keys gives exactly the reference's outputs: rows in id order, every row
// sorted by column.
//
// Sort: least-significant-digit radix sort with 8-bit digits, one pass per
// digit of the key's used bits.  Each pass: (1) per-tile digit histograms
// (tiles of 4096 keys, shared-memory atomics), (2) one exclusive scan of the
// digit-major histogram table (the single-pass scan of prims.cu), (3) a
// stable scatter: a tile is ranked in 16 rounds of 256 keys, within a warp by
// __match_any_sync peers, across the block's warps by a shared-memory table
// of per-warp digit counts (entries tagged with the round, so nothing is
// cleared between rounds), across rounds by running digit bases.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "capi_util.hpp"
#include "graph_host.hpp"
#include "graph_prep.cuh"

namespace gb {
namespace {

constexpr int kRsThreads = 256;
constexpr int kRsRounds = 16;
constexpr int kRsTile = kRsThreads * kRsRounds;  // keys per block
constexpr int kRsWarps = kRsThreads / 32;
constexpr unsigned long long kNoKey = ~0ull;

__global__ void __launch_bounds__(kRsThreads) rsHistKernel(const unsigned long long* keys, uint64_t n, int shift,
                                                           uint32_t* counts, uint32_t tiles) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * kRsTile;
    for (int r = 0; r < kRsRounds; ++r) {
        const uint64_t i = base + (uint64_t)r * kRsThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    counts[(uint64_t)threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];  // digit-major
}

__global__ void __launch_bounds__(kRsThreads) rsScatterKernel(const unsigned long long* keys,
                                                              unsigned long long* out, uint64_t n, int shift,
                                                              const uint32_t* offsets, uint32_t tiles) {
    __shared__ uint32_t base[256];              // running position of each digit in this tile
    __shared__ uint32_t wcnt[kRsWarps][256];    // (round + 1) << 16 | count of the digit in warp w
    __shared__ uint32_t wpre[kRsWarps][256];    // exclusive prefix over warps, this round
    const unsigned tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    base[tid] = offsets[(uint64_t)tid * tiles + blockIdx.x];
    for (int w = 0; w < kRsWarps; ++w) wcnt[w][tid] = 0;
    __syncthreads();
    const uint64_t tileBase = (uint64_t)blockIdx.x * kRsTile;
    for (int r = 0; r < kRsRounds; ++r) {
        const uint64_t i = tileBase + (uint64_t)r * kRsThreads + tid;
        const bool valid = i < n;
        const unsigned long long k = valid ? keys[i] : kNoKey;
        const uint32_t d = valid ? (uint32_t)((k >> shift) & 255u) : 256u + lane;  // invalid lanes: own group
        const unsigned peers = __match_any_sync(0xFFFFFFFFu, d);
        const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
        const uint32_t tag = (uint32_t)(r + 1) << 16;
        if (valid && rank == 0) wcnt[warp][d] = tag | __popc(peers);
        __syncthreads();
        {  // digit tid: prefix over warps
            uint32_t run = 0;
            for (int w = 0; w < kRsWarps; ++w) {
                wpre[w][tid] = run;
                const uint32_t e = wcnt[w][tid];
                run += (e >> 16) == (uint32_t)(r + 1) ? (e & 0xFFFFu) : 0u;
            }
            __syncthreads();
            if (valid) out[base[d] + wpre[warp][d] + rank] = k;
            __syncthreads();
            base[tid] += run;
        }
        __syncthreads();
    }
}

// keep[i] = 1 when key i starts a new value (unique) and is not a self-loop
// (dropSelf); b = column bits.
__global__ void rsKeepKernel(const unsigned long long* keys, uint64_t n, int b, bool unique, bool dropSelf,
                             uint32_t* keep) {
    const unsigned long long mask = (1ull << b) - 1ull;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned long long k = keys[i];
        bool kp = true;
        if (unique && i > 0 && keys[i - 1] == k) kp = false;
        if (dropSelf && (k >> b) == (k & mask)) kp = false;
        keep[i] = kp ? 1u : 0u;
    }
}

// Kept keys -> col_idx at their scanned positions, and row degrees.
__global__ void rsEmitKernel(const unsigned long long* keys, uint64_t n, int b, const uint32_t* keep,
                             const uint32_t* pos, uint32_t* col, uint32_t* deg) {
    const unsigned long long mask = (1ull << b) - 1ull;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (!keep[i]) continue;
        const unsigned long long k = keys[i];
        col[pos[i]] = (uint32_t)(k & mask);
        atomicAdd(&deg[(uint32_t)(k >> b)], 1u);
    }
}

__global__ void initIotaKernel(uint32_t* p, uint64_t n) {
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
        p[v] = (uint32_t)v;
}

// Keys of a CSR's entries: (map(row) or col-as-row) per mode.
//   mode 0: (row, col)             mode 1: (col, row)  (transpose)
//   mode 2: (perm[row], perm[col])  mode 3: (row, col) and (col, row) (symmetrize)
// out has m (modes 0-2) or 2m (mode 3) keys; warp per row.
__global__ void csrKeysKernel(const uint32_t* rp, const uint32_t* ci, uint64_t n, uint64_t m, int b, int mode,
                              const uint32_t* perm, unsigned long long* out) {
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    for (uint64_t v = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += nw) {
        const uint32_t s = rp[v], e = rp[v + 1];
        for (uint32_t i = s + lane; i < e; i += 32) {
            const unsigned long long u = v, w = ci[i];
            unsigned long long k;
            if (mode == 1) k = (w << b) | u;
            else if (mode == 2) k = ((unsigned long long)perm[u] << b) | perm[w];
            else k = (u << b) | w;
            out[i] = k;
            if (mode == 3) out[m + i] = (w << b) | u;
        }
    }
}

__global__ void edgeKeysKernel(const uint32_t* eu, const uint32_t* ev, uint64_t ne, int b, bool both,
                               unsigned long long* out) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ne; i += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned long long u = eu[i], v = ev[i];
        out[i] = (u << b) | v;
        if (both) out[ne + i] = (v << b) | u;
    }
}

// Input checks on the device (every id that reaches the key kernels must be
// below n): bad |= 1 row_ptr decreases, 2 column >= n, 4 edge endpoint >= n,
// 8 perm value >= n or repeated (seen: ceil(n/32) zeroed words).
__global__ void checkCsrKernel(const uint32_t* rp, const uint32_t* ci, uint64_t n, uint64_t m, unsigned* bad) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    unsigned f = 0;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
        if (rp[v] > rp[v + 1]) f |= 1u;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride)
        if (ci[i] >= n) f |= 2u;
    if (f) atomicOr(bad, f);
}

__global__ void checkEdgesKernel(const uint32_t* eu, const uint32_t* ev, uint64_t ne, uint64_t n, unsigned* bad) {
    unsigned f = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ne; i += (uint64_t)gridDim.x * blockDim.x)
        if (eu[i] >= n || ev[i] >= n) f |= 4u;
    if (f) atomicOr(bad, f);
}

__global__ void checkPermKernel(const uint32_t* perm, uint64_t n, uint32_t* seen, unsigned* bad) {
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t p = perm[v];
        if (p >= n) {
            atomicOr(bad, 8u);
            continue;
        }
        if (atomicOr(&seen[p >> 5], 1u << (p & 31)) & (1u << (p & 31))) atomicOr(bad, 8u);
    }
}

// Connected components (symmetric graph) by hooking and pointer jumping:
// every edge hooks the larger of its endpoints' roots under the smaller
// (atomicMin), then every vertex jumps to its root; repeated until no hook
// changes anything.  A root only ever moves to a smaller id, so each
// component ends rooted at its smallest vertex: the reference's component
// order (components numbered by their first, i.e. smallest, vertex).
__device__ __forceinline__ uint32_t ccRoot(const uint32_t* parent, uint32_t v) {
    uint32_t p = parent[v];
    while (p != v) {
        v = p;
        p = parent[v];
    }
    return v;
}

__global__ void ccHookKernel(const uint32_t* rp, const uint32_t* ci, uint64_t n, uint32_t* parent, unsigned* changed) {
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    bool any = false;
    for (uint64_t u = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < n; u += nw) {
        for (uint32_t i = rp[u] + lane; i < rp[u + 1]; i += 32) {
            const uint32_t v = ci[i];
            if (v <= u) continue;  // each undirected edge once
            const uint32_t ru = ccRoot(parent, (uint32_t)u), rv = ccRoot(parent, v);
            if (ru == rv) continue;
            const uint32_t hi = ru > rv ? ru : rv, lo = ru > rv ? rv : ru;
            if (atomicMin(&parent[hi], lo) > lo) any = true;
        }
    }
    if (__any_sync(0xFFFFFFFFu, any) && lane == 0) atomicOr(changed, 1u);
}

__global__ void ccJumpKernel(uint64_t n, uint32_t* parent) {
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
        parent[v] = ccRoot(parent, (uint32_t)v);
}

// size per root, then the best (largest; the smallest root among equals)
// packed as (size << 32) | (~root) into one atomicMax.
__global__ void ccSizeKernel(uint64_t n, const uint32_t* parent, uint32_t* size) {
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(&size[parent[v]], 1u);
}

__global__ void ccBestKernel(uint64_t n, const uint32_t* size, unsigned long long* best) {
    unsigned long long b = 0;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
        if (size[v]) {
            const unsigned long long key = ((unsigned long long)size[v] << 32) | (0xFFFFFFFFu - (uint32_t)v);
            b = key > b ? key : b;
        }
    if (b) atomicMax(best, b);
}

__global__ void ccMaskKernel(uint64_t n, const uint32_t* parent, const unsigned long long* best, uint8_t* ok) {
    const uint32_t root = 0xFFFFFFFFu - (uint32_t)(*best & 0xFFFFFFFFull);
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
        ok[v] = parent[v] == root ? 1 : 0;
}

}  // namespace

uint32_t prepGrid(uint64_t work, uint32_t threads) {
    const uint64_t g = (work + threads - 1) / threads;
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(g, (uint64_t)deviceSmCount() * 16));
}

int keyBits(uint64_t n) {
    int b = 1;
    while (b < 32 && (1ull << b) < n) ++b;
    return b;
}

// Sorts N keys whose used bits are [0, bits) in place (a holds the result).
void radixSortKeys(DevBuf<unsigned long long>& a, DevBuf<unsigned long long>& tmp, uint64_t N, int bits,
                   ScanScratch& sc, cudaStream_t st, DevBuf<uint32_t>* countsScratch) {
    if (N < 2) return;
    if (N >= (1ull << 32)) throw Error(GB_ERR_ARG, "graph prep: more than 2^32 entries");
    const uint32_t tiles = (uint32_t)((N + kRsTile - 1) / kRsTile);
    DevBuf<uint32_t> own;
    DevBuf<uint32_t>& counts = countsScratch ? *countsScratch : own;
    counts.ensure((uint64_t)tiles * 256 + 1);
    tmp.ensure(N);
    unsigned long long* src = a.get();
    unsigned long long* dst = tmp.get();
    int passes = 0;
    for (int shift = 0; shift < bits; shift += 8, ++passes) {
        rsHistKernel<<<tiles, kRsThreads, 0, st>>>(src, N, shift, counts.get(), tiles);
        GB_LAUNCH_CHECK();
        scanExclusive(counts.get(), counts.get(), (uint64_t)tiles * 256, nullptr, sc, st);
        rsScatterKernel<<<tiles, kRsThreads, 0, st>>>(src, dst, N, shift, counts.get(), tiles);
        GB_LAUNCH_CHECK();
        std::swap(src, dst);
    }
    if (passes & 1) GB_CUDA(cudaMemcpyAsync(a.get(), src, N * 8, cudaMemcpyDeviceToDevice, st));
}

// Sorted keys -> CSR (host arrays in *out), optionally unique / without self-loops.
void keysToCsr(DevBuf<unsigned long long>& keys, uint64_t N, uint64_t n, int b, bool unique, bool dropSelf,
               uint32_t flags, ScanScratch& sc, cudaStream_t st, gb_csr* out) {
    DevBuf<uint32_t> keep, pos, col, deg;
    keep.ensure(N + 1);
    pos.ensure(N + 1);
    col.ensure(N + 1);
    deg.ensure(n + 1);
    DevBuf<uint32_t> total;
    total.ensure(1);
    GB_CUDA(cudaMemsetAsync(deg.get(), 0, (n + 1) * 4, st));
    uint32_t m2 = 0;
    if (N) {
        rsKeepKernel<<<prepGrid(N, 256), 256, 0, st>>>(keys.get(), N, b, unique, dropSelf, keep.get());
        GB_LAUNCH_CHECK();
        scanExclusive(keep.get(), pos.get(), N, total.get(), sc, st);
        rsEmitKernel<<<prepGrid(N, 256), 256, 0, st>>>(keys.get(), N, b, keep.get(), pos.get(), col.get(), deg.get());
        GB_LAUNCH_CHECK();
        GB_CUDA(cudaMemcpyAsync(&m2, total.get(), 4, cudaMemcpyDeviceToHost, st));
    }
    // row_ptr = exclusive scan of the degrees (n + 1 entries: the last is m)
    DevBuf<uint32_t> rp;
    rp.ensure(n + 2);
    scanExclusive(deg.get(), rp.get(), n + 1, nullptr, sc, st);
    GB_CUDA(cudaStreamSynchronize(st));
    uint32_t* hrp = static_cast<uint32_t*>(std::malloc((n + 1) * 4));
    uint32_t* hci = static_cast<uint32_t*>(std::malloc(std::max<uint64_t>(m2, 1) * 4));
    if (!hrp || !hci) {
        std::free(hrp);
        std::free(hci);
        throw Error(GB_ERR_OOM, "graph prep: host allocation failed");
    }
    GB_CUDA(cudaMemcpy(hrp, rp.get(), (n + 1) * 4, cudaMemcpyDeviceToHost));
    if (m2) GB_CUDA(cudaMemcpy(hci, col.get(), (uint64_t)m2 * 4, cudaMemcpyDeviceToHost));
    out->n = n;
    out->m = m2;
    out->flags = flags;
    out->row_ptr = hrp;
    out->col_idx = hci;
}

// Connected components of a symmetric device CSR: parent[v] = the smallest
// vertex of v's component (hook + jump rounds; each round at least halves the
// number of roots that still have a smaller neighbouring root, so 64 rounds
// cover any n < 2^32 many times over).
void connectedComponents(const uint32_t* rp, const uint32_t* ci, uint64_t n, uint32_t* parent, cudaStream_t st) {
    DevBuf<unsigned> changed;
    changed.ensure(1);
    initIotaKernel<<<prepGrid(n, 256), 256, 0, st>>>(parent, n);
    GB_LAUNCH_CHECK();
    for (int round = 0; round < 64; ++round) {
        GB_CUDA(cudaMemsetAsync(changed.get(), 0, 4, st));
        ccHookKernel<<<prepGrid(n * 32, 256), 256, 0, st>>>(rp, ci, n, parent, changed.get());
        GB_LAUNCH_CHECK();
        ccJumpKernel<<<prepGrid(n, 256), 256, 0, st>>>(n, parent);
        GB_LAUNCH_CHECK();
        unsigned h = 0;
        GB_CUDA(cudaMemcpyAsync(&h, changed.get(), 4, cudaMemcpyDeviceToHost, st));
        GB_CUDA(cudaStreamSynchronize(st));
        if (h == 0) return;
    }
    throw Error(GB_ERR_STATE, "connected components did not settle in 64 rounds");
}

namespace {

// Reads the device check word; throws if any check failed.
void requireChecks(DevBuf<unsigned>& bad, cudaStream_t st) {
    unsigned h = 0;
    GB_CUDA(cudaMemcpyAsync(&h, bad.get(), 4, cudaMemcpyDeviceToHost, st));
    GB_CUDA(cudaStreamSynchronize(st));
    if (h & 1u) throw Error(GB_ERR_ARG, "graph prep: row_ptr must not decrease");
    if (h & 2u) throw Error(GB_ERR_ARG, "graph prep: column id >= n");
    if (h & 4u) throw Error(GB_ERR_ARG, "gb_csr_from_edges_gpu: edge endpoint >= n");
    if (h & 8u) throw Error(GB_ERR_ARG, "gb_csr_permute_gpu: perm is not a permutation of [0, n)");
}

// Uploads a host CSR.
void uploadCsr(const gb_csr* g, DevBuf<uint32_t>& rp, DevBuf<uint32_t>& ci, cudaStream_t st) {
    rp.ensure(g->n + 1);
    ci.ensure(g->m + 1);
    GB_CUDA(cudaMemcpyAsync(rp.get(), g->row_ptr, (g->n + 1) * 4, cudaMemcpyHostToDevice, st));
    if (g->m) GB_CUDA(cudaMemcpyAsync(ci.get(), g->col_idx, g->m * 4, cudaMemcpyHostToDevice, st));
}

}  // namespace

void checkDeviceCsr(const uint32_t* rp, const uint32_t* ci, uint64_t n, uint64_t m, cudaStream_t st) {
    DevBuf<unsigned> bad;
    bad.ensure(1);
    GB_CUDA(cudaMemsetAsync(bad.get(), 0, 4, st));
    checkCsrKernel<<<prepGrid(std::max(n, m), 256), 256, 0, st>>>(rp, ci, n, m, bad.get());
    GB_LAUNCH_CHECK();
    requireChecks(bad, st);
}

void uploadCheckedCsr(const gb_csr* g, DevBuf<uint32_t>& rp, DevBuf<uint32_t>& ci, cudaStream_t st) {
    GB_REQUIRE(g && g->row_ptr && (g->m == 0 || g->col_idx), "null CSR arrays");
    GB_REQUIRE(g->n >= 1 && g->n < 0xFFFFFFFFull, "graph prep: n must be in [1, 2^32 - 1)");
    GB_REQUIRE(g->m < (1ull << 32), "graph prep: m must fit in uint32");
    GB_REQUIRE(g->row_ptr[0] == 0 && g->row_ptr[g->n] == g->m, "graph prep: row_ptr must run from 0 to m");
    DevBuf<unsigned> bad;
    bad.ensure(1);
    GB_CUDA(cudaMemsetAsync(bad.get(), 0, 4, st));
    uploadCsr(g, rp, ci, st);
    checkCsrKernel<<<prepGrid(std::max(g->n, g->m), 256), 256, 0, st>>>(rp.get(), ci.get(), g->n, g->m, bad.get());
    GB_LAUNCH_CHECK();
    requireChecks(bad, st);
}

namespace {

constexpr uint32_t kFlagDirected = 1u, kFlagSorted = 2u, kFlagDedup = 4u;

// mode as csrKeysKernel; see the entry points for flags and uniqueness.
void csrOp(const gb_csr* g, int mode, const uint32_t* permHost, bool unique, bool dropSelf, uint32_t flags,
           gb_csr* out) {
    GB_REQUIRE(g && out, "null argument");
    GB_REQUIRE(g->n >= 1 && g->n < 0xFFFFFFFFull, "graph prep: n must be in [1, 2^32 - 1)");
    GB_REQUIRE(g->m < (1ull << 32), "graph prep: m must fit in uint32");
    GB_REQUIRE(g->row_ptr && (g->m == 0 || g->col_idx), "null CSR arrays");
    GB_REQUIRE(g->row_ptr[0] == 0 && g->row_ptr[g->n] == g->m, "graph prep: row_ptr must run from 0 to m");
    Stream st;
    ScanScratch sc;
    DevBuf<uint32_t> rp, ci, perm, seen;
    DevBuf<unsigned> bad;
    bad.ensure(1);
    GB_CUDA(cudaMemsetAsync(bad.get(), 0, 4, st.s));
    uploadCsr(g, rp, ci, st.s);
    checkCsrKernel<<<prepGrid(std::max(g->n, g->m), 256), 256, 0, st.s>>>(rp.get(), ci.get(), g->n, g->m, bad.get());
    GB_LAUNCH_CHECK();
    if (mode == 2) {
        perm.ensure(g->n);
        seen.ensure((g->n + 31) / 32);
        GB_CUDA(cudaMemcpyAsync(perm.get(), permHost, g->n * 4, cudaMemcpyHostToDevice, st.s));
        GB_CUDA(cudaMemsetAsync(seen.get(), 0, (g->n + 31) / 32 * 4, st.s));
        checkPermKernel<<<prepGrid(g->n, 256), 256, 0, st.s>>>(perm.get(), g->n, seen.get(), bad.get());
        GB_LAUNCH_CHECK();
    }
    requireChecks(bad, st.s);
    const int b = keyBits(g->n);
    const uint64_t N = mode == 3 ? 2 * g->m : g->m;
    DevBuf<unsigned long long> keys, tmp;
    keys.ensure(N + 1);
    if (g->m) {
        csrKeysKernel<<<prepGrid(g->n * 32, 256), 256, 0, st.s>>>(rp.get(), ci.get(), g->n, g->m, b, mode, perm.get(),
                                                                 keys.get());
        GB_LAUNCH_CHECK();
    }
    radixSortKeys(keys, tmp, N, 2 * b, sc, st.s);
    keysToCsr(keys, N, g->n, b, unique, dropSelf, flags, sc, st.s, out);
}

}  // namespace
}  // namespace gb

using namespace gb;

extern "C" {

int gb_csr_from_edges_gpu(uint64_t n, const uint32_t* eu, const uint32_t* ev, uint64_t ne, int directed,
                          gb_csr* out) {
    return guard([&] {
        GB_REQUIRE(out && (ne == 0 || (eu && ev)), "null argument");
        GB_REQUIRE(n >= 1 && n < 0xFFFFFFFFull, "graph prep: n must be in [1, 2^32 - 1)");
        Stream st;
        ScanScratch sc;
        DevBuf<uint32_t> du, dv;
        DevBuf<unsigned> bad;
        bad.ensure(1);
        du.ensure(ne + 1);
        dv.ensure(ne + 1);
        GB_CUDA(cudaMemsetAsync(bad.get(), 0, 4, st.s));
        if (ne) {
            GB_CUDA(cudaMemcpyAsync(du.get(), eu, ne * 4, cudaMemcpyHostToDevice, st.s));
            GB_CUDA(cudaMemcpyAsync(dv.get(), ev, ne * 4, cudaMemcpyHostToDevice, st.s));
            checkEdgesKernel<<<prepGrid(ne, 256), 256, 0, st.s>>>(du.get(), dv.get(), ne, n, bad.get());
            GB_LAUNCH_CHECK();
        }
        requireChecks(bad, st.s);
        const int b = keyBits(n);
        const uint64_t N = directed ? ne : 2 * ne;
        DevBuf<unsigned long long> keys, tmp;
        keys.ensure(N + 1);
        if (ne) {
            edgeKeysKernel<<<prepGrid(ne, 256), 256, 0, st.s>>>(du.get(), dv.get(), ne, b, !directed, keys.get());
            GB_LAUNCH_CHECK();
        }
        radixSortKeys(keys, tmp, N, 2 * b, sc, st.s);
        keysToCsr(keys, N, n, b, true, true, (directed ? kFlagDirected : 0u) | kFlagSorted | kFlagDedup, sc, st.s,
                  out);
    });
}

int gb_csr_transpose_gpu(const gb_csr* g, gb_csr* out) {
    return guard([&] { csrOp(g, 1, nullptr, false, false, g ? g->flags : 0u, out); });
}

int gb_csr_symmetrize_gpu(const gb_csr* g, gb_csr* out) {
    return guard([&] {
        GB_REQUIRE(g && out, "null argument");
        if (!(g->flags & kFlagDirected)) {  // undirected: the same graph, as given (transform.cpp:27)
            out->row_ptr = static_cast<uint32_t*>(std::malloc((g->n + 1) * 4));
            out->col_idx = static_cast<uint32_t*>(std::malloc(std::max<uint64_t>(g->m, 1) * 4));
            if (!out->row_ptr || !out->col_idx) {
                std::free(out->row_ptr);
                std::free(out->col_idx);
                out->row_ptr = out->col_idx = nullptr;
                throw Error(GB_ERR_OOM, "graph prep: host allocation failed");
            }
            std::memcpy(out->row_ptr, g->row_ptr, (g->n + 1) * 4);
            if (g->m) std::memcpy(out->col_idx, g->col_idx, g->m * 4);
            out->n = g->n;
            out->m = g->m;
            out->flags = g->flags;
            return;
        }
        GB_REQUIRE(g->flags & kFlagDedup,
                   "gb_csr_symmetrize_gpu: the input must be duplicate-free (kFlagDedup); "
                   "gb_csr_symmetrize handles lists with repeated entries");
        csrOp(g, 3, nullptr, true, false, kFlagSorted | kFlagDedup, out);
    });
}

int gb_csr_permute_gpu(const gb_csr* g, const uint32_t* perm, gb_csr* out) {
    return guard([&] {
        GB_REQUIRE(g && perm, "null argument");
        csrOp(g, 2, perm, false, false, g->flags, out);  // perm is checked on the device
    });
}

int gb_pick_sources_gpu(const gb_csr* g, int count, uint64_t seed, int any_component, uint32_t* out, int* k) {
    return guard([&] {
        GB_REQUIRE(g && g->row_ptr && out, "null argument");
        GB_REQUIRE(g->n >= 1 && g->n < 0xFFFFFFFFull, "graph prep: n must be in [1, 2^32 - 1)");
        GB_REQUIRE(g->row_ptr[0] == 0 && g->row_ptr[g->n] == g->m, "graph prep: row_ptr must run from 0 to m");
        const uint64_t n = g->n;
        std::vector<uint8_t> ok(n, 1);
        if (!any_component) {
            GB_REQUIRE(!(g->flags & kFlagDirected),
                       "gb_pick_sources_gpu: components need a symmetric graph (gb_pick_sources follows "
                       "out-edges of directed ones)");
            Stream st;
            DevBuf<uint32_t> rp, ci, parent, size;
            DevBuf<unsigned long long> best;
            DevBuf<uint8_t> dok;
            best.ensure(1);
            uploadCheckedCsr(g, rp, ci, st.s);
            parent.ensure(n);
            size.ensure(n);
            dok.ensure(n);
            connectedComponents(rp.get(), ci.get(), n, parent.get(), st.s);
            GB_CUDA(cudaMemsetAsync(size.get(), 0, n * 4, st.s));
            GB_CUDA(cudaMemsetAsync(best.get(), 0, 8, st.s));
            ccSizeKernel<<<prepGrid(n, 256), 256, 0, st.s>>>(n, parent.get(), size.get());
            ccBestKernel<<<prepGrid(n, 256), 256, 0, st.s>>>(n, size.get(), best.get());
            ccMaskKernel<<<prepGrid(n, 256), 256, 0, st.s>>>(n, parent.get(), best.get(), dok.get());
            GB_LAUNCH_CHECK();
            GB_CUDA(cudaMemcpyAsync(ok.data(), dok.get(), n, cudaMemcpyDeviceToHost, st.s));
            GB_CUDA(cudaStreamSynchronize(st.s));
        }
        auto s = drawSources(n, g->row_ptr, ok, count, seed);
        if (!s.empty()) std::memcpy(out, s.data(), s.size() * 4);
        if (k) *k = (int)s.size();
    });
}

}  // extern "C"
