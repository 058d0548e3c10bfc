// pr_prep.cpp -- host preprocessing for PageRank: in-degree bins of the
// adaptive pull (GpuPageRank::prepareAdaptive, src/metal/pagerank_gpu.mm:70-86)
// and the Gauss-Seidel update order (prepareGS, :88-192).
#include <omp.h>

#include <algorithm>
#include <cstring>

#include "pagerank.hpp"

using namespace gb;

namespace {

constexpr uint32_t kChunk = 4096;  // edges per warp chunk of a split vertex

// Chunk table of the split vertices: (vertex, start, end, hub index) per
// chunk, and per hub (first chunk | chunk count).  A zero-degree split vertex
// still gets one (empty) chunk so that its value is stored.
void buildChunks(const std::vector<uint32_t>& verts, const uint32_t* row, std::vector<uint4>& chunks,
                 std::vector<uint32_t>& first) {
    chunks.clear();
    first.clear();
    for (uint32_t h = 0; h < verts.size(); ++h) {
        const uint32_t v = verts[h], b = row[v], e = row[v + 1];
        first.push_back((uint32_t)chunks.size());
        uint32_t c = 0;
        for (uint32_t s = b; s < e || (c == 0); s += kChunk, ++c) chunks.push_back(make_uint4(v, s, std::min(e, s + kChunk), h));
        first.push_back(c);
    }
}

template <class T>
void upload(gb::DevBuf<T>& buf, const std::vector<T>& v) {
    buf.ensure(v.size() + 1);
    if (!v.empty()) GB_CUDA(cudaMemcpy(buf.get(), v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
}

}  // namespace

// Degree-adaptive pull layout.  Vertices are relabeled by descending in-degree
// (stable), so each degree class is a contiguous id range and the hottest
// contributions (the hubs') sit together at the front of the array.  Classes:
//   in-degree >= large_min            split into warp chunks of 4096 edges;
//   small_max <= in-degree < large_min a group of G = clamp(pow2ceil(deg/4), 2, 32)
//                                      lanes per vertex (more vertices in flight
//                                      per warp for short lists);
//   in-degree < small_max             one thread per vertex.
// (The reference's three bins, src/metal/pagerank_gpu.mm:70-86, with the
// medium bin refined by list length and the large bin split across warps.)
void gb_pr::prepareAdaptive(uint32_t smallMax, uint32_t largeMin) {
    if (binsReady && binSmall == smallMax && binLarge == largeMin) return;
    if (!hasIn) throw Error(GB_ERR_ARG, "gpu_pull_adaptive needs the in-CSR");
    const uint32_t* rp = hostRowIn.data();
    const uint32_t* ci = hostColIn.data();
    auto deg = [&](uint32_t v) { return rp[v + 1] - rp[v]; };
    std::vector<uint32_t> order(n);
    for (uint32_t v = 0; v < n; ++v) order[v] = v;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return deg(a) > deg(b); });
    permA.assign(n, 0);
    for (uint32_t i = 0; i < n; ++i) permA[order[i]] = i;
    std::vector<uint32_t> row(n + 1, 0), od(n);
    for (uint32_t i = 0; i < n; ++i) row[i + 1] = row[i] + deg(order[i]);
    std::vector<uint32_t> col((size_t)row[n] + 4, 0);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const uint32_t v = order[i];
        od[i] = hostOutdeg[v];
        uint32_t* out = col.data() + row[i];
        for (uint32_t e = rp[v]; e < rp[v + 1]; ++e) *out++ = permA[ci[e]];
        std::sort(col.data() + row[i], out);
    }
    auto groupOf = [&](uint32_t d) -> uint32_t {  // 0 = split
        if (d >= largeMin) return 0;
        if (d < smallMax) return 1;
        uint32_t g = 2;
        while (g < 32 && 4 * g < d) g *= 2;
        return g;
    };
    std::vector<uint32_t> hubs;
    nBins = 0;
    for (uint32_t i = 0; i < n;) {
        const uint32_t g = groupOf(row[i + 1] - row[i]);
        uint32_t j = i;
        while (j < n && groupOf(row[j + 1] - row[j]) == g) ++j;
        if (g == 0) {
            for (uint32_t v = i; v < j; ++v) hubs.push_back(v);
        } else {
            if (nBins >= 8) throw Error(GB_ERR_STATE, "adaptive layout: degree classes are not contiguous");
            binLo[nBins] = i;
            binHi[nBins] = j;
            binG[nBins] = g;
            ++nBins;
        }
        i = j;
    }
    std::vector<uint4> chunks;
    std::vector<uint32_t> first;
    buildChunks(hubs, row.data(), chunks, first);
    nHubs = (uint32_t)hubs.size();
    nChunks = (uint32_t)chunks.size();
    invalidateGraphs();
    upload(rowA, row);
    upload(colA, col);
    upload(outdegA, od);
    upload(hubChunks, chunks);
    upload(hubFirst, first);
    hubDone.ensure(nHubs + 1);
    GB_CUDA(cudaMemset(hubDone.get(), 0, (nHubs + 1) * sizeof(unsigned)));
    hubPart.ensure(2 * (size_t)nChunks + 2);
    binSmall = smallMax;
    binLarge = largeMin;
    binsReady = true;
}

// Update order of the in-place sweep.  A GPU sweep updates tens of thousands
// of vertices concurrently, so an in-place update helps only where a vertex's
// in-neighbours were updated earlier in the sweep:
//  - colored: up to 8 Jones-Plassmann rounds (a vertex joins a round's set
//    when its priority beats every uncolored in-neighbour's); if the sets
//    cover >= 95% of the vertices every edge crosses sets, so the sets are
//    swept one after another over a private color-major relabeled in-CSR;
//  - natural: one sweep in id order, with one vertex of every mutual pair
//    (u <-> v, both out-degrees in [1, K]) deferred to a second sweep so that
//    it always reads its partner's new value (greedy in id order; the
//    deferred set contains no pair).
void gb_pr::prepareGS(uint32_t pairMaxOutdeg) {
    if (gsReady && gsPairK == pairMaxOutdeg) return;
    if (!hasIn) throw Error(GB_ERR_ARG, "gpu_pull_gs needs the in-CSR");
    gsPairK = pairMaxOutdeg;
    constexpr int kRounds = 8;
    constexpr double kMinCoverage = 0.95;
    const uint32_t* rp = hostRowIn.data();
    const uint32_t* ci = hostColIn.data();
    const uint32_t* od = hostOutdeg.data();
    auto prio = [](uint32_t v) {  // pseudo-random priority, ties impossible (id in the low bits)
        uint64_t x = v + 0x632BE59BD9B4E019ull;
        x = (x ^ (x >> 33)) * 0xFF51AFD7ED558CCDull;
        x ^= x >> 33;
        return (x << 32) | v;
    };
    std::vector<uint8_t> color(n, 0xFF);
    std::vector<std::vector<uint32_t>> sets;
    uint64_t covered = 0;
    std::vector<uint8_t> pick(n);
    for (int c = 0; c < kRounds && covered < n; ++c) {
#pragma omp parallel for schedule(dynamic, 4096)
        for (int64_t v = 0; v < (int64_t)n; ++v) {
            pick[v] = 0;
            if (color[v] != 0xFF) continue;
            bool best = true;
            for (uint32_t e = rp[v]; e < rp[v + 1] && best; ++e) {
                const uint32_t u = ci[e];
                best = u == (uint32_t)v || color[u] != 0xFF || prio(u) < prio((uint32_t)v);
            }
            pick[v] = best;
        }
        std::vector<uint32_t> s;
        for (uint32_t v = 0; v < n; ++v)
            if (pick[v]) {
                color[v] = (uint8_t)c;
                s.push_back(v);
            }
        covered += s.size();
        sets.push_back(std::move(s));
    }
    gsColored = covered >= kMinCoverage * (double)n;
    gsSetStart.clear();
    gsNewId.clear();
    invalidateGraphs();
    if (gsColored) {
        std::vector<uint32_t> rest;
        for (uint32_t v = 0; v < n; ++v)
            if (color[v] == 0xFF) rest.push_back(v);
        if (!rest.empty()) sets.push_back(std::move(rest));
        std::vector<uint32_t> order;
        order.reserve(n);
        gsNewId.assign(n, 0);
        gsSetStart.push_back(0);
        for (auto& s : sets) {
            if (s.empty()) continue;
            // inside a set (swept concurrently) order by descending in-degree, so
            // the set's degree classes are contiguous id ranges
            std::stable_sort(s.begin(), s.end(),
                             [&](uint32_t x, uint32_t y) { return rp[x + 1] - rp[x] > rp[y + 1] - rp[y]; });
            for (size_t i = 0; i < s.size(); ++i) gsNewId[s[i]] = (uint32_t)(order.size() + i);
            order.insert(order.end(), s.begin(), s.end());
            gsSetStart.push_back((uint32_t)order.size());
        }
        std::vector<uint32_t> row(n + 1, 0), deg(n);
        for (uint32_t i = 0; i < n; ++i) row[i + 1] = row[i] + (rp[order[i] + 1] - rp[order[i]]);
        std::vector<uint32_t> col((size_t)row[n] + 4, 0);
#pragma omp parallel for schedule(dynamic, 1024)
        for (int64_t i = 0; i < (int64_t)n; ++i) {
            const uint32_t v = order[i];
            deg[i] = od[v];
            uint32_t* out = col.data() + row[i];
            for (uint32_t e = rp[v]; e < rp[v + 1]; ++e) *out++ = gsNewId[ci[e]];
            std::sort(col.data() + row[i], out);
        }
        rowGS.ensure(n + 1);
        colGS.ensure(col.size());
        outdegGS.ensure(n);
        GB_CUDA(cudaMemcpy(rowGS.get(), row.data(), (n + 1) * 4, cudaMemcpyHostToDevice));
        GB_CUDA(cudaMemcpy(colGS.get(), col.data(), col.size() * 4, cudaMemcpyHostToDevice));
        GB_CUDA(cudaMemcpy(outdegGS.get(), deg.data(), n * 4, cudaMemcpyHostToDevice));
        // per set: split hubs (>= kGsHubMin in-edges) into warp chunks, the rest
        // into group-size classes (thread per vertex below 16 in-edges)
        gsSetLayout.clear();
        std::vector<uint32_t> hubs;
        for (size_t k = 0; k + 1 < gsSetStart.size(); ++k) {
            GsSetLayout L{};
            const uint32_t lo = gsSetStart[k], hi = gsSetStart[k + 1];
            auto groupOf = [&](uint32_t d) -> uint32_t {
                if (d >= kGsHubMin) return 0;
                if (d < 16) return 1;
                uint32_t g = 2;
                while (g < 32 && 4 * g < d) g *= 2;
                return g;
            };
            L.chunk0 = 0;
            std::vector<uint32_t> setHubs;
            for (uint32_t i = lo; i < hi;) {
                const uint32_t g = groupOf(row[i + 1] - row[i]);
                uint32_t j = i;
                while (j < hi && groupOf(row[j + 1] - row[j]) == g) ++j;
                if (g == 0) {
                    for (uint32_t v = i; v < j; ++v) setHubs.push_back(v);
                } else if (L.nBins < 8) {
                    L.lo[L.nBins] = i;
                    L.hi[L.nBins] = j;
                    L.g[L.nBins] = g;
                    ++L.nBins;
                } else {
                    throw Error(GB_ERR_STATE, "colored layout: degree classes are not contiguous");
                }
                i = j;
            }
            L.chunk0 = (uint32_t)hubs.size();  // hub index range, turned into chunks below
            hubs.insert(hubs.end(), setHubs.begin(), setHubs.end());
            L.chunk1 = (uint32_t)hubs.size();
            gsSetLayout.push_back(L);
        }
        std::vector<uint4> chunks;
        std::vector<uint32_t> first;
        buildChunks(hubs, row.data(), chunks, first);
        for (auto& L : gsSetLayout) {  // hub index range -> chunk index range
            const uint32_t h0 = L.chunk0, h1 = L.chunk1;
            L.chunk0 = h0 < hubs.size() ? first[2 * h0] : (uint32_t)chunks.size();
            L.chunk1 = h1 < hubs.size() ? first[2 * h1] : (uint32_t)chunks.size();
        }
        gsHubs = (uint32_t)hubs.size();
        gsChunks = (uint32_t)chunks.size();
        upload(gsHubChunks, chunks);
        upload(gsHubFirst, first);
        gsHubDone.ensure(gsHubs + 1);
        GB_CUDA(cudaMemset(gsHubDone.get(), 0, (gsHubs + 1) * sizeof(unsigned)));
        gsHubPart.ensure(2 * (size_t)gsChunks + 2);
    }
    gsDeferred = 0;
    gsNatA = gsNatB = 0;
    if (!gsColored && pairMaxOutdeg > 0) {
        std::vector<uint8_t> deferred(n, 0);
        for (uint32_t v = 0; v < n; ++v) {
            if (od[v] == 0 || od[v] > pairMaxOutdeg) continue;
            bool partner = false, partnerDeferred = false;
            for (uint32_t e = rp[v]; e < rp[v + 1] && !partnerDeferred; ++e) {
                const uint32_t u = ci[e];  // u -> v
                if (u >= v || od[u] == 0 || od[u] > pairMaxOutdeg) continue;
                if (std::binary_search(ci + rp[u], ci + rp[u + 1], v)) {  // v -> u
                    partner = true;
                    partnerDeferred = deferred[u];
                }
            }
            deferred[v] = partner && !partnerDeferred;
        }
        std::vector<uint32_t> a, b;
        for (uint32_t v = 0; v < n; ++v) (deferred[v] ? b : a).push_back(v);
        if (!b.empty()) gsDeferred = b.size();
        gsNatA = (uint32_t)a.size();
        gsNatB = (uint32_t)b.size();
        a.insert(a.end(), b.begin(), b.end());
        gsNat.ensure(a.size() + 1);
        GB_CUDA(cudaMemcpy(gsNat.get(), a.data(), a.size() * 4, cudaMemcpyHostToDevice));
    } else if (!gsColored) {
        std::vector<uint32_t> a(n);
        for (uint32_t v = 0; v < n; ++v) a[v] = v;
        gsNatA = n;
        gsNatB = 0;
        gsNat.ensure(n + 1);
        GB_CUDA(cudaMemcpy(gsNat.get(), a.data(), a.size() * 4, cudaMemcpyHostToDevice));
    }
    // natural order: vertices with huge in-lists are split into warp chunks
    // (swept first, in place) instead of holding one warp for the whole list
    if (!gsColored) {
        gsHubs = gsChunks = 0;
        std::vector<uint32_t> hubs;
        for (uint32_t v = 0; v < n; ++v)
            if (rp[v + 1] - rp[v] >= kGsHubMin) hubs.push_back(v);
        std::vector<uint4> chunks;
        std::vector<uint32_t> first;
        buildChunks(hubs, rp, chunks, first);
        gsHubs = (uint32_t)hubs.size();
        gsChunks = (uint32_t)chunks.size();
        upload(gsHubChunks, chunks);
        upload(gsHubFirst, first);
        gsHubDone.ensure(gsHubs + 1);
        GB_CUDA(cudaMemset(gsHubDone.get(), 0, (gsHubs + 1) * sizeof(unsigned)));
        gsHubPart.ensure(2 * (size_t)gsChunks + 2);
    }
    gsReady = true;
}

// Blocked pull layout.  Row block k holds rows [k * rowsPer, (k + 1) * rowsPer)
// (ids as given, so blocks get near-equal edge counts on graphs without
// locality), with rowsPer <= kBlkRowCap and no more row blocks than SMs when
// the cap allows (every block then runs in one wave); part p holds columns
// [p * kBlkPart, (p + 1) * kBlkPart).  Every edge u -> v of a row v with
// fewer than kBlkHub in-edges is stored once, as
// (v - first row of its block) << 16 | (u - first column of its part), in
// tile (block of v, part of u); within a tile edges are in row order.  Tiles
// are padded with 0xFFFFFFFF to a multiple of 4 words, so each starts on a
// 16-byte boundary; blkOff holds their starts in 16-byte words.  Rows with
// kBlkHub or more in-edges are listed apart (blkHubs) and summed by a whole
// CUDA block each, with compensated sums.
void gb_pr::prepareBlocked() {
    if (blkReady) return;
    const uint32_t* rp = hostRowIn.data();
    const uint32_t* ci = hostColIn.data();
    const uint32_t sms = (uint32_t)deviceSmCount();
    const uint64_t byCap = (n + kBlkRowCap - 1) / kBlkRowCap;
    nRowBlocks = (uint32_t)std::max<uint64_t>({(uint64_t)1, (uint64_t)sms, byCap});
    rowsPer = (uint32_t)((n + nRowBlocks - 1) / nRowBlocks);
    nRowBlocks = (uint32_t)std::max<uint64_t>(1, (n + rowsPer - 1) / rowsPer);
    nParts = (uint32_t)std::max<uint64_t>(1, (n + kBlkPart - 1) / kBlkPart);
    const uint64_t tiles = (uint64_t)nRowBlocks * nParts;
    std::vector<uint32_t> hubs;
    for (uint64_t v = 0; v < n; ++v)
        if (rp[v + 1] - rp[v] >= kBlkHub) hubs.push_back((uint32_t)v);
    // per tile edge counts, then tile offsets, then the edges
    std::vector<uint32_t> cnt(tiles, 0);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t k = 0; k < (int64_t)nRowBlocks; ++k) {
        const uint64_t r0 = (uint64_t)k * rowsPer, r1 = std::min<uint64_t>(n, r0 + rowsPer);
        uint32_t* c = cnt.data() + (uint64_t)k * nParts;
        for (uint64_t v = r0; v < r1; ++v) {
            if (rp[v + 1] - rp[v] >= kBlkHub) continue;
            for (uint32_t e = rp[v]; e < rp[v + 1]; ++e) ++c[ci[e] / kBlkPart];
        }
    }
    std::vector<uint32_t> off(tiles + 1);
    uint64_t total = 0;  // 16-byte words
    for (uint64_t g = 0; g < tiles; ++g) {
        off[g] = (uint32_t)total;
        total += (cnt[g] + 3) / 4;
        if (total >= (1ull << 32)) throw Error(GB_ERR_ARG, "blocked pull: layout exceeds 2^32 16-byte words");
    }
    off[tiles] = (uint32_t)total;
    std::vector<uint32_t> packed(4 * total, 0xFFFFFFFFu);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t k = 0; k < (int64_t)nRowBlocks; ++k) {
        const uint64_t r0 = (uint64_t)k * rowsPer, r1 = std::min<uint64_t>(n, r0 + rowsPer);
        std::vector<uint64_t> pos(nParts);  // next word per part
        for (uint32_t p = 0; p < nParts; ++p) pos[p] = 4ull * off[(uint64_t)k * nParts + p];
        for (uint64_t v = r0; v < r1; ++v) {
            if (rp[v + 1] - rp[v] >= kBlkHub) continue;
            const uint32_t rowLocal = (uint32_t)(v - r0);
            for (uint32_t e = rp[v]; e < rp[v + 1]; ++e) {
                const uint32_t u = ci[e], p = u / kBlkPart;
                packed[pos[p]++] = rowLocal << 16 | (u - p * kBlkPart);
            }
        }
    }
    upload(blkEdges, packed);
    upload(blkOff, off);
    upload(blkHubs, hubs);
    nBlkHubs = (uint32_t)hubs.size();
    blkReady = true;
    invalidateGraphs();
}
