// pr_prep.cpp -- host preprocessing for PageRank: in-degree bins of the
// adaptive pull (GpuPageRank::prepareAdaptive, src/metal/pagerank_gpu.mm:70-86)
// and the Gauss-Seidel update order (prepareGS, :88-192).
#include <omp.h>

#include <algorithm>
#include <cstring>

#include "pagerank.hpp"

using namespace gb;

void gb_pr::prepareAdaptive(uint32_t smallMax, uint32_t largeMin) {
    if (binsReady && binSmall == smallMax && binLarge == largeMin) return;
    if (!hasIn) throw Error(GB_ERR_ARG, "gpu_pull_adaptive needs the in-CSR");
    std::vector<uint32_t> lists[3];
    for (uint32_t v = 0; v < n; ++v) {
        const uint32_t d = hostRowIn[v + 1] - hostRowIn[v];
        lists[d < smallMax ? 0 : (d < largeMin ? 1 : 2)].push_back(v);
    }
    std::vector<uint32_t> all;
    all.reserve(n);
    for (int b = 0; b < 3; ++b) {
        binCount[b] = (uint32_t)lists[b].size();
        all.insert(all.end(), lists[b].begin(), lists[b].end());
    }
    invalidateGraphs();
    bins.ensure(all.size() + 1);
    if (!all.empty()) GB_CUDA(cudaMemcpy(bins.get(), all.data(), all.size() * 4, cudaMemcpyHostToDevice));
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
        if (!b.empty()) {
            gsDeferred = b.size();
            gsNatA = (uint32_t)a.size();
            gsNatB = (uint32_t)b.size();
            a.insert(a.end(), b.begin(), b.end());
            gsNat.ensure(a.size());
            GB_CUDA(cudaMemcpy(gsNat.get(), a.data(), a.size() * 4, cudaMemcpyHostToDevice));
        }
    }
    gsReady = true;
}
