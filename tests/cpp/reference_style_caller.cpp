// A caller written the way the reference's gbench drives its GPU classes
// (src/bench/main.cpp:88-113 bfsVariant, :218-249 options and construction,
// :447-454 PageRank options, :539-553 the result fields), compiled unchanged
// against include/graph_b200.hpp.  graph::CSR and util::BfsLevel below are
// stand-ins with the reference's field names (src/graph/csr.hpp:29-45,
// src/util/trace.hpp:7-14); the test program checks every depth against its
// own serial BFS and the ranks against its own double-precision PageRank.
//
// Exit 0 and "OK" on success; 1 and a message on a mismatch.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "graph_b200.hpp"

namespace util {
struct BfsLevel {
    uint32_t level;
    uint64_t frontier;
    uint64_t edges;
    char direction;
    char device;
    double time_ms;
};
}  // namespace util

namespace graph {
struct CSR {
    uint64_t n = 0;
    uint64_t m = 0;
    uint32_t flags = 0;
    const uint32_t* row_ptr = nullptr;
    const uint32_t* col_idx = nullptr;
    std::shared_ptr<const void> storage;
    bool directed() const { return flags & 1u; }
    uint32_t degree(uint32_t v) const { return row_ptr[v + 1] - row_ptr[v]; }
    static CSR fromVectors(std::vector<uint32_t> rp, std::vector<uint32_t> ci, uint32_t flags) {
        auto hold = std::make_shared<std::pair<std::vector<uint32_t>, std::vector<uint32_t>>>(std::move(rp), std::move(ci));
        CSR g;
        g.n = hold->first.size() - 1;
        g.m = hold->second.size();
        g.flags = flags;
        g.row_ptr = hold->first.data();
        g.col_idx = hold->second.data();
        g.storage = hold;
        return g;
    }
};
}  // namespace graph

using graph::CSR;
using BfsFn = std::function<void(const CSR&, uint32_t, uint32_t*, std::vector<util::BfsLevel>*)>;

// src/bench/main.cpp:88-113, GPU branches.
BfsFn bfsVariant(const std::string& variant, gpu::GpuBfs* gbfs, const gpu::GpuBfsOptions& gopt) {
    if (variant == "gpu_vertex")
        return [gbfs, gopt](const CSR&, uint32_t s, uint32_t* d, std::vector<util::BfsLevel>* tr) {
            gbfs->runVertex(s, d, gopt, tr);
        };
    if (variant == "gpu_naive")
        return [gbfs, gopt](const CSR&, uint32_t s, uint32_t* d, std::vector<util::BfsLevel>* tr) {
            gbfs->runNaive(s, d, gopt, tr);
        };
    if (variant == "gpu_binned")
        return [gbfs, gopt](const CSR&, uint32_t s, uint32_t* d, std::vector<util::BfsLevel>* tr) {
            gbfs->runBinned(s, d, gopt, tr);
        };
    if (variant == "gpu_edge")
        return [gbfs, gopt](const CSR&, uint32_t s, uint32_t* d, std::vector<util::BfsLevel>* tr) {
            gbfs->runEdge(s, d, gopt, tr);
        };
    if (variant == "gpu_do")
        return [gbfs, gopt](const CSR&, uint32_t s, uint32_t* d, std::vector<util::BfsLevel>* tr) {
            gbfs->runDO(s, d, gopt, tr);
        };
    if (variant == "hybrid")
        return [gbfs, gopt](const CSR&, uint32_t s, uint32_t* d, std::vector<util::BfsLevel>* tr) {
            gbfs->runHybrid(s, d, gopt, tr);
        };
    return nullptr;
}

// A grid with its last column joined to a hub: some high-degree and many
// low-degree vertices, symmetric, sorted, no duplicates.
CSR makeGraph(uint32_t side) {
    const uint32_t n = side * side + 1, hub = side * side;
    std::vector<std::vector<uint32_t>> adj(n);
    auto link = [&](uint32_t a, uint32_t b) {
        adj[a].push_back(b);
        adj[b].push_back(a);
    };
    for (uint32_t r = 0; r < side; ++r)
        for (uint32_t c = 0; c < side; ++c) {
            uint32_t v = r * side + c;
            if (c + 1 < side) link(v, v + 1);
            if (r + 1 < side) link(v, v + side);
            if (c + 1 == side) link(v, hub);
        }
    std::vector<uint32_t> rp(n + 1, 0), ci;
    for (uint32_t v = 0; v < n; ++v) {
        std::sort(adj[v].begin(), adj[v].end());
        ci.insert(ci.end(), adj[v].begin(), adj[v].end());
        rp[v + 1] = (uint32_t)ci.size();
    }
    return CSR::fromVectors(std::move(rp), std::move(ci), 2u | 4u);
}

std::vector<uint32_t> serialBfs(const CSR& g, uint32_t s) {
    std::vector<uint32_t> d(g.n, 0xFFFFFFFFu), q{s};
    d[s] = 0;
    for (size_t h = 0; h < q.size(); ++h)
        for (uint32_t i = g.row_ptr[q[h]]; i < g.row_ptr[q[h] + 1]; ++i)
            if (d[g.col_idx[i]] == 0xFFFFFFFFu) {
                d[g.col_idx[i]] = d[q[h]] + 1;
                q.push_back(g.col_idx[i]);
            }
    return d;
}

std::vector<double> serialPagerank(const CSR& in, const std::vector<uint32_t>& od, int iters) {
    const uint64_t n = in.n;
    std::vector<double> r(n, 1.0 / n), next(n);
    for (int it = 0; it < iters; ++it) {
        double dang = 0;
        for (uint64_t u = 0; u < n; ++u)
            if (!od[u]) dang += r[u];
        for (uint64_t v = 0; v < n; ++v) {
            double s = 0;
            for (uint32_t i = in.row_ptr[v]; i < in.row_ptr[v + 1]; ++i) s += r[in.col_idx[i]] / od[in.col_idx[i]];
            next[v] = 0.15 / n + 0.85 * (s + dang / n);
        }
        r.swap(next);
    }
    return r;
}

int main() {
    CSR stored = makeGraph(120);
    // src/bench/main.cpp:218-229
    gpu::GpuBfsOptions gopt;
    gopt.tg = 256;
    gopt.smallMax = 16;
    gopt.largeMin = 256;
    gopt.ept = 2;
    gopt.alpha = 15.0;
    gopt.beta = 18.0;
    gopt.cpuThreads = 4;
    gopt.hybridT = 100000;
    // src/bench/main.cpp:236-243
    CSR g = stored;
    CSR refG = g;
    std::unique_ptr<gpu::MetalContext> ctx = std::make_unique<gpu::MetalContext>();
    std::unique_ptr<gpu::GpuBfs> gbfs = std::make_unique<gpu::GpuBfs>(*ctx, g);
    g = gbfs->graph();  // the GPU's copy of the graph, as a host CSR
    if (g.n != refG.n || g.m != refG.m) {
        std::printf("graph(): n/m differ\n");
        return 1;
    }
    uint32_t* dist = gbfs->dist();
    const uint32_t sources[] = {0, 7, 120 * 60 + 33, 120 * 120};
    for (const char* v : {"gpu_vertex", "gpu_naive", "gpu_binned", "gpu_edge", "gpu_do", "hybrid"}) {
        BfsFn fn = bfsVariant(v, gbfs.get(), gopt);
        for (uint32_t s : sources) {
            std::vector<util::BfsLevel> trace;
            fn(g, s, dist, &trace);
            std::vector<uint32_t> want = serialBfs(refG, s);
            for (uint64_t x = 0; x < g.n; ++x)
                if (dist[x] != want[x]) {
                    std::printf("%s source %u vertex %llu: got %u want %u\n", v, s, (unsigned long long)x, dist[x],
                                want[x]);
                    return 1;
                }
            if (trace.empty() || trace[0].level != 0 || trace[0].frontier != 1 || trace[0].device != 'G') {
                std::printf("%s: bad trace\n", v);
                return 1;
            }
        }
        std::printf("%s ok, %.3f ms, %u levels\n", v, gbfs->lastGpuMs(), gbfs->lastLevels());
    }
    // src/bench/main.cpp:447-454 and 539-553
    gpu::GpuPrOptions popt;
    popt.iters = 20;
    popt.tol = 0;
    popt.tg = 256;
    popt.smallMax = 16;
    popt.largeMin = 256;
    popt.inPlace = false;
    popt.tolRel = 0;
    std::vector<uint32_t> outdeg(refG.n);
    for (uint64_t v = 0; v < refG.n; ++v) outdeg[v] = refG.degree((uint32_t)v);
    auto gpr = std::make_unique<gpu::GpuPageRank>(*ctx, refG, refG, outdeg, false, true);
    gpr->prepareAdaptive(popt.smallMax, popt.largeMin);
    std::vector<double> want = serialPagerank(refG, outdeg, 20);
    double lastDelta = -1, lastMaxRel = -1;
    bool floorStop = false;
    for (const char* v : {"gpu_pull_scalar", "gpu_pull_vector", "gpu_pull_adaptive"}) {
        gpu::GpuPrResult r = gpr->run(gpu::parsePrVariant(v), popt);
        lastDelta = r.lastDelta;
        lastMaxRel = r.lastMaxRel;
        floorStop = r.floorStop;
        const float* ranks = gpr->ranks();
        double l1 = 0;
        for (uint64_t x = 0; x < refG.n; ++x) l1 += std::fabs(ranks[x] - want[x]);
        if (r.iters != 20 || l1 >= 1e-4 || !(r.gpuMs > 0)) {
            std::printf("%s: iters %d, L1 %.3g, gpuMs %.3f\n", v, r.iters, l1, r.gpuMs);
            return 1;
        }
        std::printf("%s ok, L1 %.2e, %.3f ms\n", v, l1, r.gpuMs);
    }
    popt.tol = 1e-6;
    popt.iters = 1000;
    gpu::GpuPrResult r = gpr->run(gpu::PrVariant::PullVector, popt);
    lastDelta = r.lastDelta;
    lastMaxRel = r.lastMaxRel;
    floorStop = r.floorStop;
    if (!(lastDelta >= 0 && (lastDelta < popt.tol || floorStop)) || lastMaxRel < 0) {
        std::printf("tol mode: lastDelta %.3g lastMaxRel %.3g floorStop %d\n", lastDelta, lastMaxRel, (int)floorStop);
        return 1;
    }
    std::printf("tol mode ok: %d iterations, last L1 change %.3g\nOK\n", r.iters, lastDelta);
    return 0;
}
