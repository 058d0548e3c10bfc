// graph_b200.hpp -- C++ host interface over the C ABI (graph_b200.h) with the
// reference's class and method names, so callers of gpu::GpuBfs
// (src/metal/bfs_gpu.hpp:35-105) and gpu::GpuPageRank
// (src/metal/pagerank_gpu.hpp:46-127) switch by changing the include.
// Errors come back as std::runtime_error, as the reference throws.
// Header-only; link with -lgraphb200.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "graph_b200.h"

namespace gpu {

inline void check(int status) {
    if (status != GB_OK) throw std::runtime_error(gb_last_error());
}

// util::BfsLevel (src/util/trace.hpp:7-14) with the strategy that ran.
using BfsLevel = gb_level;

// GpuBfsOptions (src/metal/bfs_gpu.hpp:23-33): same fields and defaults, plus
// the persistent-kernel fields (selector, hub_min, block, ...).
struct GpuBfsOptions : gb_bfs_options {
    GpuBfsOptions() { gb_bfs_default_options(this); }
};

class GpuBfs {
public:
    // GpuBfs(ctx, g): one upload of a symmetric CSR (the host copy may be dropped).
    GpuBfs(const uint32_t* row_ptr, const uint32_t* col_idx, uint64_t n, uint64_t m) : n_(n) {
        check(gb_bfs_create(row_ptr, col_idx, n, m, &h_));
    }
    // From a symmetric .bin file, streamed straight into GPU memory.
    explicit GpuBfs(const char* path) : n_(0) { check(gb_bfs_create_from_file(path, &h_, &n_, nullptr)); }
    ~GpuBfs() {
        gb_csr_free(&g_);
        gb_bfs_destroy(h_);
    }
    // GpuBfs::graph(): the traversed graph as a host CSR, copied back once on
    // first use (the reference's view of shared buffers; see gb_bfs_graph).
    const gb_csr& graph() const {
        if (!g_.row_ptr) check(gb_bfs_graph(h_, &g_));
        return g_;
    }
    GpuBfs(const GpuBfs&) = delete;
    GpuBfs& operator=(const GpuBfs&) = delete;

    void runVertex(uint32_t s, uint32_t* out, const GpuBfsOptions& o, std::vector<BfsLevel>* tr = nullptr) {
        run(GB_BFS_VERTEX, s, out, o, tr);
    }
    void runNaive(uint32_t s, uint32_t* out, const GpuBfsOptions& o, std::vector<BfsLevel>* tr = nullptr) {
        run(GB_BFS_NAIVE, s, out, o, tr);
    }
    void runBinned(uint32_t s, uint32_t* out, const GpuBfsOptions& o, std::vector<BfsLevel>* tr = nullptr) {
        run(GB_BFS_BINNED, s, out, o, tr);
    }
    void runEdge(uint32_t s, uint32_t* out, const GpuBfsOptions& o, std::vector<BfsLevel>* tr = nullptr) {
        run(GB_BFS_EDGE, s, out, o, tr);
    }
    void runDO(uint32_t s, uint32_t* out, const GpuBfsOptions& o, std::vector<BfsLevel>* tr = nullptr) {
        run(GB_BFS_DO, s, out, o, tr);
    }
    // hybrid: the reference's CPU/GPU level split is replaced by the
    // persistent kernel (every level on the GPU, no host round trip).
    void runHybrid(uint32_t s, uint32_t* out, const GpuBfsOptions& o, std::vector<BfsLevel>* tr = nullptr) {
        run(GB_BFS_PERSISTENT, s, out, o, tr);
    }
    void runPersistent(uint32_t s, uint32_t* out, const GpuBfsOptions& o, std::vector<BfsLevel>* tr = nullptr) {
        run(GB_BFS_PERSISTENT, s, out, o, tr);
    }
    // Up to 64 sources in one launch; out: k * n depths, source-major.
    void runBatch(const std::vector<uint32_t>& sources, uint32_t* out, const GpuBfsOptions& o,
                  std::vector<BfsLevel>* tr = nullptr) {
        size_t nl = 0;
        std::vector<BfsLevel> buf(tr ? 4 * n_ + 8 : 0);
        check(gb_bfs_run_batch(h_, sources.data(), (int)sources.size(), out, &o, tr ? buf.data() : nullptr,
                               buf.size(), &nl));
        if (tr) tr->assign(buf.begin(), buf.begin() + (long)nl);
    }
    // One traversal per source in one call (the persistent variant queues them
    // back to back and overlaps each result's copy with the next traversal);
    // out: sources.size() * stride depths (stride 0: one n-entry buffer that
    // ends with the last source's), or null to keep the last result on the device.
    void runMany(int variant, const std::vector<uint32_t>& sources, uint32_t* out, uint64_t stride,
                 const GpuBfsOptions& o, std::vector<float>* gpuMs = nullptr,
                 std::vector<uint32_t>* levels = nullptr) {
        if (gpuMs) gpuMs->assign(sources.size(), 0.0f);
        if (levels) levels->assign(sources.size(), 0);
        check(gb_bfs_run_many(h_, variant, sources.data(), (uint32_t)sources.size(), out, stride, &o,
                              gpuMs ? gpuMs->data() : nullptr, levels ? levels->data() : nullptr));
    }
    void setSelector(int which, const std::vector<float>& params) {
        check(gb_bfs_set_selector(h_, which, params.data(), params.size()));
    }
    // Hub-first adjacency order on the device (same depths, earlier bottom-up exits).
    void hubFirst() { check(gb_bfs_hub_first(h_)); }
    double lastGpuMs() const { return gb_bfs_last_gpu_ms(h_); }
    uint32_t lastLevels() const { return gb_bfs_last_levels(h_); }
    // Device pointer of the last result (GpuBfs::dist() for device-side callers).
    const uint32_t* dist() const { return gb_bfs_device_dist(h_); }
    gb_bfs* handle() { return h_; }

private:
    void run(int v, uint32_t s, uint32_t* out, const GpuBfsOptions& o, std::vector<BfsLevel>* tr) {
        size_t nl = 0;
        std::vector<BfsLevel> buf(tr ? n_ + 8 : 0);
        check(gb_bfs_run(h_, v, s, out, &o, tr ? buf.data() : nullptr, buf.size(), &nl));
        if (tr) tr->insert(tr->end(), buf.begin(), buf.begin() + (long)nl);
    }
    gb_bfs* h_ = nullptr;
    uint64_t n_;
    mutable gb_csr g_{};
};

// PrVariant / parsePrVariant (src/metal/pagerank_gpu.hpp:25, pagerank_gpu.mm:21-28).
enum class PrVariant { Push = GB_PR_PUSH, PullScalar = GB_PR_PULL_SCALAR, PullVector = GB_PR_PULL_VECTOR,
                       PullAdaptive = GB_PR_PULL_ADAPTIVE, PullGS = GB_PR_PULL_GS, PullF64 = GB_PR_PULL_F64,
                       PullBlocked = GB_PR_PULL_BLOCKED };

inline PrVariant parsePrVariant(const std::string& s) {
    if (s == "gpu_push") return PrVariant::Push;
    if (s == "gpu_pull_scalar") return PrVariant::PullScalar;
    if (s == "gpu_pull_vector") return PrVariant::PullVector;
    if (s == "gpu_pull_adaptive") return PrVariant::PullAdaptive;
    if (s == "gpu_pull_gs") return PrVariant::PullGS;
    if (s == "gpu_pull_f64") return PrVariant::PullF64;
    if (s == "gpu_pull_blocked") return PrVariant::PullBlocked;
    throw std::runtime_error("unknown GPU PageRank variant '" + s + "'");
}

struct GpuPrOptions : gb_pr_options {
    GpuPrOptions() { gb_pr_default_options(this); }
};
using GpuPrResult = gb_pr_result;

class GpuPageRank {
public:
    // out_* may be null when the push variant is not needed, in_* when no pull is.
    GpuPageRank(uint64_t n, const uint32_t* out_rp, const uint32_t* out_ci, uint64_t out_m, const uint32_t* in_rp,
                const uint32_t* in_ci, uint64_t in_m, const std::vector<uint32_t>& outdeg)
        : n_(n) {
        check(gb_pr_create(n, out_rp, out_ci, out_m, in_rp, in_ci, in_m, outdeg.data(), &h_));
    }
    ~GpuPageRank() { gb_pr_destroy(h_); }
    GpuPageRank(const GpuPageRank&) = delete;
    GpuPageRank& operator=(const GpuPageRank&) = delete;

    void prepareAdaptive(uint32_t smallMax, uint32_t largeMin) { check(gb_pr_prepare_adaptive(h_, smallMax, largeMin)); }
    void prepareGS(uint32_t pairMaxOutdeg = 2) { check(gb_pr_prepare_gs(h_, pairMaxOutdeg)); }
    size_t gsDeferred() const { return info().deferred; }
    bool gsColored() const { return info().colored; }
    size_t gsSets() const { return info().sets; }
    GpuPrResult run(PrVariant v, const GpuPrOptions& o) {
        GpuPrResult r{};
        check(gb_pr_run(h_, (int)v, &o, &r));
        return r;
    }
    // Ranks in the caller's vertex ids (copied to the host).
    const float* ranks() {
        ranks_.resize(n_);
        check(gb_pr_ranks(h_, ranks_.data()));
        return ranks_.data();
    }
    std::vector<double> ranks64() {
        std::vector<double> r(n_);
        check(gb_pr_ranks_f64(h_, r.data()));
        return r;
    }

private:
    struct Info {
        bool colored;
        size_t sets, deferred;
    };
    Info info() const {
        int c = 0;
        uint64_t s = 0, d = 0;
        check(gb_pr_gs_info(h_, &c, &s, &d));
        return {c != 0, (size_t)s, (size_t)d};
    }
    gb_pr* h_ = nullptr;
    uint64_t n_;
    std::vector<float> ranks_;
};

}  // namespace gpu
