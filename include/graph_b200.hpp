// graph_b200.hpp -- C++ host interface over the C ABI (graph_b200.h) with the
// reference's class, method, option and result names, so a caller written
// against gpu::GpuBfs (src/metal/bfs_gpu.hpp:23-105) and gpu::GpuPageRank
// (src/metal/pagerank_gpu.hpp:27-127) compiles against this header:
//
//   * GpuBfsOptions / GpuPrOptions / GpuPrResult carry the reference's member
//     names and defaults (smallMax, largeMin, hybridT, cpuThreads, tolRel,
//     inPlace, lastDelta, lastMaxRel, floorStop, gpuMs), plus this library's
//     additions (selector, hubMin, block, gridBlocks, ...);
//   * GpuBfs(ctx, g) / GpuPageRank(ctx, out, in, outdeg, needOut, needIn) take
//     any CSR type with the reference's graph::CSR fields (n, m, row_ptr,
//     col_idx; src/graph/csr.hpp:29-45) and a GpuContext (MetalContext is the
//     reference's spelling of the same thing);
//   * run*(source, out, opt, trace) accept a trace vector of any record type
//     with util::BfsLevel's fields (src/util/trace.hpp:7-14);
//   * dist() is a host buffer owned by the handle: passing it as `out` gets the
//     result there, as the reference's zero-copy buffer does.
//
// Errors come back as std::runtime_error, as the reference throws.
// Header-only; link with -lgraphb200.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "graph_b200.h"

namespace gpu {

inline void check(int status) {
    if (status != GB_OK) throw std::runtime_error(gb_last_error());
}

// The device a handle lives on.  The reference's handles take a MetalContext
// (src/metal/context.hpp); the library works on the calling thread's current
// CUDA device, so the context only records which device that is.
class GpuContext {
public:
    GpuContext() {
        char name[256] = {0};
        check(gb_device_info(name, sizeof name, &sms_, &major_, &minor_));
        name_ = name;
    }
    const std::string& name() const { return name_; }
    int smCount() const { return sms_; }

private:
    std::string name_;
    int sms_ = 0, major_ = 0, minor_ = 0;
};
// The reference's callers construct `gpu::MetalContext ctx;` and pass it on.
using MetalContext = GpuContext;

// util::BfsLevel (src/util/trace.hpp:7-14) with the strategy that ran.
using BfsLevel = gb_level;

// GpuBfsOptions (src/metal/bfs_gpu.hpp:23-33): the reference's fields and
// defaults (tg 256, smallMax 16, largeMin 256, ept 2, alpha 15, beta 18,
// hybridT 0, cpuThreads 0), then the persistent / batched kernels' fields with
// gb_bfs_default_options' defaults.
struct GpuBfsOptions {
    uint32_t tg = 256;
    uint32_t smallMax = 16;
    uint32_t largeMin = 256;
    uint32_t ept = 2;
    double alpha = 15.0;
    double beta = 18.0;
    // hybrid: the reference ran levels with less work than hybridT on the CPU
    // with cpuThreads threads.  Here hybrid runs every level in the persistent
    // kernel (no host round trip per level), so both are accepted and unused.
    uint64_t hybridT = 0;
    int cpuThreads = 0;
    uint32_t selector = GB_SELECT_RULE;  // gb_selector: per-level strategy of the persistent kernels
    int32_t forceStrategy = -1;          // >= 0: every level runs this gb_strategy (profiling)
    uint32_t hubMin = 4096;              // degree at which a vertex is split across blocks
    uint32_t block = 512;                // threads per block of the persistent / batched kernels
    uint64_t spinLimit = 0;              // grid-barrier wait bound in polls (0 = default)
    uint32_t gridBlocks = 0;             // blocks in the persistent grid (0 = every resident block)
    float selMargin = 0.5f;              // learned selector's direction margin (log2 of a time ratio)
    uint32_t inFlight = 1;               // runMany: traversals run at once (1..16), each on a share of the SMs

    gb_bfs_options c() const {
        gb_bfs_options o;
        gb_bfs_default_options(&o);
        o.tg = tg;
        o.small_max = smallMax;
        o.large_min = largeMin;
        o.ept = ept;
        o.alpha = alpha;
        o.beta = beta;
        o.selector = selector;
        o.force_strategy = forceStrategy;
        o.hub_min = hubMin;
        o.block = block;
        o.spin_limit = spinLimit;
        o.grid_blocks = gridBlocks;
        o.sel_margin = selMargin;
        o.in_flight = inFlight;
        return o;
    }
    static GpuBfsOptions fromC(const gb_bfs_options& o) {
        GpuBfsOptions r;
        r.tg = o.tg;
        r.smallMax = o.small_max;
        r.largeMin = o.large_min;
        r.ept = o.ept;
        r.alpha = o.alpha;
        r.beta = o.beta;
        r.selector = o.selector;
        r.forceStrategy = o.force_strategy;
        r.hubMin = o.hub_min;
        r.block = o.block;
        r.spinLimit = o.spin_limit;
        r.gridBlocks = o.grid_blocks;
        r.selMargin = o.sel_margin;
        r.inFlight = o.in_flight;
        return r;
    }
};

// A host CSR read back from the device (GpuBfs::graph()).  It has the
// reference's graph::CSR fields and accessors, and converts to any CSR type
// with the reference's `static T fromVectors(row_ptr, col_idx, flags)`, so
// `g = gbfs->graph();` (src/bench/main.cpp:241) compiles and copies.
struct CsrView {
    uint64_t n = 0, m = 0;
    uint32_t flags = 0;
    const uint32_t* row_ptr = nullptr;
    const uint32_t* col_idx = nullptr;

    bool directed() const { return flags & GB_FLAG_DIRECTED; }
    uint32_t degree(uint32_t v) const { return row_ptr[v + 1] - row_ptr[v]; }
    const uint32_t* begin(uint32_t v) const { return col_idx + row_ptr[v]; }
    const uint32_t* end(uint32_t v) const { return col_idx + row_ptr[v + 1]; }

    template <class T, class = decltype(T::fromVectors(std::vector<uint32_t>(), std::vector<uint32_t>(), 0u))>
    operator T() const {
        return T::fromVectors(std::vector<uint32_t>(row_ptr, row_ptr + n + 1), std::vector<uint32_t>(col_idx, col_idx + m),
                              flags);
    }
};

namespace detail {
// gb_level records into a caller's trace vector of util::BfsLevel-like records.
template <class Level>
void appendLevels(const std::vector<gb_level>& src, size_t k, std::vector<Level>* dst) {
    for (size_t i = 0; i < k; ++i) {
        Level x{};
        x.level = src[i].level;
        x.frontier = src[i].frontier;
        x.edges = src[i].edges;
        x.direction = src[i].direction;
        x.device = src[i].device;
        x.time_ms = src[i].time_ms;
        dst->push_back(x);
    }
}
inline void appendLevels(const std::vector<gb_level>& src, size_t k, std::vector<gb_level>* dst) {
    dst->insert(dst->end(), src.begin(), src.begin() + (long)k);
}
}  // namespace detail

class GpuBfs {
public:
    // GpuBfs(ctx, g) (src/metal/bfs_gpu.hpp:37): one upload of a symmetric CSR;
    // Csr is any type with the reference's n, m, row_ptr, col_idx fields.
    template <class Csr, class = decltype(std::declval<const Csr&>().row_ptr)>
    GpuBfs(GpuContext&, const Csr& g) : GpuBfs(g.row_ptr, g.col_idx, g.n, g.m) {}
    GpuBfs(const uint32_t* row_ptr, const uint32_t* col_idx, uint64_t n, uint64_t m) : n_(n) {
        check(gb_bfs_create(row_ptr, col_idx, n, m, &h_));
    }
    // From a symmetric .bin file, streamed straight into GPU memory.
    explicit GpuBfs(const char* path) : n_(0) { check(gb_bfs_create_from_file(path, &h_, &n_, nullptr)); }
    ~GpuBfs() {
        gb_csr_free(&g_);
        gb_bfs_destroy(h_);
    }
    GpuBfs(const GpuBfs&) = delete;
    GpuBfs& operator=(const GpuBfs&) = delete;

    // graph(): the traversed graph as a host CSR, copied back once on first
    // use (the reference returns a view of its unified-memory buffers).
    const CsrView& graph() const {
        if (!g_.row_ptr) {
            check(gb_bfs_graph(h_, &g_));
            view_ = CsrView{g_.n, g_.m, g_.flags, g_.row_ptr, g_.col_idx};
        }
        return view_;
    }
    // dist(): a host buffer of n depths owned by the handle.  Passing it as
    // `out` puts the result there (the reference's zero-copy use); it holds
    // whatever the last run that was given it wrote.
    uint32_t* dist() {
        if (hostDist_.size() != n_) hostDist_.assign(n_, 0xFFFFFFFFu);
        return hostDist_.data();
    }
    // The device copy of the last result (n depths), for device-side callers.
    const uint32_t* deviceDist() const { return gb_bfs_device_dist(h_); }

    // run*(source, out, opt, trace) (src/metal/bfs_gpu.hpp:43-66).  out: n host
    // depths, or nullptr to keep the result on the device (deviceDist()).
    void runVertex(uint32_t s, uint32_t* out, const GpuBfsOptions& o, std::vector<BfsLevel>* tr = nullptr) {
        run(GB_BFS_VERTEX, s, out, o, tr);
    }
    template <class Level>
    void runVertex(uint32_t s, uint32_t* out, const GpuBfsOptions& o, std::vector<Level>* tr) {
        run(GB_BFS_VERTEX, s, out, o, tr);
    }
    void runNaive(uint32_t s, uint32_t* out, const GpuBfsOptions& o, std::vector<BfsLevel>* tr = nullptr) {
        run(GB_BFS_NAIVE, s, out, o, tr);
    }
    template <class Level>
    void runNaive(uint32_t s, uint32_t* out, const GpuBfsOptions& o, std::vector<Level>* tr) {
        run(GB_BFS_NAIVE, s, out, o, tr);
    }
    void runBinned(uint32_t s, uint32_t* out, const GpuBfsOptions& o, std::vector<BfsLevel>* tr = nullptr) {
        run(GB_BFS_BINNED, s, out, o, tr);
    }
    template <class Level>
    void runBinned(uint32_t s, uint32_t* out, const GpuBfsOptions& o, std::vector<Level>* tr) {
        run(GB_BFS_BINNED, s, out, o, tr);
    }
    void runEdge(uint32_t s, uint32_t* out, const GpuBfsOptions& o, std::vector<BfsLevel>* tr = nullptr) {
        run(GB_BFS_EDGE, s, out, o, tr);
    }
    template <class Level>
    void runEdge(uint32_t s, uint32_t* out, const GpuBfsOptions& o, std::vector<Level>* tr) {
        run(GB_BFS_EDGE, s, out, o, tr);
    }
    void runDO(uint32_t s, uint32_t* out, const GpuBfsOptions& o, std::vector<BfsLevel>* tr = nullptr) {
        run(GB_BFS_DO, s, out, o, tr);
    }
    template <class Level>
    void runDO(uint32_t s, uint32_t* out, const GpuBfsOptions& o, std::vector<Level>* tr) {
        run(GB_BFS_DO, s, out, o, tr);
    }
    // hybrid: the reference's CPU/GPU level split is replaced by the
    // persistent kernel (every level on the GPU, no host round trip), so
    // hybridT and cpuThreads do not change what runs.
    void runHybrid(uint32_t s, uint32_t* out, const GpuBfsOptions& o, std::vector<BfsLevel>* tr = nullptr) {
        run(GB_BFS_PERSISTENT, s, out, o, tr);
    }
    template <class Level>
    void runHybrid(uint32_t s, uint32_t* out, const GpuBfsOptions& o, std::vector<Level>* tr) {
        run(GB_BFS_PERSISTENT, s, out, o, tr);
    }
    void runPersistent(uint32_t s, uint32_t* out, const GpuBfsOptions& o, std::vector<BfsLevel>* tr = nullptr) {
        run(GB_BFS_PERSISTENT, s, out, o, tr);
    }
    template <class Level>
    void runPersistent(uint32_t s, uint32_t* out, const GpuBfsOptions& o, std::vector<Level>* tr) {
        run(GB_BFS_PERSISTENT, s, out, o, tr);
    }
    // Up to 64 sources in one launch; out: k * n depths, source-major.
    void runBatch(const std::vector<uint32_t>& sources, uint32_t* out, const GpuBfsOptions& o,
                  std::vector<BfsLevel>* tr = nullptr) {
        size_t nl = 0;
        std::vector<BfsLevel> buf(tr ? 4 * n_ + 8 : 0);
        const gb_bfs_options c = o.c();
        check(gb_bfs_run_batch(h_, sources.data(), (int)sources.size(), out, &c, tr ? buf.data() : nullptr,
                               buf.size(), &nl));
        if (tr) tr->assign(buf.begin(), buf.begin() + (long)nl);
    }
    // One traversal per source in one call (the persistent variant queues them
    // back to back and overlaps each result's copy with the next traversal;
    // GB_BFS_BATCH runs them 64 to a launch of the batched kernel);
    // out: sources.size() * stride depths (stride 0: one n-entry buffer that
    // ends with the last source's), or null to keep the last result on the device.
    void runMany(int variant, const std::vector<uint32_t>& sources, uint32_t* out, uint64_t stride,
                 const GpuBfsOptions& o, std::vector<float>* gpuMs = nullptr,
                 std::vector<uint32_t>* levels = nullptr) {
        if (gpuMs) gpuMs->assign(sources.size(), 0.0f);
        if (levels) levels->assign(sources.size(), 0);
        const gb_bfs_options c = o.c();
        check(gb_bfs_run_many(h_, variant, sources.data(), (uint32_t)sources.size(), out, stride, &c,
                              gpuMs ? gpuMs->data() : nullptr, levels ? levels->data() : nullptr));
    }
    void setSelector(int which, const std::vector<float>& params) {
        check(gb_bfs_set_selector(h_, which, params.data(), params.size()));
    }
    // Block size, grid size and hub cut (persistent / batched) or the level
    // kernels' cuts, timed on `sources` (the reference's scripts/sweep_*.sh).
    GpuBfsOptions autotune(int variant, const std::vector<uint32_t>& sources, const GpuBfsOptions& start) {
        gb_bfs_options c = start.c();
        check(gb_bfs_autotune(h_, variant, sources.data(), (int)sources.size(), &c));
        GpuBfsOptions r = GpuBfsOptions::fromC(c);
        r.hybridT = start.hybridT;
        r.cpuThreads = start.cpuThreads;
        return r;
    }
    // Hub-first adjacency order on the device (same depths, earlier bottom-up exits).
    void hubFirst() { check(gb_bfs_hub_first(h_)); }
    double lastGpuMs() const { return gb_bfs_last_gpu_ms(h_); }
    uint32_t lastLevels() const { return gb_bfs_last_levels(h_); }
    gb_bfs* handle() { return h_; }

private:
    template <class Level>
    void run(int v, uint32_t s, uint32_t* out, const GpuBfsOptions& o, std::vector<Level>* tr) {
        size_t nl = 0;
        std::vector<gb_level> buf(tr ? n_ + 8 : 0);
        const gb_bfs_options c = o.c();
        check(gb_bfs_run(h_, v, s, out, &c, tr ? buf.data() : nullptr, buf.size(), &nl));
        if (tr) detail::appendLevels(buf, nl, tr);
    }
    gb_bfs* h_ = nullptr;
    uint64_t n_;
    std::vector<uint32_t> hostDist_;
    mutable gb_csr g_{};
    mutable CsrView view_{};
};

// PrVariant / parsePrVariant (src/metal/pagerank_gpu.hpp:25, pagerank_gpu.mm:21-28),
// plus the FP64 oracle pull and the shared-memory blocked pull.
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

// GpuPrOptions (src/metal/pagerank_gpu.hpp:27-36): same fields and defaults.
struct GpuPrOptions {
    float damping = 0.85f;
    int iters = 20;           // fixed mode: iterations; tol mode: cap
    double tol = 0;           // > 0: stop when the L1 change < tol
    double tolRel = 0;        // > 0 (tol mode): also require max relative change < tolRel
    uint32_t tg = 256;        // threads per block of the main kernels
    uint32_t smallMax = 16;   // adaptive: in-degree < smallMax -> small class
    uint32_t largeMin = 256;  // adaptive: in-degree >= largeMin -> block per vertex
    bool inPlace = false;     // any pull variant: update contributions in place

    gb_pr_options c() const {
        gb_pr_options o;
        gb_pr_default_options(&o);
        o.damping = damping;
        o.iters = iters;
        o.tol = tol;
        o.tol_rel = tolRel;
        o.tg = tg;
        o.small_max = smallMax;
        o.large_min = largeMin;
        o.inplace = inPlace ? 1u : 0u;
        return o;
    }
    static GpuPrOptions fromC(const gb_pr_options& o) {
        GpuPrOptions r;
        r.damping = o.damping;
        r.iters = o.iters;
        r.tol = o.tol;
        r.tolRel = o.tol_rel;
        r.tg = o.tg;
        r.smallMax = o.small_max;
        r.largeMin = o.large_min;
        r.inPlace = o.inplace != 0;
        return r;
    }
};

// GpuPrResult (src/metal/pagerank_gpu.hpp:38-44): same fields.
struct GpuPrResult {
    int iters = 0;
    double lastDelta = -1;   // tol mode: L1 change of the last iteration (FP64)
    double lastMaxRel = -1;  // tol mode: max relative change of the last iteration
    bool floorStop = false;  // tol mode: stopped because the L1 change stagnated above tol
    double gpuMs = 0;        // device time of the run
};

class GpuPageRank {
public:
    // GpuPageRank(ctx, out, in, outdeg, needOut, needIn)
    // (src/metal/pagerank_gpu.hpp:49-50): `out` may be empty when !needOut,
    // `in` when !needIn; Csr is any type with graph::CSR's fields.
    template <class Csr, class = decltype(std::declval<const Csr&>().row_ptr)>
    GpuPageRank(GpuContext&, const Csr& out, const Csr& in, const std::vector<uint32_t>& outdeg, bool needOut,
                bool needIn)
        : GpuPageRank(outdeg.size(), needOut ? out.row_ptr : nullptr, needOut ? out.col_idx : nullptr,
                      needOut ? out.m : 0, needIn ? in.row_ptr : nullptr, needIn ? in.col_idx : nullptr,
                      needIn ? in.m : 0, outdeg) {}
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
        const gb_pr_options c = o.c();
        gb_pr_result r{};
        check(gb_pr_run(h_, (int)v, &c, &r));
        GpuPrResult out;
        out.iters = r.iters;
        out.lastDelta = r.last_delta;
        out.lastMaxRel = r.last_max_rel;
        out.floorStop = r.floor_stop != 0;
        out.gpuMs = r.gpu_ms;
        return out;
    }
    // Degree-class cut points and block size timed on this graph.
    GpuPrOptions autotune(const GpuPrOptions& start) {
        gb_pr_options c = start.c();
        check(gb_pr_autotune(h_, &c));
        return GpuPrOptions::fromC(c);
    }
    // Ranks in the caller's vertex ids (copied to the host on each call).
    const float* ranks() const {
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
    mutable std::vector<float> ranks_;
};

}  // namespace gpu
