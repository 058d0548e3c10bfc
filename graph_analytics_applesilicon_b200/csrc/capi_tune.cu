// capi_tune.cu -- batched BFS entry points, batched-selector profiling, and
// the autotuners that replace the reference's parameter sweep scripts
// (scripts/sweep_balanced.sh, sweep_tg.sh, sweep_do.sh).
#include <algorithm>
#include <cstring>
#include <limits>
#include <vector>

#include "bfs.hpp"
#include "capi_util.hpp"
#include "pagerank.hpp"

using namespace gb;

namespace {

gb_bfs_options optsOrDefault(const gb_bfs_options* opt) {
    gb_bfs_options o;
    gb_bfs_default_options(&o);
    if (opt) o = *opt;
    return o;
}

// Device time of one configuration over the sources (first run untimed).
double timeBfs(gb_bfs* h, int variant, const uint32_t* src, int k, const gb_bfs_options& o) {
    auto once = [&]() {
        double t = 0;
        if (variant == GB_BFS_BATCH) {
            h->runBatch(src, k, o, nullptr);
            return h->lastGpuMs;
        }
        for (int i = 0; i < k; ++i) {
            switch (variant) {
                case GB_BFS_BINNED: h->runBinned(src[i], o, nullptr); break;
                case GB_BFS_EDGE: h->runEdge(src[i], o, nullptr); break;
                case GB_BFS_DO: h->runDirOpt(src[i], o, nullptr); break;
                case GB_BFS_PERSISTENT: h->runPersistent(src[i], o, nullptr); break;
                case GB_BFS_NAIVE: h->runNaive(src[i], o, nullptr); break;
                default: h->runVertex(src[i], o, nullptr); break;
            }
            t += h->lastGpuMs;
        }
        return t;
    };
    once();
    return std::min(once(), once());
}

}  // namespace

extern "C" {

int gb_bfs_run_batch(gb_bfs* h, const uint32_t* sources, int k, uint32_t* out_host, const gb_bfs_options* opt,
                     gb_level* trace, size_t cap, size_t* nlev) {
    return guard([&] {
        GB_REQUIRE(h && sources, "null argument");
        gb_bfs_options o = optsOrDefault(opt);
        std::vector<gb_level> tr;
        h->runBatch(sources, k, o, (trace || nlev) ? &tr : nullptr);
        if (out_host) copyDepthsToHost(h, h->bDist.get(), (uint64_t)k * h->n, out_host, h->lastLevels);
        if (nlev) *nlev = tr.size();
        if (trace) {
            std::memcpy(trace, tr.data(), std::min(cap, tr.size()) * sizeof(gb_level));
            if (tr.size() > cap) throw Error(GB_ERR_CAPACITY, "trace capacity too small");
        }
    });
}

// Batched training rows: a level's vertex sets do not depend on the strategy
// that ran the previous levels, and both directions of the batched kernel
// leave the next frontier in the same form, so running the whole batch with
// each strategy forced gives every level's time under every strategy.
int gb_bfs_profile_batch_levels(gb_bfs* h, const uint32_t* sources, int k, const gb_bfs_options* opt, int repeats,
                                float* feats_out, float* times_out, size_t cap, size_t* rows) {
    return guard([&] {
        GB_REQUIRE(h && sources && feats_out && times_out, "null argument");
        gb_bfs_options o = optsOrDefault(opt);
        o.selector = GB_SELECT_RULE;
        std::vector<std::vector<gb_level>> per(GB_NUM_STRATS);
        size_t L = 0;
        for (int s = 0; s < GB_NUM_STRATS; ++s) {
            o.force_strategy = s;
            for (int r = 0; r < std::max(1, repeats); ++r) {
                std::vector<gb_level> tr;
                h->runBatch(sources, k, o, &tr);
                if (per[s].empty()) {
                    per[s] = tr;
                } else {
                    for (size_t i = 0; i < std::min(tr.size(), per[s].size()); ++i)
                        per[s][i].time_ms = std::min(per[s][i].time_ms, tr[i].time_ms);
                }
            }
            if (s == 0) L = per[0].size();
            if (per[s].size() != L) throw Error(GB_ERR_STATE, "level count differs between strategies");
        }
        // features need the unexplored-edge and unreached-vertex counts, which
        // the trace does not carry: approximate them from the frontier totals.
        double edgesSeen = 0, reached = 0;
        size_t out = 0;
        for (size_t i = 0; i < L && out < cap; ++i, ++out) {
            const gb_level& lv = per[0][i];
            selectorFeatures((double)lv.frontier, (double)lv.edges, std::max(0.0, (double)h->m - edgesSeen),
                             std::max(0.0, (double)h->n - reached), (double)h->n, (double)h->m, (double)i,
                             feats_out + out * kSelFeatures);
            for (int s = 0; s < GB_NUM_STRATS; ++s) times_out[out * GB_NUM_STRATS + s] = (float)(per[s][i].time_ms * 1e3);
            edgesSeen += (double)lv.edges;
            reached += (double)lv.frontier;
        }
        if (rows) *rows = out;
    });
}

int gb_bfs_autotune(gb_bfs* h, int variant, const uint32_t* sources, int k, gb_bfs_options* o) {
    return guard([&] {
        GB_REQUIRE(h && o && sources && k > 0, "null argument");
        gb_bfs_options best = *o;
        double bestT = std::numeric_limits<double>::infinity();
        auto consider = [&](gb_bfs_options c) {
            double t = timeBfs(h, variant, sources, k, c);
            if (t < bestT) {
                bestT = t;
                best = c;
            }
        };
        gb_bfs_options c = *o;
        if (variant == GB_BFS_BINNED) {
            for (uint32_t tg : {128u, 256u, 512u})
                for (uint32_t sm : {4u, 8u, 16u, 32u, 64u})
                    for (uint32_t lm : {128u, 256u, 1024u, 4096u}) {
                        c.tg = tg;
                        c.small_max = sm;
                        c.large_min = lm;
                        consider(c);
                    }
        } else if (variant == GB_BFS_EDGE || variant == GB_BFS_DO) {
            for (uint32_t tg : {128u, 256u, 512u, 1024u})
                for (uint32_t ept : {1u, 2u, 4u, 8u, 16u}) {
                    c.tg = tg;
                    c.ept = ept;
                    consider(c);
                }
        } else if (variant == GB_BFS_PERSISTENT || variant == GB_BFS_BATCH) {
            const int sms = deviceSmCount();
            for (uint32_t block : {256u, 512u})
                for (uint32_t hub : {256u, 1024u, 4096u, 16384u}) {
                    c.block = block;
                    c.hub_min = hub;
                    c.grid_blocks = 0;
                    consider(c);
                }
            c = best;  // then the grid size at the best block / hub cut
            for (int quarters : {1, 2, 4, 8}) {  // sms/4, sms/2, sms, 2*sms blocks
                c.grid_blocks = (uint32_t)std::max(1, sms * quarters / 4);
                consider(c);
            }
        } else {
            for (uint32_t tg : {128u, 256u, 512u, 1024u}) {
                c.tg = tg;
                consider(c);
            }
        }
        *o = best;
    });
}

int gb_pr_autotune(gb_pr* h, gb_pr_options* o) {
    return guard([&] {
        GB_REQUIRE(h && o, "null argument");
        gb_pr_options best = *o, c = *o;
        c.iters = 3;
        c.tol = 0;
        double bestT = std::numeric_limits<double>::infinity();
        auto consider = [&]() {
            h->run(GB_PR_PULL_ADAPTIVE, c);
            double t = std::min(h->run(GB_PR_PULL_ADAPTIVE, c).gpu_ms, h->run(GB_PR_PULL_ADAPTIVE, c).gpu_ms);
            if (t < bestT) {
                bestT = t;
                best = *o;
                best.tg = c.tg;
                best.small_max = c.small_max;
                best.large_min = c.large_min;
            }
        };
        for (uint32_t sm : {8u, 16u, 32u, 64u})
            for (uint32_t lm : {256u, 1024u, 2048u, 4096u, 16384u})
                for (uint32_t tg : {128u, 256u, 512u}) {
                    c.small_max = sm;
                    c.large_min = lm;
                    c.tg = tg;
                    consider();
                }
        *o = best;
    });
}

}  // extern "C"
