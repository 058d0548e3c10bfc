// capi_bfs.cu -- extern "C" entry points for graphs, BFS, primitives and the
// selector (declared in include/graph_b200.h).  Every entry point catches the
// library's exceptions and returns a gb_status; gb_last_error() holds the text.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <string>

#include "bfs.hpp"
#include "capi_util.hpp"
#include "graph_prep.cuh"
#include "graph_host.hpp"

using namespace gb;

namespace gb {
thread_local std::string g_lastError;

int guardStatus(const std::exception_ptr& ep) {
    try {
        std::rethrow_exception(ep);
    } catch (const Error& e) {
        g_lastError = e.what();
        return e.status;
    } catch (const std::bad_alloc&) {
        g_lastError = "host allocation failed";
        return GB_ERR_OOM;
    } catch (const std::exception& e) {
        g_lastError = e.what();
        return GB_ERR_ARG;
    } catch (...) {
        g_lastError = "unknown error";
        return GB_ERR_ARG;
    }
}

void toC(HostCsr&& g, gb_csr* out) {
    GB_REQUIRE(out, "null output graph");
    out->n = g.n;
    out->m = g.m;
    out->flags = g.flags;
    out->row_ptr = static_cast<uint32_t*>(std::malloc((g.n + 1) * 4));
    out->col_idx = static_cast<uint32_t*>(std::malloc(std::max<uint64_t>(g.m, 1) * 4));
    if (!out->row_ptr || !out->col_idx) {
        std::free(out->row_ptr);
        std::free(out->col_idx);
        out->row_ptr = out->col_idx = nullptr;
        throw std::bad_alloc();
    }
    std::memcpy(out->row_ptr, g.row_ptr.data(), (g.n + 1) * 4);
    if (g.m) std::memcpy(out->col_idx, g.col_idx.data(), g.m * 4);
}

HostCsr fromC(const gb_csr* g) {
    GB_REQUIRE(g && g->row_ptr && (g->m == 0 || g->col_idx), "null graph");
    HostCsr h;
    h.n = g->n;
    h.m = g->m;
    h.flags = g->flags;
    h.row_ptr.assign(g->row_ptr, g->row_ptr + g->n + 1);
    if (g->m) h.col_idx.assign(g->col_idx, g->col_idx + g->m);
    return h;
}
}  // namespace gb

extern "C" {

const char* gb_last_error(void) { return g_lastError.c_str(); }

int gb_device_info(char* name, size_t cap, int* sm_count, int* cc_major, int* cc_minor) {
    return guard([&] {
        int dev = 0;
        GB_CUDA(cudaGetDevice(&dev));
        cudaDeviceProp p{};
        GB_CUDA(cudaGetDeviceProperties(&p, dev));
        if (name && cap) {
            std::strncpy(name, p.name, cap - 1);
            name[cap - 1] = 0;
        }
        if (sm_count) *sm_count = p.multiProcessorCount;
        if (cc_major) *cc_major = p.major;
        if (cc_minor) *cc_minor = p.minor;
        GB_CUDA(cudaFree(nullptr));  // creates the context now rather than inside the first timed call
    });
}

// ------------------------------------------------------------------ graphs

void gb_csr_free(gb_csr* g) {
    if (!g) return;
    if (!freePinnedArray(g->row_ptr)) std::free(g->row_ptr);
    if (!freePinnedArray(g->col_idx)) std::free(g->col_idx);
    g->row_ptr = g->col_idx = nullptr;
    g->n = g->m = 0;
}

int gb_csr_validate(const gb_csr* g, char* msg, size_t cap) {
    return guard([&] {
        std::string e = csrValidate(fromC(g));
        if (msg && cap) {
            std::strncpy(msg, e.c_str(), cap - 1);
            msg[cap - 1] = 0;
        }
    });
}

int gb_csr_from_edges(uint64_t n, const uint32_t* eu, const uint32_t* ev, uint64_t ne, int directed, gb_csr* out) {
    return guard([&] {
        GB_REQUIRE(ne == 0 || (eu && ev), "null edge arrays");
        toC(csrFromEdges(n, eu, ev, ne, directed != 0), out);
    });
}

int gb_csr_transpose(const gb_csr* g, gb_csr* out) { return guard([&] { toC(csrTranspose(fromC(g)), out); }); }
int gb_csr_symmetrize(const gb_csr* g, gb_csr* out) { return guard([&] { toC(csrSymmetrize(fromC(g)), out); }); }
int gb_csr_permute(const gb_csr* g, const uint32_t* perm, gb_csr* out) {
    return guard([&] {
        GB_REQUIRE(perm, "null permutation");
        toC(csrPermute(fromC(g), perm), out);
    });
}
int gb_random_perm(uint64_t n, uint64_t seed, uint32_t* perm) {
    return guard([&] {
        GB_REQUIRE(perm || n == 0, "null output");
        auto p = randomPerm(n, seed);
        if (n) std::memcpy(perm, p.data(), n * 4);
    });
}

int gb_reorder(const gb_csr* g, const char* ordering, uint64_t seed, uint32_t* perm) {
    return guard([&] {
        GB_REQUIRE(g && ordering && (perm || g->n == 0), "null argument");
        const std::string o = ordering;
        if (o != "original" && o != "random")
            GB_REQUIRE(!(g->flags & 1u), "gb_reorder: orderings are computed on a symmetric graph");
        auto p = orderingPerm(fromC(g), o, seed);
        if (g->n) std::memcpy(perm, p.data(), g->n * 4);
    });
}
int gb_locality(const gb_csr* g, double* mean_gap, double* same_block64) {
    return guard([&] {
        GB_REQUIRE(g && mean_gap && same_block64, "null argument");
        locality(fromC(g), mean_gap, same_block64);
    });
}

int gb_gen_path(uint32_t n, gb_csr* out) { return guard([&] { toC(genPath(n), out); }); }
int gb_gen_star(uint32_t leaves, gb_csr* out) { return guard([&] { toC(genStar(leaves), out); }); }
int gb_gen_complete(uint32_t n, gb_csr* out) { return guard([&] { toC(genComplete(n), out); }); }
int gb_gen_two_components(gb_csr* out) { return guard([&] { toC(genTwoComponents(), out); }); }
int gb_gen_empty(uint32_t n, gb_csr* out) { return guard([&] { toC(genEmpty(n), out); }); }
int gb_gen_grid2d(uint32_t rows, uint32_t cols, gb_csr* out) { return guard([&] { toC(genGrid2d(rows, cols), out); }); }
int gb_gen_rmat(uint32_t scale, uint64_t edges, int directed, uint64_t seed, gb_csr* out) {
    return guard([&] { toC(genRmat(scale, edges, directed != 0, seed), out); });
}
int gb_gen_road(uint32_t rows, uint32_t cols, double drop_frac, double diag_frac, uint64_t seed, gb_csr* out) {
    return guard([&] { toC(genRoad(rows, cols, drop_frac, diag_frac, seed), out); });
}
int gb_gen_web(uint32_t n, double out_mean, double zipf_s, uint64_t seed, gb_csr* out) {
    return guard([&] { toC(genWeb(n, out_mean, zipf_s, seed), out); });
}
int gb_gen_chung_lu(uint32_t n, double gamma, double mean_deg, uint64_t seed, gb_csr* out) {
    return guard([&] { toC(genChungLu(n, gamma, mean_deg, seed), out); });
}

int gb_pick_sources(const gb_csr* g, int count, uint64_t seed, int any_component, uint32_t* out, int* k) {
    return guard([&] {
        GB_REQUIRE(g && g->row_ptr, "null graph");
        HostCsr h;
        h.n = g->n;
        h.m = g->m;
        h.row_ptr.assign(g->row_ptr, g->row_ptr + g->n + 1);
        h.col_idx.assign(g->col_idx, g->col_idx + g->m);
        auto s = pickSources(h, count, seed, any_component != 0);
        if (!s.empty()) std::memcpy(out, s.data(), s.size() * 4);
        if (k) *k = (int)s.size();
    });
}

// --------------------------------------------------------------------- BFS

void gb_bfs_default_options(gb_bfs_options* o) {
    if (!o) return;
    *o = gb_bfs_options{};
    o->tg = 256;           // src/metal/bfs_gpu.hpp:23-33 defaults
    o->small_max = 16;
    o->large_min = 256;
    o->ept = 2;
    o->alpha = 15.0;
    o->beta = 18.0;
    o->selector = GB_SELECT_RULE;
    o->force_strategy = -1;
    o->hub_min = 4096;
    o->block = 512;
    o->spin_limit = 0;
    o->grid_blocks = 0;
    o->sel_margin = 0.5f;
    o->in_flight = 1;
}

int gb_bfs_create(const uint32_t* row_ptr, const uint32_t* col_idx, uint64_t n, uint64_t m, gb_bfs** out) {
    return guard([&] {
        GB_REQUIRE(out, "null handle output");
        GB_REQUIRE(row_ptr && (m == 0 || col_idx), "null CSR arrays");
        GB_REQUIRE(n >= 1 && n < 0xFFFFFFFFull, "GpuBfs: graph too large for uint32 vertex ids");
        GB_REQUIRE(m < (1ull << 32), "m must fit in uint32");
        GB_REQUIRE(row_ptr[0] == 0 && row_ptr[n] == m, "row_ptr must start at 0 and end at m");
        auto h = std::make_unique<gb_bfs>();
        h->n = n;
        h->m = m;
        h->hostRowPtr.assign(row_ptr, row_ptr + n + 1);
        h->rowPtr.ensure(n + 1);
        h->colIdx.ensure(m + 4);
        h->dist.ensure(n + 4);
        GB_CUDA(cudaMemcpyAsync(h->rowPtr.get(), row_ptr, (n + 1) * 4, cudaMemcpyHostToDevice, h->stream.s));
        if (m) GB_CUDA(cudaMemcpyAsync(h->colIdx.get(), col_idx, m * 4, cudaMemcpyHostToDevice, h->stream.s));
        checkDeviceCsr(h->rowPtr.get(), h->colIdx.get(), n, m, h->stream.s);  // ids below n before any traversal
        h->stats.ensure(1);
        h->hstats.ensure(1);
        h->hstage.ensure(16);
        GB_CUDA(cudaStreamSynchronize(h->stream.s));
        *out = h.release();
    });
}

int gb_bfs_graph(const gb_bfs* h, gb_csr* out) {
    return guard([&] {
        GB_REQUIRE(h && out, "null argument");
        uint32_t* rp = static_cast<uint32_t*>(std::malloc((h->n + 1) * 4));
        uint32_t* ci = static_cast<uint32_t*>(std::malloc(std::max<uint64_t>(h->m, 1) * 4));
        if (!rp || !ci) {
            std::free(rp);
            std::free(ci);
            throw Error(GB_ERR_OOM, "host allocation failed");
        }
        GB_CUDA(cudaStreamSynchronize(h->stream.s));
        std::memcpy(rp, h->hostRowPtr.data(), (h->n + 1) * 4);
        if (h->m && cudaMemcpy(ci, h->colIdx.get(), h->m * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
            std::free(rp);
            std::free(ci);
            throw Error(GB_ERR_CUDA, "gb_bfs_graph: device-to-host copy failed");
        }
        out->n = h->n;
        out->m = h->m;
        out->flags = h->hubFirst ? (h->flags & ~GB_FLAG_SORTED) : h->flags;
        out->row_ptr = rp;
        out->col_idx = ci;
    });
}

int gb_bfs_hub_first(gb_bfs* h) {
    return guard([&] {
        GB_REQUIRE(h, "null handle");
        hubFirstAdjacency(h->rowPtr.get(), h->colIdx.get(), h->n, h->m, h->stream.s);
        h->hubFirst = true;
    });
}

int gb_bfs_destroy(gb_bfs* h) {
    return guard([&] {
        if (h) {
            cudaStreamSynchronize(h->stream.s);
            delete h;
        }
    });
}

int gb_bfs_run(gb_bfs* h, int variant, uint32_t source, uint32_t* out_host, const gb_bfs_options* opt,
               gb_level* trace, size_t cap, size_t* nlev) {
    return guard([&] {
        GB_REQUIRE(h, "null handle");
        GB_REQUIRE(source < h->n, "source out of range");
        gb_bfs_options o;
        gb_bfs_default_options(&o);
        if (opt) o = *opt;
        validateOptions(o);
        std::vector<gb_level> tr;
        std::vector<gb_level>* tp = (trace || nlev) ? &tr : nullptr;
        switch (variant) {
            case GB_BFS_VERTEX: h->runVertex(source, o, tp); break;
            case GB_BFS_NAIVE: h->runNaive(source, o, tp); break;
            case GB_BFS_BINNED: h->runBinned(source, o, tp); break;
            case GB_BFS_EDGE: h->runEdge(source, o, tp); break;
            case GB_BFS_DO: h->runDirOpt(source, o, tp); break;
            case GB_BFS_PERSISTENT: h->runPersistent(source, o, tp); break;
            default: throw Error(GB_ERR_ARG, "unknown BFS variant " + std::to_string(variant));
        }
        if (out_host) copyDepthsToHost(h, h->dist.get(), h->n, out_host, h->lastLevels);
        if (nlev) *nlev = tr.size();
        if (trace) {
            std::memcpy(trace, tr.data(), std::min(cap, tr.size()) * sizeof(gb_level));
            if (tr.size() > cap) throw Error(GB_ERR_CAPACITY, "trace capacity too small");
        }
    });
}

int gb_bfs_run_many(gb_bfs* h, int variant, const uint32_t* sources, uint32_t count, uint32_t* out_host,
                    uint64_t stride, const gb_bfs_options* opt, float* gpu_ms, uint32_t* levels) {
    return guard([&] {
        GB_REQUIRE(h, "null handle");
        GB_REQUIRE(count == 0 || sources, "null sources");
        GB_REQUIRE(stride == 0 || stride >= h->n, "stride must be 0 or at least n");
        for (uint32_t i = 0; i < count; ++i) GB_REQUIRE(sources[i] < h->n, "source out of range");
        gb_bfs_options o;
        gb_bfs_default_options(&o);
        if (opt) o = *opt;
        validateOptions(o);
        if (variant == GB_BFS_PERSISTENT) {
            h->runPersistentMany(sources, count, out_host, stride, o, gpu_ms, levels);
            return;
        }
        if (variant == GB_BFS_BATCH) {
            h->runBatchMany(sources, count, out_host, stride, o, gpu_ms, levels);
            return;
        }
        for (uint32_t i = 0; i < count; ++i) {
            switch (variant) {
                case GB_BFS_VERTEX: h->runVertex(sources[i], o, nullptr); break;
                case GB_BFS_NAIVE: h->runNaive(sources[i], o, nullptr); break;
                case GB_BFS_BINNED: h->runBinned(sources[i], o, nullptr); break;
                case GB_BFS_EDGE: h->runEdge(sources[i], o, nullptr); break;
                case GB_BFS_DO: h->runDirOpt(sources[i], o, nullptr); break;
                default: throw Error(GB_ERR_ARG, "unknown BFS variant " + std::to_string(variant));
            }
            if (out_host) copyDepthsToHost(h, h->dist.get(), h->n, out_host + (uint64_t)i * stride, h->lastLevels);
            if (gpu_ms) gpu_ms[i] = (float)h->lastGpuMs;
            if (levels) levels[i] = h->lastLevels;
        }
    });
}

double gb_bfs_last_gpu_ms(const gb_bfs* h) { return h ? h->lastGpuMs : -1.0; }
uint32_t gb_bfs_last_levels(const gb_bfs* h) { return h ? h->lastLevels : 0; }
const uint32_t* gb_bfs_device_dist(const gb_bfs* h) { return h ? h->dist.get() : nullptr; }
void* gb_bfs_stream(const gb_bfs* h) { return h ? (void*)h->stream.s : nullptr; }

int gb_bfs_profile_levels(gb_bfs* h, uint32_t source, const gb_bfs_options* opt, int repeats, float* feats_out,
                          float* times_out, size_t cap, size_t* rows) {
    return guard([&] {
        GB_REQUIRE(h && feats_out && times_out, "null argument");
        GB_REQUIRE(source < h->n, "source out of range");
        gb_bfs_options o;
        gb_bfs_default_options(&o);
        if (opt) o = *opt;
        size_t r = h->profileLevels(source, o, repeats < 1 ? 1 : repeats, feats_out, times_out, cap);
        if (rows) *rows = r;
    });
}

// ------------------------------------------------------------- selector

int gb_selector_shape(int* nf, int* nh, int* no) {
    if (nf) *nf = kSelFeatures;
    if (nh) *nh = kSelHidden;
    if (no) *no = kSelOutputs;
    return GB_OK;
}

size_t gb_selector_param_count(void) { return (size_t)kSelParams; }

int gb_bfs_set_selector(gb_bfs* h, int which, const float* params, size_t count) {
    return guard([&] {
        GB_REQUIRE(h, "null handle");
        GB_REQUIRE(which == 0 || which == 1, "selector index must be 0 (single source) or 1 (batched)");
        if (!params) {
            h->selLoaded[which] = false;
            return;
        }
        GB_REQUIRE(count == (size_t)kSelParams, "selector parameter count mismatch");
        h->selParams[which].ensure(kSelParams);
        GB_CUDA(cudaMemcpy(h->selParams[which].get(), params, kSelParams * 4, cudaMemcpyHostToDevice));
        h->selLoaded[which] = true;
    });
}

// ----------------------------------------------------------- primitives

int gb_prim_scan(const uint32_t* in, uint64_t n, uint32_t* out, uint32_t* total) {
    return guard([&] {
        GB_REQUIRE(n == 0 || (in && out), "null argument");
        Stream st;
        ScanScratch scratch;
        DevBuf<uint32_t> d, t;
        d.ensure(n + 1);
        t.ensure(1);
        if (n) GB_CUDA(cudaMemcpyAsync(d.get(), in, n * 4, cudaMemcpyHostToDevice, st.s));
        scanExclusive(d.get(), d.get(), n, t.get(), scratch, st.s);
        if (n) GB_CUDA(cudaMemcpyAsync(out, d.get(), n * 4, cudaMemcpyDeviceToHost, st.s));
        uint32_t tot = 0, errFlag = 0;
        GB_CUDA(cudaMemcpyAsync(&tot, t.get(), 4, cudaMemcpyDeviceToHost, st.s));
        if (n) GB_CUDA(cudaMemcpyAsync(&errFlag, scratch.counters.get() + 1, 4, cudaMemcpyDeviceToHost, st.s));
        GB_CUDA(cudaStreamSynchronize(st.s));
        if (errFlag) throw Error(GB_ERR_TIMEOUT, "scan look-back wait exceeded its limit");
        if (total) *total = tot;
    });
}

int gb_prim_reduce(const uint32_t* in, uint64_t n, uint32_t* sum, uint32_t* max) {
    return guard([&] {
        GB_REQUIRE(n == 0 || in, "null argument");
        Stream st;
        DevBuf<uint32_t> d, r;
        d.ensure(n + 1);
        r.ensure(2);
        GB_CUDA(cudaMemsetAsync(r.get(), 0, 8, st.s));
        if (n) GB_CUDA(cudaMemcpyAsync(d.get(), in, n * 4, cudaMemcpyHostToDevice, st.s));
        reduceSumMax(d.get(), n, r.get(), r.get() + 1, st.s);
        uint32_t res[2];
        GB_CUDA(cudaMemcpyAsync(res, r.get(), 8, cudaMemcpyDeviceToHost, st.s));
        GB_CUDA(cudaStreamSynchronize(st.s));
        if (sum) *sum = res[0];
        if (max) *max = res[1];
    });
}

int gb_prim_queue_bitmap(const uint32_t* queue, uint64_t size, uint64_t n, uint32_t* bitmap_out, uint32_t* queue_out,
                         uint64_t* count_out) {
    return guard([&] {
        GB_REQUIRE(size <= n, "queue longer than n");
        GB_REQUIRE(size == 0 || queue, "null queue");
        Stream st;
        const uint64_t words = (n + 31) / 32;
        DevBuf<uint32_t> q, bm, q2, cnt;
        q.ensure(size + 1);
        bm.ensure(words + 1);
        q2.ensure(n + 1);
        cnt.ensure(1);
        GB_CUDA(cudaMemsetAsync(bm.get(), 0xFF, (words + 1) * 4, st.s));  // must be cleared by the conversion
        GB_CUDA(cudaMemsetAsync(cnt.get(), 0, 4, st.s));
        if (size) GB_CUDA(cudaMemcpyAsync(q.get(), queue, size * 4, cudaMemcpyHostToDevice, st.s));
        queueToBitmap(q.get(), size, bm.get(), n, st.s);
        bitmapToQueue(bm.get(), n, q2.get(), cnt.get(), nullptr, nullptr, st.s);
        uint32_t c = 0;
        GB_CUDA(cudaMemcpyAsync(&c, cnt.get(), 4, cudaMemcpyDeviceToHost, st.s));
        if (bitmap_out && words) GB_CUDA(cudaMemcpyAsync(bitmap_out, bm.get(), words * 4, cudaMemcpyDeviceToHost, st.s));
        GB_CUDA(cudaStreamSynchronize(st.s));
        if (queue_out && c) GB_CUDA(cudaMemcpy(queue_out, q2.get(), (size_t)c * 4, cudaMemcpyDeviceToHost));
        if (count_out) *count_out = c;
    });
}

}  // extern "C"

namespace {
__global__ void barrierTimeoutKernel(unsigned* ctl, unsigned long long spin) {
    // Expects two blocks, runs as one: the wait cannot complete and must give up.
    gb::gridBarrierN(&ctl[0], &ctl[1], spin, 2);
}
}  // namespace

extern "C" int gb_debug_barrier_timeout(uint64_t spin_limit) {
    int st = guard([&] {
        Stream s;
        DevBuf<unsigned> ctl;
        ctl.ensure(2);
        GB_CUDA(cudaMemsetAsync(ctl.get(), 0, 8, s.s));
        barrierTimeoutKernel<<<1, 32, 0, s.s>>>(ctl.get(), spin_limit ? spin_limit : 1000);
        GB_LAUNCH_CHECK();
        unsigned h[2];
        GB_CUDA(cudaMemcpyAsync(h, ctl.get(), 8, cudaMemcpyDeviceToHost, s.s));
        GB_CUDA(cudaStreamSynchronize(s.s));
        if (h[1]) throw Error(GB_ERR_TIMEOUT, "grid barrier gave up after its spin limit (expected)");
    });
    return st;
}
