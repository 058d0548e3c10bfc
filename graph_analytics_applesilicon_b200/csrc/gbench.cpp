// gbench -- benchmark + validation CLI with the reference's surface
// (src/bench/main.cpp:1-26): same flags, variant names, methodology
// (sources from the largest component, seed 1; 2 warm-ups; per source
// 1 warm-up + 5 timed trials; harmonic-mean GTEPS), CSV schema and exit codes
// (exception -> 1, unknown variant -> 2, validation failure -> 1).
//
//   gbench --graph file.bin|synth:NAME --algo bfs --variant V [--validate] ...
//   gbench --graph ... --algo pr --variant V [--iters 20 | --tol 1e-6] ...
//
// GPU variants call the B200 library through include/graph_b200.hpp.  New:
// gpu_do_persistent (and hybrid, which maps to it), --selector rule|learned,
// --batch 64 (sources in batches of up to 64 per launch), --block, --hub-min, --grid-blocks, --sel-margin,
// --hub-first (adjacency lists re-sorted hub-first on the device),
// gpu_pull_f64, gpu_pull_blocked, and the benchmark graphs synth:rmat22, synth:road1400,
// synth:web875k, synth:chunglu3m.  Graph preparation (symmetrize, transpose,
// permute, source picking) runs on the GPU; --host-prep keeps it on the host.
// cpu_serial / cpu_omp / cpu_do are this
// program's own CPU implementations of the reference's CPU variants
// (src/cpu/bfs_cpu.cpp, src/cpu/pagerank_cpu.cpp); --validate uses cpu_serial.
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <fstream>
#include <functional>
#include <map>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <string>
#include <sys/stat.h>
#include <unistd.h>
#include <vector>

#include "graph_b200.hpp"

namespace {

constexpr uint32_t kUnreached = 0xFFFFFFFFu;

struct Args {  // "--k v", "--k=v", bare "--flag" (src/util/args.hpp:11-47)
    std::map<std::string, std::string> kv;
    Args(int argc, char** argv) {
        for (int i = 1; i < argc; ++i) {
            std::string a = argv[i];
            if (a.rfind("--", 0) != 0) continue;
            a = a.substr(2);
            auto eq = a.find('=');
            if (eq != std::string::npos) kv[a.substr(0, eq)] = a.substr(eq + 1);
            else if (i + 1 < argc && std::string(argv[i + 1]).rfind("--", 0) != 0) kv[a] = argv[++i];
            else kv[a] = "";
        }
    }
    bool has(const std::string& k) const { return kv.count(k) != 0; }
    std::string get(const std::string& k, const std::string& d = "") const {
        auto it = kv.find(k);
        return it == kv.end() ? d : it->second;
    }
    long long getInt(const std::string& k, long long d) const {
        auto it = kv.find(k);
        return (it == kv.end() || it->second.empty()) ? d : std::atoll(it->second.c_str());
    }
    double getDouble(const std::string& k, double d) const {
        auto it = kv.find(k);
        return (it == kv.end() || it->second.empty()) ? d : std::atof(it->second.c_str());
    }
};

struct Graph {  // owning host CSR
    gb_csr c{};
    Graph() = default;
    Graph(Graph&& o) noexcept : c(o.c) { o.c = gb_csr{}; }
    Graph& operator=(Graph&& o) noexcept {
        if (this != &o) {
            gb_csr_free(&c);
            c = o.c;
            o.c = gb_csr{};
        }
        return *this;
    }
    ~Graph() { gb_csr_free(&c); }
    uint64_t n() const { return c.n; }
    uint64_t m() const { return c.m; }
    bool directed() const { return c.flags & GB_FLAG_DIRECTED; }
    uint32_t degree(uint64_t v) const { return c.row_ptr[v + 1] - c.row_ptr[v]; }
};

template <class F>
Graph make(F f) {
    Graph g;
    gpu::check(f(&g.c));
    return g;
}

double msSince(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// Graph preparation runs on the GPU (gb_csr_*_gpu, identical results) unless
// --host-prep is given; symmetrize of a directed list with repeated entries
// (no duplicate-free flag) keeps the host merge, which defines that case.
bool gHostPrep = false;
int prepSymmetrize(const gb_csr* g, gb_csr* out) {
    const bool gpuOk = !(g->flags & 1u) || (g->flags & 4u);
    return (!gHostPrep && gpuOk) ? gb_csr_symmetrize_gpu(g, out) : gb_csr_symmetrize(g, out);
}
int prepTranspose(const gb_csr* g, gb_csr* out) {
    return gHostPrep ? gb_csr_transpose(g, out) : gb_csr_transpose_gpu(g, out);
}
int prepPermute(const gb_csr* g, const uint32_t* perm, gb_csr* out) {
    return gHostPrep ? gb_csr_permute(g, perm, out) : gb_csr_permute_gpu(g, perm, out);
}
int prepReorder(const gb_csr* g, const char* ordering, uint64_t seed, uint32_t* perm) {
    return gHostPrep ? gb_reorder(g, ordering, seed, perm) : gb_reorder_gpu(g, ordering, seed, perm);
}
int prepPickSources(const gb_csr* g, int count, uint64_t seed, int any, uint32_t* out, int* k) {
    return (gHostPrep || (g->flags & 1u)) ? gb_pick_sources(g, count, seed, any, out, k)
                                          : gb_pick_sources_gpu(g, count, seed, any, out, k);
}

Graph loadGraph(const std::string& spec, std::string& name) {
    if (spec.rfind("synth:", 0) == 0) {
        name = spec.substr(6);
        if (name == "path1000") return make([](gb_csr* o) { return gb_gen_path(1000, o); });
        if (name == "star100k") return make([](gb_csr* o) { return gb_gen_star(100000, o); });
        if (name == "complete200") return make([](gb_csr* o) { return gb_gen_complete(200, o); });
        if (name == "two_components") return make([](gb_csr* o) { return gb_gen_two_components(o); });
        if (name == "empty1000") return make([](gb_csr* o) { return gb_gen_empty(1000, o); });
        if (name == "grid100x100") return make([](gb_csr* o) { return gb_gen_grid2d(100, 100, o); });
        if (name == "rmat12") return make([](gb_csr* o) { return gb_gen_rmat(12, 16u << 12, 0, 42, o); });
        if (name == "rmat12_directed") return make([](gb_csr* o) { return gb_gen_rmat(12, 16u << 12, 1, 43, o); });
        if (name == "rmat22") {  // the R-MAT scale-22 benchmark graph, ids permuted (seed 1)
            Graph g = make([](gb_csr* o) { return gb_gen_rmat(22, 35651584ull, 0, 22, o); });
            std::vector<uint32_t> p(g.n());
            gpu::check(gb_random_perm(g.n(), 1, p.data()));
            return make([&](gb_csr* o) { return prepPermute(&g.c, p.data(), o); });
        }
        if (name == "road1400") return make([](gb_csr* o) { return gb_gen_road(1400, 1400, 0.04, 0.005, 1400, o); });
        if (name == "web875k") return make([](gb_csr* o) { return gb_gen_web(875000, 5.8, 2.1, 875, o); });
        if (name == "chunglu3m") return make([](gb_csr* o) { return gb_gen_chung_lu(3070000, 2.2, 76.0, 307, o); });
        throw std::runtime_error("unknown synthetic graph '" + name + "'");
    }
    size_t s = spec.find_last_of('/');
    name = spec.substr(s == std::string::npos ? 0 : s + 1);
    name = name.substr(0, name.find('.'));
    return make([&](gb_csr* o) { return gb_csr_load(spec.c_str(), o); });
}

// ------------------------------------------------------------- CPU variants

void cpuBfsSerial(const Graph& g, uint32_t src, uint32_t* dist) {
    std::fill(dist, dist + g.n(), kUnreached);
    std::vector<uint32_t> q(g.n());
    size_t head = 0, tail = 0;
    dist[src] = 0;
    q[tail++] = src;
    while (head < tail) {
        uint32_t u = q[head++];
        for (uint32_t i = g.c.row_ptr[u]; i < g.c.row_ptr[u + 1]; ++i) {
            uint32_t w = g.c.col_idx[i];
            if (dist[w] == kUnreached) {
                dist[w] = dist[u] + 1;
                q[tail++] = w;
            }
        }
    }
}

// cpu_omp's loop schedule (--schedule, src/cpu/bfs_cpu.hpp:16-19): the same
// three choices and CSV names as the reference.
enum class Schedule { Static, Dynamic64, Guided };

Schedule parseSchedule(const std::string& s) {
    if (s == "static") return Schedule::Static;
    if (s == "dynamic" || s == "dynamic,64" || s == "dynamic/64") return Schedule::Dynamic64;
    if (s == "guided") return Schedule::Guided;
    throw std::runtime_error("unknown schedule '" + s + "' (static | dynamic,64 | guided)");
}

const char* scheduleName(Schedule s) {
    return s == Schedule::Static ? "static" : s == Schedule::Guided ? "guided" : "dynamic/64";
}

void setSchedule(Schedule s) {
    if (s == Schedule::Static) omp_set_schedule(omp_sched_static, 0);
    else if (s == Schedule::Guided) omp_set_schedule(omp_sched_guided, 0);
    else omp_set_schedule(omp_sched_dynamic, 64);
}

// Level-synchronous top-down with CAS claims; per-thread buffers are
// concatenated after the parallel loop.  The loop takes the schedule set by
// setSchedule (dynamic,64 unless cpu_omp's --schedule says otherwise).
uint64_t cpuTopDown(const Graph& g, uint32_t* dist, const std::vector<uint32_t>& front, std::vector<uint32_t>& next,
                    uint32_t d, int nt, uint64_t* scout) {
    std::vector<std::vector<uint32_t>> parts(nt);
    uint64_t sc = 0;
#pragma omp parallel num_threads(nt) reduction(+ : sc)
    {
        std::vector<uint32_t>& local = parts[omp_get_thread_num()];
#pragma omp for schedule(runtime)
        for (int64_t i = 0; i < (int64_t)front.size(); ++i) {
            uint32_t u = front[i];
            for (uint32_t k = g.c.row_ptr[u]; k < g.c.row_ptr[u + 1]; ++k) {
                uint32_t w = g.c.col_idx[k];
                uint32_t cur = __atomic_load_n(&dist[w], __ATOMIC_RELAXED);
                if (cur == kUnreached && __atomic_compare_exchange_n(&dist[w], &cur, d, false, __ATOMIC_RELAXED,
                                                                     __ATOMIC_RELAXED)) {
                    local.push_back(w);
                    sc += g.degree(w);
                }
            }
        }
    }
    next.clear();
    for (auto& p : parts) next.insert(next.end(), p.begin(), p.end());
    if (scout) *scout = sc;
    return next.size();
}

void cpuBfsOmp(const Graph& g, uint32_t src, uint32_t* dist, int nt, Schedule schedule,
               std::vector<gpu::BfsLevel>* tr) {
    setSchedule(schedule);
    std::fill(dist, dist + g.n(), kUnreached);
    dist[src] = 0;
    std::vector<uint32_t> front{src}, next;
    for (uint32_t level = 0; !front.empty(); ++level) {
        auto t0 = std::chrono::steady_clock::now();
        uint64_t edges = 0;
        for (uint32_t u : front) edges += g.degree(u);
        cpuTopDown(g, dist, front, next, level + 1, nt, nullptr);
        if (tr) tr->push_back({level, 'T', 'C', 1, 0, front.size(), edges, msSince(t0)});
        front.swap(next);
    }
}

// Direction-optimizing BFS: the rule of src/cpu/bfs_cpu.cpp:227-283.
void cpuBfsDO(const Graph& g, uint32_t src, uint32_t* dist, double alpha, double beta, int nt,
              std::vector<gpu::BfsLevel>* tr) {
    setSchedule(Schedule::Dynamic64);
    const uint64_t n = g.n();
    std::fill(dist, dist + n, kUnreached);
    dist[src] = 0;
    std::vector<uint32_t> q{src}, nq;
    std::vector<uint64_t> front((n + 63) / 64 + 1), next(front.size());
    uint64_t toCheck = g.m(), scout = g.degree(src);
    uint32_t level = 0;
    while (!q.empty()) {
        if ((double)scout > (double)toCheck / alpha) {
            std::fill(front.begin(), front.end(), 0);
            for (uint32_t v : q) front[v >> 6] |= 1ull << (v & 63);
            uint64_t awake = q.size(), old;
            do {
                auto t0 = std::chrono::steady_clock::now();
                old = awake;
                std::fill(next.begin(), next.end(), 0);
                uint64_t found = 0, exam = 0;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1024) reduction(+ : found, exam)
                for (int64_t v = 0; v < (int64_t)n; ++v) {
                    if (dist[v] != kUnreached) continue;
                    uint32_t b = g.c.row_ptr[v], e = g.c.row_ptr[v + 1], p = b;
                    for (; p < e; ++p) {
                        uint32_t u = g.c.col_idx[p];
                        if ((front[u >> 6] >> (u & 63)) & 1) {
                            dist[v] = level + 1;
                            __atomic_fetch_or(&next[v >> 6], 1ull << (v & 63), __ATOMIC_RELAXED);
                            ++found;
                            ++p;
                            break;
                        }
                    }
                    exam += p - b;
                }
                if (tr) tr->push_back({level, 'B', 'C', 4, 0, old, exam, msSince(t0)});
                awake = found;
                front.swap(next);
                ++level;
            } while (awake >= old || (double)awake > (double)n / beta);
            q.clear();
            for (uint64_t w = 0; w < front.size(); ++w)
                for (uint64_t x = front[w]; x; x &= x - 1) {
                    uint64_t v = w * 64 + __builtin_ctzll(x);
                    if (v < n) q.push_back((uint32_t)v);
                }
            scout = 1;
        } else {
            auto t0 = std::chrono::steady_clock::now();
            toCheck -= std::min(toCheck, scout);
            uint64_t edges = 0;
            for (uint32_t u : q) edges += g.degree(u);
            cpuTopDown(g, dist, q, nq, level + 1, nt, &scout);
            if (tr) tr->push_back({level, 'T', 'C', 1, 0, q.size(), edges, msSince(t0)});
            q.swap(nq);
            ++level;
        }
    }
}

// FP64 Jacobi PageRank (src/cpu/pagerank_cpu.cpp:20-53); returns iterations.
int cpuPagerank(const Graph& in, const std::vector<uint32_t>& od, std::vector<double>& r, int iters, double tol,
                int nt, double* lastDelta) {
    const uint64_t n = in.n();
    r.assign(n, n ? 1.0 / n : 0.0);
    if (!n) return 0;
    const double d = 0.85, base = (1 - d) / n;
    std::vector<double> contrib(n), next(n);
    int it = 0;
    for (; it < iters;) {
        double dang = 0;
#pragma omp parallel for num_threads(nt) reduction(+ : dang)
        for (int64_t u = 0; u < (int64_t)n; ++u) {
            if (od[u]) contrib[u] = r[u] / od[u];
            else {
                contrib[u] = 0;
                dang += r[u];
            }
        }
        const double add = base + d * dang / n;
        double delta = 0;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 256) reduction(+ : delta)
        for (int64_t v = 0; v < (int64_t)n; ++v) {
            double s = 0;
            for (uint32_t i = in.c.row_ptr[v]; i < in.c.row_ptr[v + 1]; ++i) s += contrib[in.c.col_idx[i]];
            next[v] = add + d * s;
            delta += std::fabs(next[v] - r[v]);
        }
        r.swap(next);
        ++it;
        if (lastDelta) *lastDelta = delta;
        if (tol > 0 && delta < tol) break;
    }
    return it;
}

struct PrCheck {
    double l1 = 0, maxRelTop = 0, sum = 0;
    bool ok() const { return l1 < 1e-4 && maxRelTop < 1e-3 && std::fabs(sum - 1.0) < 1e-4; }
};

template <class T>
PrCheck checkRanks(const std::vector<double>& ref, const T* got) {  // src/cpu/pagerank_cpu.hpp:42-60
    PrCheck c;
    const size_t n = ref.size();
    for (size_t v = 0; v < n; ++v) {
        c.l1 += std::fabs(ref[v] - (double)got[v]);
        c.sum += (double)got[v];
    }
    std::vector<uint32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0u);
    size_t k = std::min<size_t>(1000, n);
    std::partial_sort(idx.begin(), idx.begin() + k, idx.end(), [&](uint32_t a, uint32_t b) { return ref[a] > ref[b]; });
    for (size_t i = 0; i < k; ++i)
        c.maxRelTop = std::max(c.maxRelTop, std::fabs(ref[idx[i]] - (double)got[idx[i]]) / ref[idx[i]]);
    return c;
}

bool gsNoWorse(const PrCheck& gs, const PrCheck& j) {  // src/cpu/pagerank_cpu.hpp:80-84
    const double b = std::max(1e-4, j.l1);
    return gs.l1 <= b && std::fabs(gs.sum - 1.0) <= b && gs.maxRelTop <= std::max(1e-3, j.maxRelTop * (1 + 1e-4));
}

double median(std::vector<double> v) {
    std::sort(v.begin(), v.end());
    size_t k = v.size();
    return k == 0 ? 0 : (k % 2 ? v[k / 2] : 0.5 * (v[k / 2 - 1] + v[k / 2]));
}

bool fileExists(const std::string& p) {
    struct stat st;
    return stat(p.c_str(), &st) == 0;
}

std::string timestamp() {
    std::time_t t = std::time(nullptr);
    char b[32];
    std::strftime(b, sizeof b, "%Y-%m-%dT%H:%M:%S", std::localtime(&t));
    return b;
}

// Short hash of the checkout the binary runs from, "+" when tracked files
// are modified, "unknown" outside a git checkout (the CSV's git_commit field,
// src/util/sysinfo.hpp:27-42).
std::string gitCommit() {
    auto run = [](const char* cmd) {
        std::string out;
        if (FILE* p = popen(cmd, "r")) {
            char buf[128];
            while (std::fgets(buf, sizeof buf, p)) out += buf;
            pclose(p);
        }
        while (!out.empty() && std::isspace((unsigned char)out.back())) out.pop_back();
        return out;
    };
    std::string h = run("git rev-parse --short HEAD 2>/dev/null");
    if (h.empty()) return "unknown";
    if (!run("git status --porcelain --untracked-files=no 2>/dev/null").empty()) h += "+";
    return h;
}

double loadAverage1() {
    double l[3];
    return getloadavg(l, 3) > 0 ? l[0] : -1;
}

std::string chipName() {
    char name[256] = "unknown";
    int sms = 0, ma = 0, mi = 0;
    if (gb_device_info(name, sizeof name, &sms, &ma, &mi) != GB_OK) return "unknown";
    return name;
}

std::vector<float> loadSelector(const std::string& path) {
    std::vector<float> p(gb_selector_param_count());
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open selector parameters " + path);
    bool ok = std::fread(p.data(), 4, p.size(), f) == p.size();
    std::fclose(f);
    if (!ok) throw std::runtime_error(path + ": wrong size for the selector parameters");
    return p;
}

std::string exeDir() {
    char buf[4096];
    ssize_t k = readlink("/proc/self/exe", buf, sizeof buf - 1);
    if (k <= 0) return ".";
    buf[k] = 0;
    std::string s(buf);
    return s.substr(0, s.find_last_of('/'));
}

const std::vector<std::string> kVariants = {"cpu_serial", "cpu_omp", "cpu_do", "gpu_vertex", "gpu_naive",
                                            "gpu_binned", "gpu_edge", "gpu_do", "gpu_do_persistent", "hybrid"};

// Keep the header and every row whose first field is not key, then append row
// (the reference's util::csvUpsert, src/util/csv.hpp:18-37).
void csvUpsert(const std::string& path, const std::string& header, const std::string& key, const std::string& row) {
    std::vector<std::string> keep;
    {
        std::ifstream in(path);
        std::string line;
        bool first = true;
        while (std::getline(in, line)) {
            if (first) {
                first = false;
                continue;
            }
            if (!line.empty() && line.substr(0, line.find(',')) != key) keep.push_back(line);
        }
    }
    std::ofstream out(path, std::ios::trunc);
    out << header << '\n';
    for (auto& l : keep) out << l << '\n';
    out << row << '\n';
}

// --ordering original|random|degree|rcm: perm[old] = new computed on the
// symmetric graph (empty for original); --locality-csv records the relabelled
// graph's locality (src/bench/main.cpp:179-200).
std::vector<uint32_t> orderingPerm(const Args& args, const Graph& sym, const std::string& dataset) {
    const std::string ordering = args.get("ordering", "original");
    std::vector<uint32_t> perm;
    auto t0 = std::chrono::steady_clock::now();
    if (ordering != "original") {
        perm.resize(sym.n());
        gpu::check(prepReorder(&sym.c, ordering.c_str(), (uint64_t)args.getInt("order-seed", 1), perm.data()));
    }
    const double orderMs = msSince(t0);
    if (args.has("locality-csv")) {
        Graph relabeled;
        if (!perm.empty()) relabeled = make([&](gb_csr* o) { return prepPermute(&sym.c, perm.data(), o); });
        const Graph& L = perm.empty() ? sym : relabeled;
        double gap = 0, same = 0;
        gpu::check(gb_locality(&L.c, &gap, &same));
        char row[256];
        std::snprintf(row, sizeof row, "%s/%s,%s,%s,%llu,%llu,%.2f,%.6f,%.0f", dataset.c_str(), ordering.c_str(),
                      dataset.c_str(), ordering.c_str(), (unsigned long long)sym.n(), (unsigned long long)sym.m(), gap,
                      same, orderMs);
        csvUpsert(args.get("locality-csv"), "key,dataset,ordering,n,m_sym,mean_gap,same_block64,order_ms",
                  dataset + "/" + ordering, row);
        std::printf("locality (%s): mean |u-v| %.1f, same 64-block %.2f%%, ordering took %.0f ms\n", ordering.c_str(),
                    gap, 100 * same, orderMs);
    }
    return perm;
}

int runBfs(const Args& args, const Graph& stored, const std::string& dataset) {
    const std::string variant = args.get("variant", "cpu_serial");
    if (std::find(kVariants.begin(), kVariants.end(), variant) == kVariants.end()) {
        std::fprintf(stderr, "unknown BFS variant '%s'. Available:", variant.c_str());
        for (auto& k : kVariants) std::fprintf(stderr, " %s", k.c_str());
        std::fprintf(stderr, "\n");
        return 2;
    }
    const bool gpuVariant = variant.rfind("gpu_", 0) == 0 || variant == "hybrid";
    const int threads = (int)args.getInt("threads", 0);
    const int nt = threads > 0 ? threads : omp_get_max_threads();
    gpu::GpuBfsOptions o;
    o.tg = (uint32_t)args.getInt("tg", 256);
    o.smallMax = (uint32_t)args.getInt("small-max", 16);
    o.largeMin = (uint32_t)args.getInt("large-min", 256);
    o.ept = (uint32_t)args.getInt("ept", 2);
    o.alpha = args.getDouble("alpha", 15.0);
    o.beta = args.getDouble("beta", 18.0);
    o.block = (uint32_t)args.getInt("block", 512);
    o.hubMin = (uint32_t)args.getInt("hub-min", 4096);
    o.gridBlocks = (uint32_t)args.getInt("grid-blocks", 0);
    o.selMargin = (float)args.getDouble("sel-margin", o.selMargin);
    // --T: the reference's hybrid threshold (levels below it ran on the CPU).
    // hybrid runs every level in the persistent kernel here, so the value is
    // accepted, recorded in params and does not change what runs.
    const std::string tArg = args.get("T", "100000");
    o.hybridT = tArg == "inf" ? UINT64_MAX : (uint64_t)std::stoull(tArg);
    o.cpuThreads = (variant == "hybrid" && !args.has("threads")) ? 4 : threads;
    // --schedule: cpu_omp's OpenMP loop schedule (src/cpu/bfs_cpu.cpp:9-14)
    const Schedule schedule = parseSchedule(args.get("schedule", "dynamic,64"));
    const std::string sel = args.get("selector", "rule");
    if (sel != "rule" && sel != "learned") throw std::runtime_error("--selector must be rule or learned");
    o.selector = sel == "learned" ? GB_SELECT_LEARNED : GB_SELECT_RULE;
    const int batch = (int)args.getInt("batch", 0);

    auto prep0 = std::chrono::steady_clock::now();
    Graph g = make([&](gb_csr* out) { return prepSymmetrize(&stored.c, out); });
    const std::string ordering = args.get("ordering", "original");
    std::vector<uint32_t> perm = orderingPerm(args, g, dataset);
    Graph refG;  // original labels: sources, reference, TEPS denominators
    if (!perm.empty()) {
        refG = std::move(g);
        g = make([&](gb_csr* out) { return prepPermute(&refG.c, perm.data(), out); });
    }
    const Graph& R = perm.empty() ? g : refG;
    auto toRun = [&](uint32_t s) { return perm.empty() ? s : perm[s]; };
    std::unique_ptr<gpu::GpuBfs> gbfs;
    if (gpuVariant) {
        gbfs = std::make_unique<gpu::GpuBfs>(g.c.row_ptr, g.c.col_idx, g.n(), g.m());
        if (args.has("hub-first")) gbfs->hubFirst();
        if (o.selector == GB_SELECT_LEARNED) {
            std::string p = args.get("selector-params", exeDir() + "/../selector_single.bin");
            gbfs->setSelector(0, loadSelector(p));
            std::string pb = exeDir() + "/../selector_batch.bin";
            if (fileExists(pb)) gbfs->setSelector(1, loadSelector(pb));
        }
    }
    const double prepMs = msSince(prep0);

    std::vector<uint32_t> sources;
    if (args.has("source")) sources = {(uint32_t)args.getInt("source", 0)};
    else {
        sources.resize(std::max<long long>(1, args.getInt("sources", 64)));
        int k = 0;
        gpu::check(prepPickSources(&R.c, (int)sources.size(), (uint64_t)args.getInt("seed", 1),
                                   args.has("any-component"), sources.data(), &k));
        sources.resize(k);
    }
    if (sources.empty()) {
        std::fprintf(stderr, "no vertex with degree > 0\n");
        return 1;
    }
    for (uint32_t s : sources)
        if (s >= g.n()) {
            std::fprintf(stderr, "source %u out of range\n", s);
            return 2;
        }
    const int warmup = (int)args.getInt("warmup", 2), trials = (int)args.getInt("trials", 5);
    const int sourceWarmup = (int)args.getInt("source-warmup", 1);
    const bool validate = args.has("validate");

    using Fn = std::function<void(uint32_t, uint32_t*, std::vector<gpu::BfsLevel>*)>;
    Fn fn;
    if (variant == "cpu_serial") fn = [&](uint32_t s, uint32_t* d, std::vector<gpu::BfsLevel>*) { cpuBfsSerial(g, s, d); };
    else if (variant == "cpu_omp")
        fn = [&](uint32_t s, uint32_t* d, std::vector<gpu::BfsLevel>* t) { cpuBfsOmp(g, s, d, nt, schedule, t); };
    else if (variant == "cpu_do")
        fn = [&](uint32_t s, uint32_t* d, std::vector<gpu::BfsLevel>* t) { cpuBfsDO(g, s, d, o.alpha, o.beta, nt, t); };
    else if (variant == "gpu_vertex") fn = [&](uint32_t s, uint32_t* d, std::vector<gpu::BfsLevel>* t) { gbfs->runVertex(s, d, o, t); };
    else if (variant == "gpu_naive") fn = [&](uint32_t s, uint32_t* d, std::vector<gpu::BfsLevel>* t) { gbfs->runNaive(s, d, o, t); };
    else if (variant == "gpu_binned") fn = [&](uint32_t s, uint32_t* d, std::vector<gpu::BfsLevel>* t) { gbfs->runBinned(s, d, o, t); };
    else if (variant == "gpu_edge") fn = [&](uint32_t s, uint32_t* d, std::vector<gpu::BfsLevel>* t) { gbfs->runEdge(s, d, o, t); };
    else if (variant == "gpu_do") fn = [&](uint32_t s, uint32_t* d, std::vector<gpu::BfsLevel>* t) { gbfs->runDO(s, d, o, t); };
    else fn = [&](uint32_t s, uint32_t* d, std::vector<gpu::BfsLevel>* t) { gbfs->runPersistent(s, d, o, t); };

    std::string params;
    if (variant == "cpu_omp" || variant == "cpu_do") params = "threads=" + std::to_string(nt);
    if (variant == "cpu_omp") params += std::string(" schedule=") + scheduleName(schedule);
    if (gpuVariant) params = "tg=" + std::to_string(o.tg);
    if (variant == "gpu_binned")
        params += " small_max=" + std::to_string(o.smallMax) + " large_min=" + std::to_string(o.largeMin);
    if (variant == "gpu_edge" || variant == "gpu_do") params += " ept=" + std::to_string(o.ept);
    if (variant == "gpu_do" || variant == "cpu_do" || variant == "gpu_do_persistent" || variant == "hybrid") {
        char b[96];
        std::snprintf(b, sizeof b, " alpha=%g beta=%g", o.alpha, o.beta);
        params += b;
    }
    if (variant == "gpu_do_persistent" || variant == "hybrid")
        params += " selector=" + sel + " block=" + std::to_string(o.block) + " hub_min=" + std::to_string(o.hubMin);
    if (variant == "hybrid")
        params += " T=" + tArg + " threads=" + std::to_string(o.cpuThreads > 0 ? o.cpuThreads : omp_get_max_threads());
    if (batch > 0) params += " batch=" + std::to_string(batch);

    std::printf("%s: n %llu, symmetrized m %llu (%llu undirected edges), prep %.0f ms\n", dataset.c_str(),
                (unsigned long long)g.n(), (unsigned long long)g.m(), (unsigned long long)(g.m() / 2), prepMs);
    std::printf("bfs %s [%s], %zu source(s), %d warm-up + %d trial(s)%s\n", variant.c_str(), params.c_str(),
                sources.size(), warmup, trials, validate ? ", validating" : "");

    std::vector<uint32_t> dist(g.n()), ref(g.n());
    auto matches = [&](const uint32_t* d, const std::vector<uint32_t>& r, uint64_t* bad) {
        for (uint64_t v = 0; v < g.n(); ++v)
            if (d[toRun((uint32_t)v)] != r[v]) {
                *bad = v;
                return false;
            }
        return true;
    };
    auto compEdgesOf = [&](const std::vector<uint32_t>& r) {
        uint64_t s = 0;
        for (uint64_t v = 0; v < R.n(); ++v)
            if (r[v] != kUnreached) s += R.degree(v);
        return s / 2;
    };

    const std::string csvPath = args.get("csv", "");
    std::ofstream csv;
    if (!csvPath.empty()) {
        bool fresh = !fileExists(csvPath);
        csv.open(csvPath, std::ios::app);
        if (fresh)
            csv << "timestamp,git_commit,chip,dataset,n,m,ordering,algo,variant,params,source,trial,"
                   "time_ms_e2e,time_ms_gpu,gteps,iters,validated,load1\n";
    }
    const std::string ts = timestamp(), chip = chipName(), commit = gitCommit();
    const double load1 = loadAverage1();
    auto row = [&](uint32_t s, int t, double ms, double gpuMs, double gteps) {
        if (!csv.is_open()) return;
        char gpuField[32] = "";
        if (gpuMs >= 0) std::snprintf(gpuField, sizeof gpuField, "%.4f", gpuMs);
        char b[1024];
        std::snprintf(b, sizeof b, "%s,%s,%s,%s,%llu,%llu,%s,bfs,%s,%s,%u,%d,%.4f,%s,%.6f,,%d,%.2f\n", ts.c_str(),
                      commit.c_str(), chip.c_str(), dataset.c_str(), (unsigned long long)g.n(), (unsigned long long)g.m(),
                      ordering.c_str(), variant.c_str(), params.c_str(), s, t, ms, gpuField, gteps, validate ? 1 : 0,
                      load1);
        csv << b;
    };

    std::vector<double> allTimes, allGpu, perSource;
    if (batch > 0) {
        if (!gpuVariant) throw std::runtime_error("--batch needs a GPU variant");
        const int bsz = std::min(batch, 64);
        std::vector<uint32_t> out;
        for (int w = 0; w < warmup; ++w) {
            std::vector<uint32_t> s(sources.begin(), sources.begin() + std::min<size_t>(bsz, sources.size()));
            for (auto& x : s) x = toRun(x);
            out.resize(s.size() * g.n());
            gbfs->runBatch(s, out.data(), o);
        }
        for (size_t b0 = 0; b0 < sources.size(); b0 += bsz) {
            std::vector<uint32_t> s(sources.begin() + b0, sources.begin() + std::min(sources.size(), b0 + bsz));
            std::vector<uint32_t> sr(s);
            for (auto& x : sr) x = toRun(x);
            out.resize(s.size() * g.n());
            uint64_t edges = 0;
            std::vector<std::vector<uint32_t>> refs;
            for (uint32_t x : s) {
                cpuBfsSerial(R, x, ref.data());
                edges += compEdgesOf(ref);
                if (validate) refs.push_back(ref);
            }
            std::vector<double> times;
            for (int t = 0; t < trials; ++t) {
                auto t0 = std::chrono::steady_clock::now();
                gbfs->runBatch(sr, out.data(), o);
                double ms = msSince(t0);
                for (size_t i = 0; validate && i < s.size(); ++i) {
                    uint64_t bad = 0;
                    if (!matches(out.data() + i * g.n(), refs[i], &bad)) {
                        std::fprintf(stderr, "VALIDATION FAILED: %s batch source %u: vertex %llu\n", variant.c_str(),
                                     s[i], (unsigned long long)bad);
                        return 1;
                    }
                }
                times.push_back(ms);
                allTimes.push_back(ms);
                allGpu.push_back(gbfs->lastGpuMs());
                row(s[0], t, ms, gbfs->lastGpuMs(), edges / (ms * 1e6));
            }
            perSource.push_back(edges / (median(times) * 1e6));
        }
    } else {
        for (int w = 0; w < warmup; ++w) fn(toRun(sources[w % sources.size()]), dist.data(), nullptr);
        for (uint32_t s : sources) {
            cpuBfsSerial(R, s, ref.data());
            const uint64_t compEdges = compEdgesOf(ref);
            for (int w = 0; w < sourceWarmup && trials > 0; ++w) fn(toRun(s), dist.data(), nullptr);
            std::vector<double> times;
            for (int t = 0; t < trials; ++t) {
                auto t0 = std::chrono::steady_clock::now();
                fn(toRun(s), dist.data(), nullptr);
                double ms = msSince(t0);
                double gpuMs = gbfs ? gbfs->lastGpuMs() : -1;
                uint64_t bad = 0;
                if (validate && !matches(dist.data(), ref, &bad)) {
                    std::fprintf(stderr, "VALIDATION FAILED: %s [%s] source %u trial %d: vertex %llu: got %u, expected %u\n",
                                 variant.c_str(), ordering.c_str(), s, t, (unsigned long long)bad,
                                 dist[toRun((uint32_t)bad)], ref[bad]);
                    return 1;
                }
                times.push_back(ms);
                allTimes.push_back(ms);
                if (gpuMs >= 0) allGpu.push_back(gpuMs);
                row(s, t, ms, gpuMs, compEdges / (ms * 1e6));
            }
            if (trials > 0) perSource.push_back(compEdges / (median(times) * 1e6));
        }
    }
    double hsum = 0;
    size_t hc = 0;
    for (double x : perSource)
        if (x > 0) {
            hsum += 1.0 / x;
            ++hc;
        }
    if (!allTimes.empty()) {
        char gpuPart[64] = "";
        if (!allGpu.empty()) std::snprintf(gpuPart, sizeof gpuPart, " | GPU-only median %.3f", median(allGpu));
        std::printf("time ms: median %.3f, min %.3f%s | GTEPS harmonic mean %.4f%s\n", median(allTimes),
                    *std::min_element(allTimes.begin(), allTimes.end()), gpuPart, hc ? hc / hsum : 0.0,
                    validate ? " | validated OK" : "");
    }
    const std::string tracePath = args.get("trace", "");
    if (!tracePath.empty() && batch == 0) {
        bool fresh = !fileExists(tracePath);
        std::ofstream tr(tracePath, std::ios::app);
        if (fresh) tr << "dataset,ordering,variant,params,source,level,frontier,edges,direction,device,time_ms\n";
        for (uint32_t s : sources) {
            std::vector<gpu::BfsLevel> levels;
            fn(toRun(s), dist.data(), &levels);
            for (auto& L : levels) {
                char b[512];
                std::snprintf(b, sizeof b, "%s,%s,%s,%s,%u,%u,%llu,%llu,%c,%c,%.4f\n", dataset.c_str(),
                              ordering.c_str(), variant.c_str(), params.c_str(), s, L.level,
                              (unsigned long long)L.frontier, (unsigned long long)L.edges, L.direction, L.device,
                              L.time_ms);
                tr << b;
            }
        }
        std::printf("trace written to %s\n", tracePath.c_str());
    }
    const std::string dumpPath = args.get("dump-dist", "");
    if (!dumpPath.empty()) {
        fn(toRun(sources.back()), dist.data(), nullptr);
        std::vector<uint32_t> orig(g.n());
        for (uint64_t v = 0; v < g.n(); ++v) orig[v] = dist[toRun((uint32_t)v)];
        std::ofstream out(dumpPath, std::ios::binary);
        out.write(reinterpret_cast<const char*>(orig.data()), g.n() * 4);
    }
    return 0;
}

const std::vector<std::string> kPrVariants = {"cpu_serial", "cpu_omp", "gpu_push", "gpu_pull_scalar",
                                              "gpu_pull_vector", "gpu_pull_adaptive", "gpu_pull_gs", "gpu_pull_f64",
                                              "gpu_pull_blocked"};

int runPr(const Args& args, const Graph& stored, const std::string& dataset) {
    const std::string variant = args.get("variant", "cpu_serial");
    if (std::find(kPrVariants.begin(), kPrVariants.end(), variant) == kPrVariants.end()) {
        std::fprintf(stderr, "unknown PageRank variant '%s'. Available:", variant.c_str());
        for (auto& k : kPrVariants) std::fprintf(stderr, " %s", k.c_str());
        std::fprintf(stderr, "\n");
        return 2;
    }
    const bool gpuVariant = variant.rfind("gpu_", 0) == 0;
    const double tol = args.getDouble("tol", 0);
    const int iters = (int)args.getInt("iters", tol > 0 ? 1000 : 20);
    const int threads = (int)args.getInt("threads", 0);
    const int nt = threads > 0 ? threads : omp_get_max_threads();
    gpu::GpuPrOptions o;
    o.iters = iters;
    o.tol = tol;
    o.tg = (uint32_t)args.getInt("tg", 256);
    o.smallMax = (uint32_t)args.getInt("small-max", 16);
    o.largeMin = (uint32_t)args.getInt("large-min", 256);
    o.inPlace = args.has("inplace");
    o.tolRel = args.getDouble("tol-rel", 0);
    const bool validate = args.has("validate");
    const bool gsCheck = variant == "gpu_pull_gs" || o.inPlace;
    // --ref-tol: the Jacobi reference's tolerance when it should differ from
    // --tol (Gauss-Seidel at a tighter tol judged against Jacobi at 1e-6)
    const double refTol = args.getDouble("ref-tol", tol);

    auto prep0 = std::chrono::steady_clock::now();
    // --ordering: perm from the symmetric graph, applied to the stored graph
    // (src/bench/main.cpp:459-500); ranks are reported in the original ids.
    std::vector<uint32_t> perm;
    if (args.get("ordering", "original") != "original" || args.has("locality-csv")) {
        if (stored.directed()) {
            Graph sym = make([&](gb_csr* out) { return prepSymmetrize(&stored.c, out); });
            perm = orderingPerm(args, sym, dataset);
        } else {
            perm = orderingPerm(args, stored, dataset);
        }
    }
    const bool permuted = !perm.empty();
    Graph relabeled;
    if (permuted) relabeled = make([&](gb_csr* out) { return prepPermute(&stored.c, perm.data(), out); });
    const Graph& G = permuted ? relabeled : stored;  // what the variant runs on
    Graph inOwn;
    if (G.directed()) inOwn = make([&](gb_csr* out) { return prepTranspose(&G.c, out); });
    const Graph& in = G.directed() ? inOwn : G;
    std::vector<uint32_t> od(G.n());
    for (uint64_t v = 0; v < G.n(); ++v) od[v] = G.degree(v);
    std::vector<double> ref, refConv;
    PrCheck jacobiErr;
    int refIters = 0;
    if (validate) {  // the reference in the original ids
        Graph inO;
        if (permuted && stored.directed()) inO = make([&](gb_csr* out) { return prepTranspose(&stored.c, out); });
        const Graph& RI = !permuted ? in : stored.directed() ? inO : stored;
        std::vector<uint32_t> odO(stored.n());
        for (uint64_t v = 0; v < stored.n(); ++v) odO[v] = stored.degree(v);
        double ld = 0;
        refIters = cpuPagerank(RI, odO, ref, iters, tol, nt, &ld);
        if (gsCheck && refTol != tol)
            refIters = cpuPagerank(RI, odO, ref, refTol > 0 ? 1000 : iters, refTol, nt, &ld);
        if (gsCheck) {
            cpuPagerank(RI, odO, refConv, 1000, 1e-10, nt, &ld);
            jacobiErr = checkRanks(refConv, ref.data());
        }
    }
    std::unique_ptr<gpu::GpuPageRank> gpr;
    if (gpuVariant) {
        const bool needOut = variant == "gpu_push";
        gpr = std::make_unique<gpu::GpuPageRank>(G.n(), needOut ? G.c.row_ptr : nullptr,
                                                 needOut ? G.c.col_idx : nullptr, G.m(), in.c.row_ptr,
                                                 in.c.col_idx, in.m(), od);
        if (variant == "gpu_pull_adaptive") gpr->prepareAdaptive(o.smallMax, o.largeMin);
        if (variant == "gpu_pull_gs") gpr->prepareGS((uint32_t)args.getInt("gs-pairs", 2));
    }
    const double prepMs = msSince(prep0);
    std::printf("%s: n %llu, m %llu (directed=%d), prep %.0f ms\npr %s [%s]\n", dataset.c_str(),
                (unsigned long long)stored.n(), (unsigned long long)stored.m(), (int)stored.directed(), prepMs,
                variant.c_str(), tol > 0 ? "tol mode" : ("iters=" + std::to_string(iters)).c_str());
    std::vector<double> rcpu;
    const gpu::PrVariant pv = gpuVariant ? gpu::parsePrVariant(variant) : gpu::PrVariant::PullVector;
    int lastIters = 0;
    double lastDelta = -1, lastMaxRel = -1;
    bool floorStop = false;
    auto runOnce = [&]() -> double {
        if (!gpuVariant) {
            lastIters = cpuPagerank(in, od, rcpu, iters, tol, variant == "cpu_serial" ? 1 : nt, &lastDelta);
            return -1;
        }
        gpu::GpuPrResult r = gpr->run(pv, o);
        lastIters = r.iters;
        lastDelta = r.lastDelta;
        lastMaxRel = r.lastMaxRel;
        floorStop = r.floorStop;
        return r.gpuMs;
    };
    auto ranksD = [&]() {  // original ids: rank of v = result[perm[v]]
        std::vector<double> out(stored.n()), r64;
        const float* r = nullptr;
        if (gpuVariant && pv == gpu::PrVariant::PullF64) r64 = gpr->ranks64();
        else if (gpuVariant) r = gpr->ranks();
        for (uint64_t v = 0; v < stored.n(); ++v) {
            const uint64_t x = permuted ? perm[v] : v;
            out[v] = !gpuVariant ? rcpu[x] : r ? (double)r[x] : r64[x];
        }
        return out;
    };
    const int warmup = (int)args.getInt("warmup", 2), trials = (int)args.getInt("trials", 5);
    for (int w = 0; w < warmup; ++w) runOnce();

    // CSV rows: one per trial, same schema as BFS (src/bench/main.cpp:571-620);
    // source empty, gteps = m * iterations / time, iters = iterations run.
    char tolStr[32];  // %g: tolerances below 1e-6 must not print as 0.000000
    std::snprintf(tolStr, sizeof tolStr, "%g", tol);
    std::string params = tol > 0 ? std::string("tol=") + tolStr + " cap=" + std::to_string(iters)
                                 : "iters=" + std::to_string(iters);
    if (variant == "cpu_omp") params += " threads=" + std::to_string(nt);
    if (gpuVariant) params += " tg=" + std::to_string(o.tg);
    if (o.tolRel > 0) {
        char r[32];
        std::snprintf(r, sizeof r, " tol_rel=%g", o.tolRel);
        params += r;
    }
    if (o.inPlace) params += " inplace";
    if (variant == "gpu_pull_adaptive")
        params += " small_max=" + std::to_string(o.smallMax) + " large_min=" + std::to_string(o.largeMin);
    const std::string csvPath = args.get("csv", "");
    const std::string ordering = args.get("ordering", "original");
    std::ofstream csv;
    if (!csvPath.empty()) {
        bool fresh = !fileExists(csvPath);
        csv.open(csvPath, std::ios::app);
        if (fresh)
            csv << "timestamp,git_commit,chip,dataset,n,m,ordering,algo,variant,params,source,trial,"
                   "time_ms_e2e,time_ms_gpu,gteps,iters,validated,load1\n";
    }
    const std::string ts = timestamp(), chip = chipName(), commit = gitCommit();
    const double load1 = loadAverage1();

    std::vector<double> times, gpuTimes;
    PrCheck worst;
    for (int t = 0; t < trials; ++t) {
        auto t0 = std::chrono::steady_clock::now();
        double gms = runOnce();
        double ms = msSince(t0);
        if (validate) {
            std::vector<double> got = ranksD();
            PrCheck c = checkRanks(gsCheck ? refConv : ref, got.data());
            bool ok = !gsCheck ? c.ok() : tol > 0 ? gsNoWorse(c, jacobiErr) : std::fabs(c.sum - 1.0) < 1e-4;
            if (!ok) {
                std::fprintf(stderr, "VALIDATION FAILED: %s trial %d: L1 %.6g, max rel (top-1000) %.6g, sum %.8f\n",
                             variant.c_str(), t, c.l1, c.maxRelTop, c.sum);
                return 1;
            }
            if (c.l1 >= worst.l1) worst = c;
        }
        times.push_back(ms);
        if (gms >= 0) gpuTimes.push_back(gms);
        if (csv.is_open()) {
            char gpuField[32] = "";
            if (gms >= 0) std::snprintf(gpuField, sizeof gpuField, "%.4f", gms);
            char row[1024];
            std::snprintf(row, sizeof row, "%s,%s,%s,%s,%llu,%llu,%s,pr,%s,%s,,%d,%.4f,%s,%.6f,%d,%d,%.2f\n",
                          ts.c_str(), commit.c_str(), chip.c_str(), dataset.c_str(), (unsigned long long)stored.n(),
                          (unsigned long long)stored.m(), ordering.c_str(), variant.c_str(), params.c_str(), t, ms,
                          gpuField, (double)stored.m() * lastIters / (ms * 1e6), lastIters, validate ? 1 : 0, load1);
            csv << row;
        }
    }
    if (!times.empty()) {
        const double med = median(times), perIt = med / std::max(1, lastIters);
        std::printf("time ms: median %.3f, min %.3f | %d iterations, %.4f ms/iteration", med,
                    *std::min_element(times.begin(), times.end()), lastIters, perIt);
        if (!gpuTimes.empty()) std::printf(" (GPU-only %.4f)", median(gpuTimes) / std::max(1, lastIters));
        if (tol > 0)
            std::printf(" | final L1 change %.3g%s", lastDelta,
                        lastDelta < tol ? "" : floorStop ? " (stopped at float precision floor)" : " (NOT converged)");
        if (tol > 0 && lastMaxRel >= 0) std::printf(", max rel change %.3g", lastMaxRel);
        const double bytes = 4.0 * (stored.n() + 1) + 8.0 * stored.m() + 4.0 * stored.n();
        std::printf(" | eff. %.1f GB/s", bytes / (perIt * 1e6));
        if (validate) std::printf(" | validated OK (ref %d iters; worst L1 %.2e)", refIters, worst.l1);
        std::printf("\n");
    }
    const std::string dumpPath = args.get("dump-ranks", "");
    if (!dumpPath.empty()) {
        if (trials == 0) runOnce();
        std::vector<double> r = ranksD();
        std::ofstream out(dumpPath, std::ios::binary);
        out.write(reinterpret_cast<const char*>(r.data()), r.size() * sizeof(double));
    }
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    Args args(argc, argv);
    if (!args.has("graph")) {
        std::fprintf(stderr, "usage: gbench --graph <file.bin | synth:NAME> --algo bfs|pr --variant V [options]\n");
        return 2;
    }
    gHostPrep = args.has("host-prep");
    gb_device_info(nullptr, 0, nullptr, nullptr, nullptr);  // context up front; CPU-only runs ignore a failure
    try {
        std::string dataset;
        Graph g = loadGraph(args.get("graph"), dataset);
        if (args.has("save-graph")) {
            gpu::check(gb_csr_save(&g.c, args.get("save-graph").c_str()));
            return 0;
        }
        const std::string algo = args.get("algo", "bfs");
        if (algo == "bfs") return runBfs(args, g, dataset);
        if (algo == "pr") return runPr(args, g, dataset);
        std::fprintf(stderr, "unknown --algo '%s' (bfs | pr)\n", algo.c_str());
        return 2;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "gbench: %s\n", e.what());
        return 1;
    }
}
