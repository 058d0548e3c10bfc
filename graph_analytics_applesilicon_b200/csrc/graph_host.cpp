// graph_host.cpp -- host CSR builders, transforms, generators and .bin I/O.
//
// Same graphs as the reference's src/graph layer, byte for byte (checked by
// the tests against golden fixtures produced by the reference's own code),
// built in parallel with OpenMP: lists are filled by atomic cursors in any
// order and then sorted, which gives the canonical sorted/deduplicated CSR
// whatever the schedule.
#include "graph_host.hpp"

#include <omp.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>

#include "common.cuh"

namespace gb {

namespace {

constexpr char kMagic[8] = {'G', 'G', 'P', 'U', 'C', 'S', 'R', '1'};

struct FileHeader {  // src/graph/csr.hpp:20-27
    char magic[8];
    uint32_t version;
    uint32_t flags;
    uint64_t num_vertices;
    uint64_t num_edges;
};
static_assert(sizeof(FileHeader) == 32, "GGPUCSR1 header is 32 bytes");

inline uint32_t atomicInc32(uint32_t* p) { return __atomic_fetch_add(p, 1u, __ATOMIC_RELAXED); }

// Exclusive prefix of counts into offsets (n + 1 entries); throws if m >= 2^32.
void prefixOffsets(const std::vector<uint32_t>& cnt, std::vector<uint32_t>& rp) {
    const uint64_t n = cnt.size();
    rp.assign(n + 1, 0);
    uint64_t run = 0;
    for (uint64_t v = 0; v < n; ++v) {
        rp[v] = (uint32_t)run;
        run += cnt[v];
        if (run >= (1ull << 32)) throw Error(GB_ERR_ARG, "graph has 2^32 or more adjacency entries");
    }
    rp[n] = (uint32_t)run;
}

// Sort every list of (rp, ci), drop self-loops (if dropSelf) and duplicates,
// and compact into a fresh CSR (src/graph/csr.cpp:112-144 semantics).
void sortDedupCompact(uint64_t n, const std::vector<uint32_t>& rp, std::vector<uint32_t>& ci,
                      bool dedup, HostCsr& out) {
    std::vector<uint32_t> newDeg(n);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t v = 0; v < (int64_t)n; ++v) {
        uint32_t* b = ci.data() + rp[v];
        uint32_t* e = ci.data() + rp[v + 1];
        std::sort(b, e);
        if (!dedup) {
            newDeg[v] = (uint32_t)(e - b);
            continue;
        }
        uint32_t* o = b;
        for (uint32_t* p = b; p != e; ++p) {
            if (*p == (uint32_t)v) continue;
            if (o != b && o[-1] == *p) continue;
            *o++ = *p;
        }
        newDeg[v] = (uint32_t)(o - b);
    }
    out.n = n;
    prefixOffsets(newDeg, out.row_ptr);
    out.m = out.row_ptr[n];
    out.col_idx.resize(out.m);
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t v = 0; v < (int64_t)n; ++v)
        if (newDeg[v]) std::memcpy(out.col_idx.data() + out.row_ptr[v], ci.data() + rp[v], 4ull * newDeg[v]);
}

}  // namespace

HostCsr csrFromEdges(uint64_t n, const uint32_t* eu, const uint32_t* ev, uint64_t ne, bool directed) {
    if (n >= 0xFFFFFFFFull) throw Error(GB_ERR_ARG, "too many vertices for uint32 ids");
    std::vector<uint32_t> cnt(n, 0);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)ne; ++i) {
        if (eu[i] >= n || ev[i] >= n) continue;  // validated below
        atomicInc32(&cnt[eu[i]]);
        if (!directed) atomicInc32(&cnt[ev[i]]);
    }
    for (uint64_t i = 0; i < ne; ++i)
        if (eu[i] >= n || ev[i] >= n) throw Error(GB_ERR_ARG, "edge endpoint out of range");
    std::vector<uint32_t> rp;
    prefixOffsets(cnt, rp);
    std::vector<uint32_t> ci(rp[n]);
    std::vector<uint32_t> cur(rp.begin(), rp.end() - 1);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)ne; ++i) {
        ci[atomicInc32(&cur[eu[i]])] = ev[i];
        if (!directed) ci[atomicInc32(&cur[ev[i]])] = eu[i];
    }
    HostCsr g;
    sortDedupCompact(n, rp, ci, true, g);
    g.flags = (directed ? GB_FLAG_DIRECTED : 0u) | GB_FLAG_SORTED | GB_FLAG_DEDUP;
    return g;
}

HostCsr csrTranspose(const HostCsr& g) {
    const uint64_t n = g.n;
    std::vector<uint32_t> cnt(n, 0);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)g.m; ++i) atomicInc32(&cnt[g.col_idx[i]]);
    std::vector<uint32_t> rp;
    prefixOffsets(cnt, rp);
    std::vector<uint32_t> ci(g.m);
    std::vector<uint32_t> cur(rp.begin(), rp.end() - 1);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t u = 0; u < (int64_t)n; ++u)
        for (uint32_t i = g.row_ptr[u]; i < g.row_ptr[u + 1]; ++i) ci[atomicInc32(&cur[g.col_idx[i]])] = (uint32_t)u;
    HostCsr t;
    sortDedupCompact(n, rp, ci, false, t);  // in-lists sorted by source, as a serial scatter gives
    t.flags = g.flags;
    return t;
}

HostCsr csrSymmetrize(const HostCsr& g) {
    if (!(g.flags & GB_FLAG_DIRECTED)) return g;
    HostCsr t = csrTranspose(g);
    const int64_t n = (int64_t)g.n;
    auto merge = [&](int64_t v, uint32_t* out) -> uint32_t {  // union of two sorted lists
        const uint32_t *a = g.col_idx.data() + g.row_ptr[v], *ae = g.col_idx.data() + g.row_ptr[v + 1];
        const uint32_t *b = t.col_idx.data() + t.row_ptr[v], *be = t.col_idx.data() + t.row_ptr[v + 1];
        uint32_t k = 0;
        while (a != ae || b != be) {
            uint32_t x;
            if (b == be || (a != ae && *a < *b)) x = *a++;
            else if (a == ae || *b < *a) x = *b++;
            else { x = *a++; ++b; }
            if (out) out[k] = x;
            ++k;
        }
        return k;
    };
    std::vector<uint32_t> cnt(n);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t v = 0; v < n; ++v) cnt[v] = merge(v, nullptr);
    HostCsr s;
    s.n = g.n;
    prefixOffsets(cnt, s.row_ptr);
    s.m = s.row_ptr[n];
    s.col_idx.resize(s.m);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t v = 0; v < n; ++v) merge(v, s.col_idx.data() + s.row_ptr[v]);
    s.flags = GB_FLAG_SORTED | GB_FLAG_DEDUP;
    return s;
}

HostCsr csrPermute(const HostCsr& g, const uint32_t* perm) {
    const uint64_t n = g.n;
    std::vector<uint32_t> inv(n);
    std::vector<uint8_t> seen(n, 0);
    for (uint64_t v = 0; v < n; ++v) {
        if (perm[v] >= n || seen[perm[v]]) throw Error(GB_ERR_ARG, "permute: not a permutation");
        seen[perm[v]] = 1;
        inv[perm[v]] = (uint32_t)v;
    }
    std::vector<uint32_t> cnt(n);
    for (uint64_t nv = 0; nv < n; ++nv) cnt[nv] = g.degree(inv[nv]);
    HostCsr p;
    p.n = n;
    prefixOffsets(cnt, p.row_ptr);
    p.m = g.m;
    p.col_idx.resize(g.m);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t nv = 0; nv < (int64_t)n; ++nv) {
        uint32_t* out = p.col_idx.data() + p.row_ptr[nv];
        uint32_t k = 0, old = inv[nv];
        for (uint32_t i = g.row_ptr[old]; i < g.row_ptr[old + 1]; ++i) out[k++] = perm[g.col_idx[i]];
        std::sort(out, out + k);
    }
    p.flags = g.flags;
    return p;
}

std::vector<uint32_t> randomPerm(uint64_t n, uint64_t seed) {
    std::vector<uint32_t> p(n);
    std::iota(p.begin(), p.end(), 0u);
    uint64_t k = 0;
    for (uint64_t i = n; i > 1; --i) std::swap(p[i - 1], p[belowAt(seed, ++k, i)]);
    return p;
}

namespace {

// Vertices sorted by (degree, id), ascending or by descending degree.
std::vector<uint32_t> byDegree(const HostCsr& g, bool descending) {
    std::vector<uint32_t> v(g.n);
    std::iota(v.begin(), v.end(), 0u);
    std::stable_sort(v.begin(), v.end(), [&](uint32_t a, uint32_t b) {
        return descending ? g.degree(a) > g.degree(b) : g.degree(a) < g.degree(b);
    });
    return v;
}

// One Cuthill-McKee breadth-first pass (src/graph/reorder.cpp:40-62): from
// start over unmarked vertices, each vertex's newly marked neighbours appended
// in (degree, id) order.  Returns the index in out where the last level begins.
size_t cuthillMcKee(const HostCsr& g, uint32_t start, std::vector<uint8_t>& mark, std::vector<uint32_t>& out,
                    std::vector<uint32_t>& fresh) {
    size_t head = out.size(), levelBegin = head;
    out.push_back(start);
    mark[start] = 1;
    auto less = [&](uint32_t a, uint32_t b) { return g.degree(a) != g.degree(b) ? g.degree(a) < g.degree(b) : a < b; };
    while (head < out.size()) {
        levelBegin = head;
        for (const size_t end = out.size(); head < end; ++head) {
            const uint32_t u = out[head];
            fresh.clear();
            for (uint32_t i = g.row_ptr[u]; i < g.row_ptr[u + 1]; ++i)
                if (!mark[g.col_idx[i]]) {
                    mark[g.col_idx[i]] = 1;
                    fresh.push_back(g.col_idx[i]);
                }
            std::sort(fresh.begin(), fresh.end(), less);
            out.insert(out.end(), fresh.begin(), fresh.end());
        }
    }
    return levelBegin;
}

}  // namespace

std::vector<uint32_t> orderingPerm(const HostCsr& g, const std::string& ordering, uint64_t seed) {
    std::vector<uint32_t> perm(g.n);
    if (ordering == "original") {
        std::iota(perm.begin(), perm.end(), 0u);
    } else if (ordering == "random") {
        perm = randomPerm(g.n, seed);
    } else if (ordering == "degree") {  // src/graph/reorder.cpp:27-38
        const auto order = byDegree(g, true);
        for (uint64_t i = 0; i < g.n; ++i) perm[order[i]] = (uint32_t)i;
    } else if (ordering == "rcm") {  // src/graph/reorder.cpp:64-92
        std::vector<uint8_t> mark(g.n, 0), probe(g.n, 0);
        std::vector<uint32_t> order, pass, fresh;
        order.reserve(g.n);
        for (uint32_t s : byDegree(g, false)) {
            if (mark[s]) continue;
            pass.clear();
            const size_t last = cuthillMcKee(g, s, probe, pass, fresh);
            uint32_t start = pass[last];
            for (size_t i = last; i < pass.size(); ++i)
                if (g.degree(pass[i]) < g.degree(start)) start = pass[i];
            cuthillMcKee(g, start, mark, order, fresh);
        }
        for (uint64_t i = 0; i < g.n; ++i) perm[order[i]] = (uint32_t)(g.n - 1 - i);
    } else {
        throw Error(GB_ERR_ARG, "unknown ordering '" + ordering + "' (original|random|degree|rcm)");
    }
    return perm;
}

void locality(const HostCsr& g, double* meanGap, double* sameBlock64) {
    double gap = 0;
    uint64_t same = 0;
    for (uint64_t u = 0; u < g.n; ++u)
        for (uint32_t i = g.row_ptr[u]; i < g.row_ptr[u + 1]; ++i) {
            const uint64_t w = g.col_idx[i];
            gap += (double)(u > w ? u - w : w - u);
            same += (u >> 6) == (w >> 6);
        }
    *meanGap = g.m ? gap / (double)g.m : 0.0;
    *sameBlock64 = g.m ? (double)same / (double)g.m : 0.0;
}

std::string csrValidate(const HostCsr& g) {
    if (g.m >= (1ull << 32)) return "m does not fit in uint32";
    if (g.row_ptr.size() != g.n + 1) return "row_ptr must have n+1 entries";
    if (g.row_ptr[0] != 0) return "row_ptr[0] != 0";
    if (g.row_ptr[g.n] != g.m) return "row_ptr[n] != m";
    const bool strict = (g.flags & GB_FLAG_SORTED) && (g.flags & GB_FLAG_DEDUP);
    for (uint64_t v = 0; v < g.n; ++v) {
        uint32_t b = g.row_ptr[v], e = g.row_ptr[v + 1];
        if (e < b) return "row_ptr decreases at v=" + std::to_string(v);
        for (uint32_t i = b; i < e; ++i) {
            uint32_t u = g.col_idx[i];
            if (u >= g.n) return "col_idx out of range at v=" + std::to_string(v);
            if (strict) {
                if (u == v) return "self-loop at v=" + std::to_string(v);
                if (i > b && g.col_idx[i - 1] >= u) return "list not strictly sorted at v=" + std::to_string(v);
            }
        }
    }
    return "";
}

// ------------------------------------------------------------ generators

namespace {
struct Edges {
    std::vector<uint32_t> u, v;
    void add(uint32_t a, uint32_t b) {
        u.push_back(a);
        v.push_back(b);
    }
    HostCsr build(uint64_t n, bool directed) const { return csrFromEdges(n, u.data(), v.data(), u.size(), directed); }
};
void addGrid(Edges& e, uint32_t base, uint32_t rows, uint32_t cols) {  // src/graph/generators.cpp:27-34
    for (uint32_t r = 0; r < rows; ++r)
        for (uint32_t c = 0; c < cols; ++c) {
            uint32_t v = base + r * cols + c;
            if (c + 1 < cols) e.add(v, v + 1);
            if (r + 1 < rows) e.add(v, v + cols);
        }
}
}  // namespace

HostCsr genPath(uint32_t n) {
    Edges e;
    for (uint32_t i = 0; i + 1 < n; ++i) e.add(i, i + 1);
    return e.build(n, false);
}

HostCsr genStar(uint32_t leaves) {
    Edges e;
    for (uint32_t i = 1; i <= leaves; ++i) e.add(0, i);
    return e.build((uint64_t)leaves + 1, false);
}

HostCsr genComplete(uint32_t n) {
    Edges e;
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t j = i + 1; j < n; ++j) e.add(i, j);
    return e.build(n, false);
}

HostCsr genTwoComponents() {
    Edges e;
    for (uint32_t i = 0; i + 1 < 300; ++i) e.add(i, i + 1);
    addGrid(e, 300, 10, 10);
    return e.build(400, false);
}

HostCsr genEmpty(uint32_t n) { return csrFromEdges(n, nullptr, nullptr, 0, false); }

HostCsr genGrid2d(uint32_t rows, uint32_t cols) {
    Edges e;
    addGrid(e, 0, rows, cols);
    return e.build((uint64_t)rows * cols, false);
}

// Graph500-parameter R-MAT (src/graph/generators.cpp:51-75), `edges` draws.
// Edge i uses stream outputs i*scale+1 .. i*scale+scale, as the reference's
// sequential loop does.
HostCsr genRmat(uint32_t scale, uint64_t edges, bool directed, uint64_t seed) {
    if (scale == 0 || scale > 31) throw Error(GB_ERR_ARG, "rmat: scale must be in [1, 31]");
    const double a = 0.57, b = 0.19, c = 0.19;
    std::vector<uint32_t> eu(edges), ev(edges);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)edges; ++i) {
        uint32_t u = 0, v = 0;
        uint64_t k = (uint64_t)i * scale;
        for (uint32_t bit = 0; bit < scale; ++bit) {
            double r = unitAt(seed, ++k);
            uint32_t ub = 0, vb = 0;
            if (r < a) {
            } else if (r < a + b) {
                vb = 1;
            } else if (r < a + b + c) {
                ub = 1;
            } else {
                ub = 1;
                vb = 1;
            }
            u = (u << 1) | ub;
            v = (v << 1) | vb;
        }
        eu[i] = u;
        ev[i] = v;
    }
    return csrFromEdges(1ull << scale, eu.data(), ev.data(), edges, directed);
}

// Road-shaped graph (no reference counterpart): the rows x cols 4-neighbour
// grid of gen::grid2d with each edge k (addGrid order) dropped when
// U_k < dropFrac (U_k = output k+1 of SplitMix64(seed)), plus round(diagFrac*n)
// attempted diagonal links: attempt j draws v = below(n) and a direction
// below(4) in {(-1,-1), (-1,+1), (+1,-1), (+1,+1)} from SplitMix64(seed ^
// 0x5DEECE66D) outputs 2j+1, 2j+2; links leaving the grid are skipped.
// Degree <= 4 grid + 4 distinct diagonal neighbours = 8.
HostCsr genRoad(uint32_t rows, uint32_t cols, double dropFrac, double diagFrac, uint64_t seed) {
    const uint64_t n = (uint64_t)rows * cols;
    const uint64_t perRow = 2ull * cols - 1;  // right + down edges of a non-final row, interleaved
    const uint64_t gridEdges = (rows ? (uint64_t)(rows - 1) * perRow + (cols - 1) : 0);
    std::vector<uint32_t> eu(gridEdges), ev(gridEdges);
    std::vector<uint8_t> keep(gridEdges);
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < (int64_t)rows; ++r) {
        uint64_t k = (uint64_t)r * perRow;
        for (uint32_t c = 0; c < cols; ++c) {
            uint32_t v = (uint32_t)(r * cols + c);
            if (c + 1 < cols) {
                eu[k] = v;
                ev[k] = v + 1;
                keep[k] = unitAt(seed, k + 1) >= dropFrac;
                ++k;
            }
            if ((uint64_t)r + 1 < rows) {
                eu[k] = v;
                ev[k] = v + cols;
                keep[k] = unitAt(seed, k + 1) >= dropFrac;
                ++k;
            }
        }
    }
    std::vector<uint32_t> u2, v2;
    u2.reserve(gridEdges);
    v2.reserve(gridEdges);
    for (uint64_t k = 0; k < gridEdges; ++k)
        if (keep[k]) {
            u2.push_back(eu[k]);
            v2.push_back(ev[k]);
        }
    const uint64_t seed2 = seed ^ 0x5DEECE66Dull;
    const uint64_t diag = (uint64_t)std::llround(diagFrac * (double)n);
    static const int dr[4] = {-1, -1, 1, 1}, dc[4] = {-1, 1, -1, 1};
    for (uint64_t j = 0; j < diag && n; ++j) {
        uint64_t v = belowAt(seed2, 2 * j + 1, n);
        int d = (int)belowAt(seed2, 2 * j + 2, 4);
        int64_t r = (int64_t)(v / cols) + dr[d], c = (int64_t)(v % cols) + dc[d];
        if (r < 0 || c < 0 || r >= rows || c >= cols) continue;
        u2.push_back((uint32_t)v);
        v2.push_back((uint32_t)(r * cols + c));
    }
    return csrFromEdges(n, u2.data(), v2.data(), u2.size(), false);
}

// Web-shaped directed graph (no reference counterpart).  Vertex u's
// out-degree is Geometric on {0,1,...} with mean outMean (p = 1/(1+outMean);
// K = floor(log(1-U)/log(1-p)), U = output u+1 of SplitMix64(seed)); each
// out-edge slot e picks a popularity rank r with density ~ (r+1)^(-1/(s-1))
// by inverse CDF of the continuous power law on [1, n+1) (U = output e+1 of
// SplitMix64(seed+1)), and targets vertex perm[r], perm = randomPerm(n, seed+2).
// In-degrees then follow a power law with exponent s; duplicates and
// self-loops are removed by fromEdgeList.
HostCsr genWeb(uint32_t n, double outMean, double zipfS, uint64_t seed) {
    if (zipfS <= 1.0 || outMean <= 0) throw Error(GB_ERR_ARG, "web: need zipf_s > 1 and out_mean > 0");
    const double p = 1.0 / (1.0 + outMean), lq = std::log1p(-p);
    std::vector<uint32_t> od(n);
#pragma omp parallel for schedule(static)
    for (int64_t u = 0; u < (int64_t)n; ++u) {
        double U = unitAt(seed, (uint64_t)u + 1);
        double k = std::floor(std::log1p(-U) / lq);
        od[u] = (uint32_t)std::min(k, 1e6);
    }
    std::vector<uint64_t> off(n + 1, 0);
    for (uint32_t u = 0; u < n; ++u) off[u + 1] = off[u] + od[u];
    const uint64_t ne = off[n];
    const std::vector<uint32_t> perm = randomPerm(n, seed + 2);
    const double a = 1.0 / (zipfS - 1.0), e1 = 1.0 - a;
    const double top = std::pow((double)n + 1.0, e1) - 1.0;
    std::vector<uint32_t> eu(ne), ev(ne);
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t u = 0; u < (int64_t)n; ++u)
        for (uint64_t e = off[u]; e < off[u + 1]; ++e) {
            double U = unitAt(seed + 1, e + 1);
            double x = std::fabs(e1) < 1e-12 ? std::exp(U * std::log((double)n + 1.0))
                                             : std::pow(1.0 + U * top, 1.0 / e1);
            uint64_t r = (uint64_t)std::floor(x);
            r = r < 1 ? 0 : std::min<uint64_t>(r - 1, n - 1);
            eu[e] = (uint32_t)u;
            ev[e] = perm[r];
        }
    return csrFromEdges(n, eu.data(), ev.data(), ne, true);
}

// Chung-Lu graph (no reference counterpart): weights w_i = c (i + i0)^(-1/(gamma-1)),
// i0 and c chosen so that sum w = meanDeg * n and w_0 = sqrt(sum w) (the cap
// that keeps every w_i w_j / sum w <= 1).  round(sum w / 2) undirected edges
// are drawn with both endpoints ~ w (Vose alias table; draw j uses outputs
// 4j+1..4j+4 of SplitMix64(seed)); duplicates and self-loops are removed, and
// ids are relabeled by randomPerm(n, 1).
HostCsr genChungLu(uint32_t n, double gamma, double meanDeg, uint64_t seed) {
    if (gamma <= 1.0 || meanDeg <= 0 || n < 2) throw Error(GB_ERR_ARG, "chung_lu: bad parameters");
    const double a = 1.0 / (gamma - 1.0);
    const double total = meanDeg * n, wmax = std::sqrt(total);
    auto sumExact = [&](double i0) {  // sum_i (i + i0)^-a
        double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
        for (int64_t i = 0; i < (int64_t)n; ++i) s += std::pow((double)i + i0, -a);
        return s;
    };
    auto sumApprox = [&](double i0) {  // Euler-Maclaurin: integral + end correction
        double integral = std::fabs(1.0 - a) < 1e-12
                              ? std::log((n + i0) / i0)
                              : (std::pow(n + i0, 1.0 - a) - std::pow(i0, 1.0 - a)) / (1.0 - a);
        return integral + 0.5 * (std::pow(i0, -a) - std::pow(n + i0, -a));
    };
    // w_0 / mean = i0^-a / (sum / n): decreasing in i0.  Solve w_0 = wmax.
    double lo = 1e-3, hi = (double)n;
    for (int it = 0; it < 100; ++it) {
        double mid = std::sqrt(lo * hi);
        double w0 = std::pow(mid, -a) * total / sumApprox(mid);
        if (w0 > wmax) lo = mid; else hi = mid;
    }
    const double i0 = hi, c = total / sumExact(i0);
    std::vector<double> w(n);
    for (uint32_t i = 0; i < n; ++i) w[i] = std::min(wmax, c * std::pow(i + i0, -a));
    // Vose alias table over w.
    std::vector<double> prob(n);
    std::vector<uint32_t> alias(n, 0), small, large;
    double sw = 0;
    for (double x : w) sw += x;
    for (uint32_t i = 0; i < n; ++i) {
        prob[i] = w[i] * n / sw;
        (prob[i] < 1.0 ? small : large).push_back(i);
    }
    while (!small.empty() && !large.empty()) {
        uint32_t s = small.back(), l = large.back();
        small.pop_back();
        alias[s] = l;
        prob[l] = (prob[l] + prob[s]) - 1.0;
        if (prob[l] < 1.0) {
            large.pop_back();
            small.push_back(l);
        }
    }
    for (uint32_t i : large) prob[i] = 1.0;
    for (uint32_t i : small) prob[i] = 1.0;
    const uint64_t ne = (uint64_t)std::llround(sw / 2.0);
    const std::vector<uint32_t> perm = randomPerm(n, 1);
    std::vector<uint32_t> eu(ne), ev(ne);
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < (int64_t)ne; ++j) {
        uint64_t k = 4ull * j;
        uint64_t i1 = belowAt(seed, k + 1, n);
        uint32_t x = unitAt(seed, k + 2) < prob[i1] ? (uint32_t)i1 : alias[i1];
        uint64_t i2 = belowAt(seed, k + 3, n);
        uint32_t y = unitAt(seed, k + 4) < prob[i2] ? (uint32_t)i2 : alias[i2];
        eu[j] = perm[x];
        ev[j] = perm[y];
    }
    return csrFromEdges(n, eu.data(), ev.data(), ne, false);
}

// ------------------------------------------------------------------- I/O

void csrSave(const HostCsr& g, const std::string& path) {  // src/graph/csr.cpp:30-44
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) throw Error(GB_ERR_IO, "cannot write " + path);
    FileHeader h{};
    std::memcpy(h.magic, kMagic, 8);
    h.version = 1;
    h.flags = g.flags;
    h.num_vertices = g.n;
    h.num_edges = g.m;
    bool ok = std::fwrite(&h, sizeof h, 1, f) == 1 &&
              std::fwrite(g.row_ptr.data(), 4, g.n + 1, f) == g.n + 1 &&
              (g.m == 0 || std::fwrite(g.col_idx.data(), 4, g.m, f) == g.m);
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) throw Error(GB_ERR_IO, "short write to " + path);
}

HostCsr csrLoad(const std::string& path) {  // src/graph/csr.cpp:54-84 (read instead of mmap)
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw Error(GB_ERR_IO, "cannot open " + path);
    std::fseek(f, 0, SEEK_END);
    long len = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    FileHeader h{};
    if (len < (long)sizeof h || std::fread(&h, sizeof h, 1, f) != 1) {
        std::fclose(f);
        throw Error(GB_ERR_IO, path + ": too small");
    }
    if (std::memcmp(h.magic, kMagic, 8) != 0) {
        std::fclose(f);
        throw Error(GB_ERR_IO, path + ": bad magic");
    }
    if (h.version != 1) {
        std::fclose(f);
        throw Error(GB_ERR_IO, path + ": unsupported version");
    }
    uint64_t expect = sizeof h + 4 * (h.num_vertices + 1) + 4 * h.num_edges;
    if (expect != (uint64_t)len) {
        std::fclose(f);
        throw Error(GB_ERR_IO, path + ": size does not match header");
    }
    HostCsr g;
    g.n = h.num_vertices;
    g.m = h.num_edges;
    g.flags = h.flags;
    g.row_ptr.resize(g.n + 1);
    g.col_idx.resize(g.m);
    bool ok = std::fread(g.row_ptr.data(), 4, g.n + 1, f) == g.n + 1 &&
              (g.m == 0 || std::fread(g.col_idx.data(), 4, g.m, f) == g.m);
    std::fclose(f);
    if (!ok) throw Error(GB_ERR_IO, path + ": short read");
    return g;
}

// ------------------------------------------------------------ sources

// gbench's largestComponent + pickSources (src/bench/main.cpp:130-169).
std::vector<uint32_t> pickSources(const HostCsr& g, int count, uint64_t seed, bool anyComponent) {
    const uint64_t n = g.n;
    std::vector<uint8_t> ok(n, 1);
    if (!anyComponent && n) {
        std::vector<uint32_t> comp(n, kInf), q(n);
        uint32_t best = 0, id = 0;
        uint64_t bestSize = 0;
        for (uint64_t r = 0; r < n; ++r) {
            if (comp[r] != kInf) continue;
            uint64_t head = 0, tail = 0;
            comp[r] = id;
            q[tail++] = (uint32_t)r;
            while (head < tail) {
                uint32_t u = q[head++];
                for (uint32_t i = g.row_ptr[u]; i < g.row_ptr[u + 1]; ++i)
                    if (comp[g.col_idx[i]] == kInf) {
                        comp[g.col_idx[i]] = id;
                        q[tail++] = g.col_idx[i];
                    }
            }
            if (tail > bestSize) {
                bestSize = tail;
                best = id;
            }
            ++id;
        }
        for (uint64_t v = 0; v < n; ++v) ok[v] = comp[v] == best;
    }
    return drawSources(n, g.row_ptr.data(), ok, count, seed);
}

// The drawing half of pickSources: distinct vertices v = below(n) in the
// seeded stream, kept when ok[v] and degree(v) > 0.
std::vector<uint32_t> drawSources(uint64_t n, const uint32_t* row_ptr, const std::vector<uint8_t>& ok, int count,
                                  uint64_t seed) {
    uint64_t candidates = 0;
    for (uint64_t v = 0; v < n; ++v) candidates += ok[v] && row_ptr[v + 1] > row_ptr[v];
    count = (int)std::min<uint64_t>((uint64_t)std::max(count, 0), candidates);
    std::vector<uint32_t> out;
    std::vector<uint8_t> used(n, 0);
    uint64_t k = 0;
    while ((int)out.size() < count) {
        uint32_t v = (uint32_t)belowAt(seed, ++k, n);
        if (ok[v] && row_ptr[v + 1] > row_ptr[v] && !used[v]) {
            used[v] = 1;
            out.push_back(v);
        }
    }
    return out;
}

}  // namespace gb
