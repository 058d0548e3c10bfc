// ref_shim.cpp -- extern "C" access to the reference's own CPU code.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with
// the reference's unmodified sources (src/cpu/{bfs_cpu,pagerank_cpu}.cpp,
// src/graph/{csr,transform,generators,reorder,snap}.cpp, read in place) into
// oracle/_ref/libgref.so.  Tests use it to pin the C restatement in oracle.c,
// tests/golden/make_golden.py uses it to write the golden fixtures, and
// bench.py times it as the CPU baseline (cpu_do / cpu_omp on all host cores).
// Nothing here re-implements an algorithm: every call goes to the reference.
#include "cpu/bfs_cpu.hpp"
#include "cpu/pagerank_cpu.hpp"
#include "graph/csr.hpp"
#include "graph/generators.hpp"
#include "graph/reorder.hpp"
#include "graph/snap.hpp"
#include "graph/transform.hpp"

#include <omp.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {
struct Handle {
    graph::CSR g;
};
Handle* wrap(graph::CSR g) { return new Handle{std::move(g)}; }
const graph::CSR& csr(void* h) { return static_cast<Handle*>(h)->g; }
}  // namespace

extern "C" {

int gref_max_threads() { return omp_get_max_threads(); }

void* gref_suite(const char* name) {
    for (auto& [n, g] : graph::gen::suite())
        if (n == name) return wrap(g);
    return nullptr;
}
void* gref_path(uint32_t n) { return wrap(graph::gen::path(n)); }
void* gref_star(uint32_t leaves) { return wrap(graph::gen::star(leaves)); }
void* gref_complete(uint32_t n) { return wrap(graph::gen::complete(n)); }
void* gref_grid2d(uint32_t r, uint32_t c) { return wrap(graph::gen::grid2d(r, c)); }
void* gref_rmat(uint32_t scale, uint32_t ef, int directed, uint64_t seed) {
    return wrap(graph::gen::rmat(scale, ef, directed != 0, seed));
}
void* gref_from_arrays(uint64_t n, uint64_t m, uint32_t flags, const uint32_t* rp, const uint32_t* ci) {
    std::vector<uint32_t> r(rp, rp + n + 1), c(ci, ci + m);
    return wrap(graph::CSR::fromVectors(std::move(r), std::move(c), flags));
}
void* gref_from_edges(uint64_t n, const uint32_t* eu, const uint32_t* ev, uint64_t ne, int directed) {
    std::vector<std::pair<uint32_t, uint32_t>> e(ne);
    for (uint64_t i = 0; i < ne; ++i) e[i] = {eu[i], ev[i]};
    return wrap(graph::fromEdgeList(n, e, directed != 0));
}
void* gref_symmetrize(void* h) { return wrap(graph::symmetrize(csr(h))); }
void* gref_transpose(void* h) { return wrap(graph::transpose(csr(h))); }
void* gref_permute(void* h, const uint32_t* perm) {
    return wrap(graph::permute(csr(h), std::vector<uint32_t>(perm, perm + csr(h).n)));
}
void gref_ordering(void* h, const char* ordering, uint64_t seed, uint32_t* out) {
    auto p = graph::reorder::compute(csr(h), ordering, seed);
    std::memcpy(out, p.data(), p.size() * 4);
}
void gref_locality(void* h, double* mean_gap, double* same_block64) {
    graph::reorder::Locality l = graph::reorder::locality(csr(h));
    *mean_gap = l.meanGap;
    *same_block64 = l.sameBlock64;
}
uint64_t gref_n(void* h) { return csr(h).n; }
uint64_t gref_m(void* h) { return csr(h).m; }
uint32_t gref_flags(void* h) { return csr(h).flags; }
void gref_copy(void* h, uint32_t* rp, uint32_t* ci) {
    const graph::CSR& g = csr(h);
    std::memcpy(rp, g.row_ptr, (g.n + 1) * 4);
    if (g.m) std::memcpy(ci, g.col_idx, g.m * 4);
}
int gref_validate(void* h) { return graph::validate(csr(h)).empty() ? 0 : 1; }
void gref_free(void* h) { delete static_cast<Handle*>(h); }

void gref_bfs_serial(void* h, uint32_t src, uint32_t* dist) { cpu::bfsSerial(csr(h), src, dist); }

void gref_bfs_omp(void* h, uint32_t src, uint32_t* dist, int threads) {
    cpu::BfsOptions o;
    o.threads = threads;
    cpu::bfsOmp(csr(h), src, dist, o);
}

// Returns the number of levels; per-level records go to the arrays (cap entries).
int gref_bfs_do(void* h, uint32_t src, uint32_t* dist, double alpha, double beta, int threads,
                uint32_t* level, char* dir, uint64_t* frontier, uint64_t* edges, int cap) {
    cpu::BfsOptions o;
    o.alpha = alpha;
    o.beta = beta;
    o.threads = threads;
    std::vector<util::BfsLevel> tr;
    cpu::bfsDO(csr(h), src, dist, o, level ? &tr : nullptr);
    for (int i = 0; i < (int)tr.size() && i < cap; ++i) {
        level[i] = tr[i].level;
        dir[i] = tr[i].direction;
        frontier[i] = tr[i].frontier;
        edges[i] = tr[i].edges;
    }
    return (int)tr.size();
}

// threads < 0: pagerankSerial; otherwise pagerankOmp with that many threads (0 = all).
int gref_pagerank(void* in, const uint32_t* outdeg, double* r, int iters, double tol, int threads,
                  double* last_delta) {
    cpu::PrOptions o;
    o.iters = iters;
    o.tol = tol;
    o.threads = threads < 0 ? 0 : threads;
    cpu::PrResult res = threads < 0 ? cpu::pagerankSerial(csr(in), outdeg, r, o)
                                    : cpu::pagerankOmp(csr(in), outdeg, r, o);
    if (last_delta) *last_delta = res.lastDelta;
    return res.iters;
}

void gref_check_ranks_f32(const double* ref, const float* got, uint64_t n, double* l1, double* rel,
                          double* sum) {
    std::vector<double> r(ref, ref + n);
    cpu::PrCheck c = cpu::checkRanks(r, got);
    *l1 = c.l1;
    *rel = c.maxRelTop;
    *sum = c.sum;
}

// graph::convertSnap then graph::load of its output.  Returns the loaded
// graph, or null with the exception's text in msg.  stats: lines, raw_max_id,
// n, m_before, m.
void* gref_convert_snap(const char* in, const char* out, int directed, uint64_t* stats, char* msg,
                        size_t cap) {
    try {
        graph::ConvertStats st = graph::convertSnap(in, out, directed != 0);
        stats[0] = st.lines;
        stats[1] = st.raw_max_id;
        stats[2] = st.n;
        stats[3] = st.m_before;
        stats[4] = st.m;
        return wrap(graph::load(out));
    } catch (const std::exception& e) {
        std::snprintf(msg, cap, "%s", e.what());
        return nullptr;
    }
}

}  // extern "C"
