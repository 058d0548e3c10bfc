// graph_host.hpp -- host-side CSR type and builders (the src/graph layer of the
// reference: src/graph/csr.hpp:29-70, transform.hpp:11-19, generators.hpp:12-24).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace gb {

struct HostCsr {
    uint64_t n = 0, m = 0;
    uint32_t flags = 0;
    std::vector<uint32_t> row_ptr;  // n + 1
    std::vector<uint32_t> col_idx;  // m
    uint32_t degree(uint64_t v) const { return row_ptr[v + 1] - row_ptr[v]; }
};

// Counter-based SplitMix64: the k-th output (k >= 1) of the stream seeded with
// `seed` is mix(seed + k * golden).  Identical to stepping util::Rng
// (src/util/rng.hpp:8-26) k times, but lets threads draw disjoint stretches.
inline uint64_t splitmixAt(uint64_t seed, uint64_t k) {
    uint64_t z = seed + k * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
inline double unitAt(uint64_t seed, uint64_t k) {
    return (double)(splitmixAt(seed, k) >> 11) * (1.0 / 9007199254740992.0);
}
inline uint64_t belowAt(uint64_t seed, uint64_t k, uint64_t bound) {
    return (uint64_t)(((unsigned __int128)splitmixAt(seed, k) * bound) >> 64);
}

HostCsr csrFromEdges(uint64_t n, const uint32_t* eu, const uint32_t* ev, uint64_t ne, bool directed);
HostCsr csrTranspose(const HostCsr& g);
HostCsr csrSymmetrize(const HostCsr& g);
HostCsr csrPermute(const HostCsr& g, const uint32_t* perm);
std::vector<uint32_t> randomPerm(uint64_t n, uint64_t seed);
// reorder::compute (src/graph/reorder.cpp:94-100) on a symmetric graph:
// perm[old] = new for "original" | "random" | "degree" | "rcm".
std::vector<uint32_t> orderingPerm(const HostCsr& sym, const std::string& ordering, uint64_t seed);
// reorder::locality (src/graph/reorder.cpp:111-125).
void locality(const HostCsr& g, double* meanGap, double* sameBlock64);
std::string csrValidate(const HostCsr& g);

HostCsr genPath(uint32_t n);
HostCsr genStar(uint32_t leaves);
HostCsr genComplete(uint32_t n);
HostCsr genTwoComponents();
HostCsr genEmpty(uint32_t n);
HostCsr genGrid2d(uint32_t rows, uint32_t cols);
HostCsr genRmat(uint32_t scale, uint64_t edges, bool directed, uint64_t seed);
HostCsr genRoad(uint32_t rows, uint32_t cols, double dropFrac, double diagFrac, uint64_t seed);
HostCsr genWeb(uint32_t n, double outMean, double zipfS, uint64_t seed);
HostCsr genChungLu(uint32_t n, double gamma, double meanDeg, uint64_t seed);

void csrSave(const HostCsr& g, const std::string& path);
HostCsr csrLoad(const std::string& path);

std::vector<uint32_t> pickSources(const HostCsr& g, int count, uint64_t seed, bool anyComponent);
std::vector<uint32_t> drawSources(uint64_t n, const uint32_t* row_ptr, const std::vector<uint8_t>& ok, int count,
                                  uint64_t seed);

}  // namespace gb
