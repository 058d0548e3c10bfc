// pagerank.hpp -- the PageRank handle behind gb_pr_* (the role of
// gpu::GpuPageRank, src/metal/pagerank_gpu.hpp:46-127).
#pragma once

#include <map>
#include <tuple>
#include <vector>

#include "common.cuh"

constexpr uint32_t kGsHubMin = 4096;  // natural-order GS: split vertices with this many in-edges
constexpr uint32_t kGsNatSlices = 8;    // natural-order GS: the main list runs as this many ordered launches

// Iteration control, updated on the device by the last block of every
// iteration kernel: which rank buffer is current, how many iterations ran,
// and the tol-mode stop rule (L1 change, max relative change, stagnation
// guard of src/metal/pagerank_gpu.mm:384-402).  Kernels launched after a stop
// return immediately, so iteration batches can be CUDA-graph replays.
struct GbPrControl {
    int cur;
    int iters;
    int stopped;
    int floorStop;
    int sinceBest;
    int cap;
    unsigned done;  // last-block-done ticket
    int withDelta;
    double best;
    double lastDelta;
    double lastMaxRel;
    double tol;
    double tolRel;
    float dangHi, dangLo;   // dangling rank of the current iterate (float-float)
    double dang64;          // same, double-precision variant
    double sum64;           // in-place variants: sum of the new iterate
    int error;              // a bounded device wait gave up (the run is invalid)
};

// Blocked pull (GB_PR_PULL_BLOCKED): rows in blocks of at most kBlkRowCap
// (their sums in shared memory, one CUDA block per row block), columns in
// parts of kBlkPart vertices (their contributions staged in shared memory by
// TMA, kBlkCStages parts at a time); tile (row block, part) holds that block's
// edges from that part as packed 32-bit words, staged by TMA in chunks of at
// most kBlkChunk 16-byte words, kBlkEStages chunks at a time.  One producer
// warp issues the copies; kBlkConsumerWarps warps add the edges.  Rows with
// kBlkHub or more in-edges are summed apart.
constexpr uint32_t kBlkPart = 8192;
constexpr uint32_t kBlkRowCap = 21504;
constexpr int kBlkCStages = 2;
constexpr int kBlkEStages = 4;
constexpr int kBlkThreads = 1024;
constexpr int kBlkConsumerWarps = kBlkThreads / 32 - 1;
constexpr uint32_t kBlkChunk = kBlkConsumerWarps * 32;  // one 16-byte word per consumer thread
constexpr uint32_t kBlkHub = 4096;  // rows with this many in-edges are summed apart, one block each

struct gb_pr {
    uint64_t n = 0, mOut = 0, mIn = 0;
    bool hasOut = false, hasIn = false;
    gb::DevBuf<uint32_t> rowOut, colOut, rowIn, colIn, outdeg;
    gb::DevBuf<float> r[2], contrib[2], acc, accLo;
    gb::DevBuf<double> r64[2], contrib64[2];
    gb::DevBuf<GbPrControl> ctl;
    gb::DevBuf<float> partF;       // per-block float partials (2 per block)
    gb::DevBuf<double> partD;      // per-block double partials (2 per block)
    gb::Stream stream;
    gb::EventPair ev;
    std::vector<uint32_t> hostRowIn, hostColIn, hostOutdeg;

    // adaptive pull: hub-first relabeled in-CSR (new id = rank by descending
    // in-degree), so every degree bin is a contiguous id range
    gb::DevBuf<uint32_t> rowA, colA, outdegA;
    gb::DevBuf<uint4> hubChunks;     // (vertex, start, end, hub index) per chunk
    gb::DevBuf<uint32_t> hubFirst;   // per hub: first chunk | chunk count
    gb::DevBuf<unsigned> hubDone;    // per hub: chunks finished (reset by the last)
    gb::DevBuf<float> hubPart;       // per chunk: Kahan sum, compensation
    std::vector<uint32_t> permA;     // old id -> new id
    uint32_t nHubs = 0, nChunks = 0;
    uint32_t binLo[8] = {0}, binHi[8] = {0}, binG[8] = {0};  // group-size ranges (G = 1..32)
    int nBins = 0;
    uint32_t binSmall = 0, binLarge = 0;
    bool binsReady = false;
    // Gauss-Seidel natural order: vertices of in-degree >= kGsHubMin are split
    // into warp chunks (natural ids) and swept first, in place
    gb::DevBuf<uint4> gsHubChunks;
    gb::DevBuf<uint32_t> gsHubFirst;
    gb::DevBuf<unsigned> gsHubDone;
    gb::DevBuf<float> gsHubPart;
    uint32_t gsHubs = 0, gsChunks = 0;
    // colored order: per colour set, its degree classes and its chunk range
    struct GsSetLayout {
        uint32_t lo[8], hi[8], g[8];
        int nBins;
        uint32_t chunk0, chunk1;
    };
    std::vector<GsSetLayout> gsSetLayout;

    // Gauss-Seidel order (prepareGS)
    bool gsReady = false, gsColored = false;
    uint32_t gsPairK = 0;
    size_t gsDeferred = 0;
    gb::DevBuf<uint32_t> gsNat;          // natural order: list A | list B
    uint32_t gsNatA = 0, gsNatB = 0;
    std::vector<uint32_t> gsSetStart;    // colored: set k = ids [start[k], start[k+1])
    gb::DevBuf<uint32_t> rowGS, colGS, outdegGS;
    std::vector<uint32_t> gsNewId;
    bool gsLastRun = false;
    int lastVariant = -1;

    // blocked pull: packed (row in block << 16 | column in part) per edge,
    // grouped by row block then part; blkOff[k * nParts + p] starts tile
    // (k, p), in 16-byte words
    gb::DevBuf<uint32_t> blkEdges, blkOff, blkHubs;
    uint32_t nRowBlocks = 0, rowsPer = 0, nParts = 0, nBlkHubs = 0;
    bool blkReady = false;

    // cached CUDA graphs of iteration batches
    std::map<std::tuple<int, int, int, int, int, int, int>, cudaGraphExec_t> graphs;
    int grid = 0;

    ~gb_pr();
    void invalidateGraphs();
    void prepareAdaptive(uint32_t smallMax, uint32_t largeMin);
    void prepareGS(uint32_t pairMaxOutdeg);
    void prepareBlocked();
    gb_pr_result run(int variant, const gb_pr_options& o);
    void ranks(float* out);
    void ranks64(double* out);
};
