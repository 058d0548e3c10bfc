// pagerank.hpp -- the PageRank handle behind gb_pr_* (the role of
// gpu::GpuPageRank, src/metal/pagerank_gpu.hpp:46-127).
#pragma once

#include <map>
#include <tuple>
#include <vector>

#include "common.cuh"

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
};

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

    // adaptive bins (in-degree): one buffer holding list0 | list1 | list2
    gb::DevBuf<uint32_t> bins;
    uint32_t binCount[3] = {0, 0, 0};
    uint32_t binSmall = 0, binLarge = 0;
    bool binsReady = false;

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

    // cached CUDA graphs of iteration batches
    std::map<std::tuple<int, int, int, int, int, int, int>, cudaGraphExec_t> graphs;
    int grid = 0;

    ~gb_pr();
    void invalidateGraphs();
    void prepareAdaptive(uint32_t smallMax, uint32_t largeMin);
    void prepareGS(uint32_t pairMaxOutdeg);
    gb_pr_result run(int variant, const gb_pr_options& o);
    void ranks(float* out);
    void ranks64(double* out);
};
