// bfs.hpp -- the BFS handle behind gb_bfs_* (the role of gpu::GpuBfs,
// src/metal/bfs_gpu.hpp:35-105).
#pragma once

#include <memory>
#include <vector>

#include "common.cuh"
#include "prims.cuh"
#include "selector.cuh"

// Per-level counters of the host-driven forms (layout of the reference's
// stats buffer, src/shaders/bfs.metal:7-21, widened to 64-bit sums).
struct GbLevelStats {
    unsigned found;      // vertices discovered (next frontier size / queue tail)
    unsigned bin[3];     // gpu_binned: next-level small / medium / large queue tails
    unsigned long long frontier;   // vertices in the input frontier
    unsigned long long edges;      // adjacency entries examined
    unsigned long long nextEdges;  // sum of the discovered vertices' degrees
};

// Counters of one level of the persistent kernels (triple-buffered by level).
struct GbPCounters {
    unsigned qtail;              // next frontier: entries in the vertex queue
    unsigned work;               // dynamic work-item ticket of this level
    unsigned long long hubPack;  // next frontier hubs: (count << 40) | sum of their degrees
    unsigned long long nextEdges;// sum of degrees of everything discovered this level
    unsigned long long examined; // adjacency entries examined (bottom-up)
    unsigned long long found;    // vertices discovered this level
    unsigned long long pad[2];
};

struct gb_bfs;
namespace gb {
// Copies count depths from device d to host out (uint32, unreached ~0), packed
// to 1 or 2 bytes per depth over PCIe when `levels` allows (depth_out.cu).
void copyDepthsToHost(gb_bfs* h, const uint32_t* d, uint64_t count, uint32_t* out, uint32_t levels);
// The same packing as stages of a pipeline: packFormat picks the width for a
// traversal of `levels` levels (0: 4 bits, 1: 1 byte, 2: 2 bytes per depth;
// -1: send uint32), enqueuePack packs on `st` (sets *overflow when a depth does
// not fit), widenPacked turns the copied bytes back into uint32 on the host.
int packFormat(uint64_t count, uint32_t levels);
uint64_t packedBytes(int fmt, uint64_t count);
void enqueuePack(int fmt, const uint32_t* d, uint64_t count, uint8_t* dev, unsigned* overflow, cudaStream_t st);
void widenPacked(int fmt, const uint8_t* in, uint64_t count, uint32_t* out);
constexpr int kMaxInFlight = 16;              // traversals at once in gb_bfs::runPersistentMany
constexpr int kManySlots = kMaxInFlight + 2;  // depth buffers it rotates (in flight + 2)
}  // namespace gb

struct gb_bfs {
    uint64_t n = 0, m = 0;
    std::vector<uint32_t> hostRowPtr;  // degrees of sources on the host
    gb::DevBuf<uint32_t> rowPtr, colIdx, dist;
    bool hubFirst = false;  // adjacency lists re-sorted hub-first (gb_bfs_hub_first)
    uint32_t flags = 0;     // the graph's GGPUCSR1 flags when known (file handles)
    gb::Stream stream;
    gb::EventPair ev;
    gb::ScanScratch scan;

    // host-driven forms
    gb::DevBuf<GbLevelStats> stats;
    gb::HostPinned<GbLevelStats> hstats;
    gb::HostPinned<uint32_t> hstage;
    gb::DevBuf<uint32_t> qA, qB, degA, degB, bins[2][3], bmFront, bmNext;

    // persistent single-source
    gb::DevBuf<uint32_t> pq[2][3];       // queue: vertex, adjacency start, degree
    gb::DevBuf<uint32_t> phub[2][2];     // hub list: vertex, adjacency start
    gb::DevBuf<unsigned long long> phubOff[2];
    gb::DevBuf<uint32_t> pbm[3];         // frontier bitmaps
    gb::DevBuf<uint32_t> pvisited;       // visited bitmap
    gb::DevBuf<uint32_t> pIso;           // degree-0 vertices, a bit each (visited from the start)
    bool pIsoReady = false;
    gb::DevBuf<GbPCounters> pctr;        // [3]
    gb::DevBuf<unsigned> pctl;           // [0] barrier, [1] error, [2] levels, [3] flags
    gb::DevBuf<gb_level> ptrace;
    gb::DevBuf<double> pstate;           // level state for resumable (profiling) runs
    int pGrid = 0, pBlock = 0, pMax = 0, pWant = 0;
    // further traversals in flight in runPersistentMany: the same per-traversal
    // state (slot 0 is the members above) and a stream each
    struct PSlot {
        gb::DevBuf<uint32_t> q[2][3], hub[2][2], bm[3], visited;
        gb::DevBuf<unsigned long long> hubOff[2];
        gb::DevBuf<GbPCounters> ctr;
        gb::DevBuf<gb_level> trace;
        gb::DevBuf<double> state;
    };
    PSlot pSlot[gb::kMaxInFlight - 1];
    std::unique_ptr<gb::Stream> pStream[gb::kMaxInFlight - 1];  // created on first use

    // batched (64 sources)
    gb::DevBuf<unsigned long long> bSeen, bFront[2], bNext;
    gb::DevBuf<uint32_t> bActive[2], bCand, bHubV[2];
    gb::DevBuf<unsigned long long> bHubOff[2];
    gb::DevBuf<uint32_t> bDist;          // k * n results
    gb::DevBuf<uint2> bDefer;            // bottom-up: lists whose rest a whole block scans
    int bGrid = 0, bBlock = 0, bMax = 0;

    // learned selector parameters (single-source, batched)
    gb::DevBuf<float> selParams[2];
    bool selLoaded[2] = {false, false};

    // packed depth transfer to the host (depth_out.cu)
    gb::DevBuf<uint8_t> packDev;
    gb::HostPinned<uint8_t> packHost;
    gb::DevBuf<unsigned> packFlag;
    gb::HostPinned<unsigned> packFlagHost;
    std::vector<cudaEvent_t> packEv;

    // several sources per call (runPersistentMany): depth buffers besides
    // dist, per-slot packed copies, per-source control words and events
    gb::DevBuf<uint32_t> mDist[gb::kManySlots - 1];
    gb::DevBuf<uint8_t> mPackDev[gb::kManySlots];
    gb::HostPinned<uint8_t> mPackHost[gb::kManySlots];
    gb::DevBuf<unsigned> mCtl, mFlag;
    gb::HostPinned<unsigned> mCtlHost, mFlagHost;
    std::vector<cudaEvent_t> mEv, mSlotEv;
    gb::Stream copyStream;
    ~gb_bfs() {
        for (cudaEvent_t e : packEv) cudaEventDestroy(e);
        for (cudaEvent_t e : mEv) cudaEventDestroy(e);
        for (cudaEvent_t e : mSlotEv) cudaEventDestroy(e);
    }

    double lastGpuMs = 0;
    uint32_t lastLevels = 0;

    uint32_t degree(uint32_t v) const { return hostRowPtr[v + 1] - hostRowPtr[v]; }

    void runVertex(uint32_t src, const gb_bfs_options& o, std::vector<gb_level>* tr);
    void runNaive(uint32_t src, const gb_bfs_options& o, std::vector<gb_level>* tr);
    void runBinned(uint32_t src, const gb_bfs_options& o, std::vector<gb_level>* tr);
    void runEdge(uint32_t src, const gb_bfs_options& o, std::vector<gb_level>* tr);
    void runDirOpt(uint32_t src, const gb_bfs_options& o, std::vector<gb_level>* tr);
    void runPersistent(uint32_t src, const gb_bfs_options& o, std::vector<gb_level>* tr);
    void runBatch(const uint32_t* src, int k, const gb_bfs_options& o, std::vector<gb_level>* tr);
    void runPersistentMany(const uint32_t* src, uint32_t count, uint32_t* out, uint64_t stride,
                           const gb_bfs_options& o, float* ms, uint32_t* levels);
    void runBatchMany(const uint32_t* src, uint32_t count, uint32_t* out, uint64_t stride,
                      const gb_bfs_options& o, float* ms, uint32_t* levels);
    // Profiling (selector training data).
    size_t profileLevels(uint32_t src, const gb_bfs_options& o, int repeats, float* feats, float* times,
                         size_t cap);
    size_t profileBatchLevels(const uint32_t* src, int k, const gb_bfs_options& o, int repeats,
                              float* feats, float* times, size_t cap);

    // internal helpers
    void beginLevel();
    void endLevel();  // copy stats, sync, accumulate GPU time
    void initDist(uint32_t src);
    void ensureEdgeBuffers();
    void ensurePersistent(const gb_bfs_options& o);
    void ensureBatch(const gb_bfs_options& o, int k);
};

namespace gb {
uint32_t checkTg(uint32_t tg);
void validateOptions(const gb_bfs_options& o);
}  // namespace gb
