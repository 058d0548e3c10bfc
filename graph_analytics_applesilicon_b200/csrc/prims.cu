// prims.cu -- device-wide uint32 primitives.
//
// The reference scans frontier degrees with a recursive three-kernel scan
// (src/metal/primitives.mm:69-101, src/shaders/primitives.metal:75-120).  Here
// it is one launch: each block takes a ticket (so every lower tile has
// started), scans 2048 elements, publishes its aggregate and looks back over
// its predecessors' published values with one warp (Merrill & Garland's
// decoupled look-back).  Reductions use one atomic per warp; the
// queue<->bitmap conversions use a thread per 32-vertex word with
// warp-aggregated appends.
#include "prims.cuh"

#include <cuda.h>

#include <mutex>
#include <string>

#include "capi_util.hpp"

namespace gb {

namespace {

constexpr unsigned long long kFlagAgg = 1ull << 32, kFlagIncl = 2ull << 32;
constexpr unsigned long long kScanSpinLimit = 1ull << 24;

// Exclusive scan of one value per thread over a block of NT threads.
template <int NT>
__device__ __forceinline__ uint32_t blockExclusiveScan(uint32_t v, uint32_t* total, uint32_t* sm) {
    constexpr int W = NT / 32;
    const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(kFull, x, o);
        if ((int)lane >= o) x += y;
    }
    if (lane == 31) sm[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = lane < W ? sm[lane] : 0u, incl = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(kFull, incl, o);
            if ((int)lane >= o) incl += y;
        }
        if (lane < W) sm[lane] = incl - w;
        if (lane == W - 1) sm[W] = incl;
    }
    __syncthreads();
    uint32_t r = sm[wid] + x - v;
    *total = sm[W];
    __syncthreads();
    return r;
}

__device__ __forceinline__ unsigned long long ldStatus(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void stStatus(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__global__ void __launch_bounds__(kScanThreads) scanKernel(const uint32_t* in, uint32_t* out, uint64_t n,
                                                           uint32_t* total, unsigned long long* status,
                                                           unsigned* counters) {
    __shared__ uint32_t sTile, sPrefix;
    __shared__ uint32_t sWarp[kScanThreads / 32 + 1];
    if (threadIdx.x == 0) sTile = atomicAdd(&counters[0], 1u);
    __syncthreads();
    const uint32_t tile = sTile;
    const uint64_t base = (uint64_t)tile * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    const bool vec = base + kScanItems <= n && ((reinterpret_cast<uintptr_t>(in + base) & 15) == 0);
    if (vec) {
        uint4 a = *reinterpret_cast<const uint4*>(in + base);
        uint4 b = *reinterpret_cast<const uint4*>(in + base + 4);
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
        v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
    } else {
#pragma unroll
        for (int i = 0; i < kScanItems; ++i) v[i] = base + i < n ? in[base + i] : 0u;
    }
    uint32_t tsum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) tsum += v[i];
    uint32_t agg;
    const uint32_t excl = blockExclusiveScan<kScanThreads>(tsum, &agg, sWarp);

    if (threadIdx.x < 32) {
        const unsigned lane = threadIdx.x;
        uint32_t prefix = 0;
        if (tile == 0) {
            if (lane == 0) stStatus(&status[0], kFlagIncl | agg);
        } else {
            if (lane == 0) stStatus(&status[tile], kFlagAgg | agg);
            int64_t look = (int64_t)tile - 1;
            bool done = false;
            while (!done) {
                const int64_t idx = look - (int64_t)lane;
                unsigned long long s = kFlagIncl;  // below tile 0: an inclusive zero
                if (idx >= 0) {
                    unsigned long long polls = 0;
                    while (((s = ldStatus(&status[idx])) >> 32) == 0) {
                        if (++polls > kScanSpinLimit || ldVolatile(&counters[1])) {
                            atomicOr(&counters[1], 1u);
                            s = kFlagIncl;
                            break;
                        }
                    }
                }
                const unsigned incl = __ballot_sync(kFull, (s >> 32) == 2);
                const int first = incl ? __ffs(incl) - 1 : 32;
                uint32_t val = (int)lane <= first ? (uint32_t)s : 0u;
                prefix += warpSum(val);
                done = incl != 0;
                look -= 32;
            }
            if (lane == 0) stStatus(&status[tile], kFlagIncl | (uint32_t)(prefix + agg));
        }
        if (lane == 0) sPrefix = prefix;
    }
    __syncthreads();
    uint32_t run = sPrefix + excl;
    uint32_t o[kScanItems];
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        o[i] = run;
        run += v[i];
    }
    if (vec && ((reinterpret_cast<uintptr_t>(out + base) & 15) == 0)) {
        *reinterpret_cast<uint4*>(out + base) = make_uint4(o[0], o[1], o[2], o[3]);
        *reinterpret_cast<uint4*>(out + base + 4) = make_uint4(o[4], o[5], o[6], o[7]);
    } else {
#pragma unroll
        for (int i = 0; i < kScanItems; ++i)
            if (base + i < n) out[base + i] = o[i];
    }
    if (total && tile == gridDim.x - 1 && threadIdx.x == kScanThreads - 1) *total = run;
}

__global__ void reduceKernel(const uint32_t* in, uint64_t n, uint32_t* sum, uint32_t* mx) {
    uint32_t s = 0, m = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t x = in[i];
        s += x;
        m = max(m, x);
    }
    s = warpSum(s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(kFull, m, o));
    if (laneId() == 0) {
        if (sum && s) atomicAdd(sum, s);
        if (mx && m) atomicMax(mx, m);
    }
}

__global__ void queueToBitmapKernel(const uint32_t* queue, uint64_t size, uint32_t* bitmap) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < size; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t v = queue[i];
        atomicOr(&bitmap[v >> 5], 1u << (v & 31));
    }
}

// Thread per bitmap word; one atomic per warp reserves the warp's slots.
__global__ void bitmapToQueueKernel(const uint32_t* bitmap, uint64_t n, uint32_t* queue, uint32_t* count,
                                    const uint32_t* row_ptr, uint32_t* deg) {
    const uint64_t words = (n + 31) / 32;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t w0 = (uint64_t)blockIdx.x * blockDim.x; w0 < words; w0 += stride) {
        const uint64_t w = w0 + threadIdx.x;
        uint32_t word = 0;
        if (w < words) {
            word = bitmap[w];
            if (w == words - 1 && (n & 31)) word &= (1u << (n & 31)) - 1u;
        }
        uint32_t c = __popc(word), x = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(kFull, x, o);
            if ((int)laneId() >= o) x += y;
        }
        uint32_t warpTotal = __shfl_sync(kFull, x, 31), base = 0;
        if (laneId() == 31 && warpTotal) base = atomicAdd(count, warpTotal);
        base = __shfl_sync(kFull, base, 31);
        uint32_t pos = base + x - c;
        while (word) {
            uint32_t v = (uint32_t)(w * 32 + __ffs(word) - 1);
            word &= word - 1;
            queue[pos] = v;
            if (deg) deg[pos] = row_ptr[v + 1] - row_ptr[v];
            ++pos;
        }
    }
}

__global__ void fillKernel(uint32_t* p, uint32_t value, uint64_t n) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        p[i] = value;
}

uint32_t gridFor(uint64_t work, uint32_t threads) {
    uint64_t b = (work + threads - 1) / threads;
    uint64_t cap = (uint64_t)deviceSmCount() * 16;
    return (uint32_t)std::max<uint64_t>(1, std::min(b, cap));
}

}  // namespace

void scanExclusive(const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* total, ScanScratch& s,
                   cudaStream_t st) {
    if (n == 0) {
        if (total) GB_CUDA(cudaMemsetAsync(total, 0, 4, st));
        return;
    }
    const uint32_t tiles = divUp(n, kScanTile);
    s.status.ensure(tiles);
    s.counters.ensure(2);
    GB_CUDA(cudaMemsetAsync(s.status.get(), 0, (size_t)tiles * 8, st));
    GB_CUDA(cudaMemsetAsync(s.counters.get(), 0, 8, st));
    scanKernel<<<tiles, kScanThreads, 0, st>>>(in, out, n, total, s.status.get(), s.counters.get());
    GB_LAUNCH_CHECK();
}

void reduceSumMax(const uint32_t* in, uint64_t n, uint32_t* sum, uint32_t* max, cudaStream_t st) {
    if (n == 0) return;
    reduceKernel<<<gridFor(n, 256), 256, 0, st>>>(in, n, sum, max);
    GB_LAUNCH_CHECK();
}

void queueToBitmap(const uint32_t* queue, uint64_t size, uint32_t* bitmap, uint64_t n, cudaStream_t st) {
    const uint64_t words = (n + 31) / 32;
    if (words) GB_CUDA(cudaMemsetAsync(bitmap, 0, words * 4, st));
    if (size == 0) return;
    queueToBitmapKernel<<<gridFor(size, 256), 256, 0, st>>>(queue, size, bitmap);
    GB_LAUNCH_CHECK();
}

void bitmapToQueue(const uint32_t* bitmap, uint64_t n, uint32_t* queue, uint32_t* count,
                   const uint32_t* row_ptr, uint32_t* deg, cudaStream_t st) {
    const uint64_t words = (n + 31) / 32;
    if (words == 0) return;
    bitmapToQueueKernel<<<gridFor(words, 256), 256, 0, st>>>(bitmap, n, queue, count, row_ptr, deg);
    GB_LAUNCH_CHECK();
}

void fillU32(uint32_t* p, uint32_t value, uint64_t n, cudaStream_t st) {
    if (n == 0) return;
    fillKernel<<<gridFor(n, 256), 256, 0, st>>>(p, value, n);
    GB_LAUNCH_CHECK();
}

}  // namespace gb

// ------------------------------------------------------------------------
// Exclusive scan into caller-owned device memory that allocates nothing.
//
// scanExclusive above takes its look-back scratch from a buffer the caller's
// handle grows on demand.  Some callers cannot allocate device memory at the
// point where they need a scan: a host program that hands the whole GPU memory
// to its own pool at start-up and has none left to give, or a stream pipeline
// that must not call cudaMalloc / cudaFree between launches because those
// calls can wait for the whole device.  For them the same single-pass kernel
// runs here with its scratch in a fixed array in this module's global memory,
// which the CUDA runtime places when the module loads.
//
// Limits and rules (repeated in include/graph_b200.h):
//  * n <= kNoAllocScanMax (4096 tiles of 2048 elements = 8,388,608); larger n
//    is rejected with GB_ERR_CAPACITY before anything is enqueued.
//  * Every status word of the tiles in use, the tile ticket and the timeout
//    word must be zero when the kernel starts; each call clears them on its
//    stream (cudaMemsetAsync, which allocates nothing) before the launch.
//  * There is one scratch array per device, so two calls whose kernels
//    overlap on the same GPU (different streams, or host threads) race on it
//    and both results are undefined.  Order them on one stream or with events.
//  * The first call on a device looks up the array's device address
//    (cudaGetSymbolAddress, with that device current); make that first call
//    before any stream capture begins.  The address is remembered per device
//    together with the driver's unique id of the context it was found in: a
//    call under another context of that device (after cudaDeviceReset, or
//    under a context the caller created) looks the address up again, since
//    the module, and so the array, may then sit elsewhere.
// ------------------------------------------------------------------------
// [0, 4096): per-tile look-back status words; [4096]: tile ticket (low 32
// bits) and timeout flag (high 32 bits).  32 KiB + 8 bytes per device.
static __device__ __align__(256) unsigned long long gNoAllocScanScratch[4096 + 1];

namespace gb {
namespace {

constexpr uint32_t kNoAllocScanTiles = 4096;  // the size of gNoAllocScanScratch - 1
constexpr uint64_t kNoAllocScanMax = (uint64_t)kNoAllocScanTiles * kScanTile;
static_assert(sizeof(gNoAllocScanScratch) == (kNoAllocScanTiles + 1) * sizeof(unsigned long long),
              "scratch array and tile limit disagree");
constexpr int kNoAllocMaxDevices = 64;

std::mutex gNoAllocMu;
unsigned long long* gNoAllocScratchPtr[kNoAllocMaxDevices] = {};
unsigned long long gNoAllocCtxId[kNoAllocMaxDevices] = {};

// The driver's unique id of the calling thread's current context (ids are
// never reused within a process), or 0 when there is none yet or the driver
// cannot tell.  The two driver calls are reached through the runtime's entry
// point table, so the library needs no link against the driver library.
unsigned long long currentContextId() {
    struct Fns {
        CUresult (*current)(CUcontext*) = nullptr;
        CUresult (*id)(CUcontext, unsigned long long*) = nullptr;
    };
    static const Fns f = [] {
        Fns r;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            r.current = reinterpret_cast<CUresult (*)(CUcontext*)>(p);
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            r.id = reinterpret_cast<CUresult (*)(CUcontext, unsigned long long*)>(p);
        return r;
    }();
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (f.current && f.id && f.current(&c) == CUDA_SUCCESS && c && f.id(c, &id) == CUDA_SUCCESS) return id;
    return 0;
}

// Device address of the scratch array on the current device; looked up on
// the first call for that device and again whenever the current context of
// that device is not the one the address was found in.
unsigned long long* noAllocScanScratch() {
    int dev = 0;
    GB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices)
        throw Error(GB_ERR_ARG, "no-allocation scan supports device ordinals below 64");
    std::lock_guard<std::mutex> lock(gNoAllocMu);
    const unsigned long long ctx = currentContextId();
    if (!gNoAllocScratchPtr[dev] || ctx == 0 || ctx != gNoAllocCtxId[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, gNoAllocScanScratch);
        if (e != cudaSuccess || !p)
            throw Error(GB_ERR_CUDA, std::string("cudaGetSymbolAddress(scan scratch) failed: ") +
                                         cudaGetErrorString(e));
        gNoAllocScratchPtr[dev] = static_cast<unsigned long long*>(p);
        gNoAllocCtxId[dev] = currentContextId();  // the lookup made the context current if none was
    }
    return gNoAllocScratchPtr[dev];
}

}  // namespace
}  // namespace gb

extern "C" int gb_prim_scan_device_noalloc(const uint32_t* in, uint64_t n, uint32_t* out, uint32_t* total,
                                           uint32_t* timeout_flag, void* stream) {
    using namespace gb;
    return guard([&] {
        GB_REQUIRE(n == 0 || (in && out), "null argument");
        if (n > kNoAllocScanMax)
            throw Error(GB_ERR_CAPACITY, "no-allocation scan: n = " + std::to_string(n) + " exceeds its limit of " +
                                             std::to_string(kNoAllocScanMax) + " elements");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        unsigned long long* scratch = noAllocScanScratch();
        unsigned* counters = reinterpret_cast<unsigned*>(scratch + kNoAllocScanTiles);
        if (n == 0) {
            if (total) GB_CUDA(cudaMemsetAsync(total, 0, 4, st));
            if (timeout_flag) GB_CUDA(cudaMemsetAsync(timeout_flag, 0, 4, st));
            return;
        }
        const uint32_t tiles = divUp(n, kScanTile);
        GB_CUDA(cudaMemsetAsync(scratch, 0, (size_t)tiles * sizeof(unsigned long long), st));
        GB_CUDA(cudaMemsetAsync(counters, 0, 2 * sizeof(unsigned), st));
        scanKernel<<<tiles, kScanThreads, 0, st>>>(in, out, n, total, scratch, counters);
        GB_LAUNCH_CHECK();
        if (timeout_flag)
            GB_CUDA(cudaMemcpyAsync(timeout_flag, counters + 1, sizeof(unsigned), cudaMemcpyDeviceToDevice, st));
    });
}
