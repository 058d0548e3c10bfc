// gather_bound.cu -- the rate at which one sweep's 4-byte contribution gathers can run
// on this GPU, measured on a graph's real in-lists.  Every kernel sums
// contrib[col[e]] over all edges with every lane busy and the column indices
// read as coalesced 16-byte words, so no PageRank pull (which must also find
// row boundaries and store ranks) can gather faster than these:
//   gbEdgeSum   contributions gathered through the read-only path (ld.global.nc)
//   gbEdgeSmem  contributions of ids < H served from a shared-memory copy
//   gbRandSum   the same number of gathers at uniform random ids (a hash of
//               the edge index) over the same array: no graph locality
// Every index is read from a column array whose entries are < n, or reduced
// modulo n; `nvec` 16-byte words of `col` must be readable.  Built and driven by
// gather_bound.py in this directory.
#include <cstdint>
#include <cuda_runtime.h>

namespace {

__device__ __forceinline__ uint4 ldWord(const uint32_t* p) {
    uint4 v;
    asm("ld.global.nc.L1::no_allocate.v4.u32 {%0, %1, %2, %3}, [%4];"
        : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
        : "l"(p));
    return v;
}

__device__ __forceinline__ void addOut(float acc, float* out) {
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, acc);
}

__global__ void gbEdgeSum(const uint32_t* __restrict__ col, uint64_t nvec, const float* __restrict__ contrib,
                          float* out) {
    float acc = 0.f;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nvec; i += stride) {
        const uint4 q = ldWord(col + 4 * i);
        acc += __ldg(contrib + q.x) + __ldg(contrib + q.y) + __ldg(contrib + q.z) + __ldg(contrib + q.w);
    }
    addOut(acc, out);
}

__device__ __forceinline__ float pick(const float* sm, const float* __restrict__ g, uint32_t u, uint32_t h) {
    return u < h ? sm[u] : __ldg(g + u);
}

__global__ void gbEdgeSmem(const uint32_t* __restrict__ col, uint64_t nvec, const float* __restrict__ contrib,
                           float* out, uint32_t h) {
    extern __shared__ float sm[];
    for (uint32_t i = threadIdx.x; i < h; i += blockDim.x) sm[i] = __ldg(contrib + i);
    __syncthreads();
    float acc = 0.f;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nvec; i += stride) {
        const uint4 q = ldWord(col + 4 * i);
        acc += pick(sm, contrib, q.x, h) + pick(sm, contrib, q.y, h) + pick(sm, contrib, q.z, h) +
               pick(sm, contrib, q.w, h);
    }
    addOut(acc, out);
}

__device__ __forceinline__ uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

__global__ void gbRandSum(uint64_t nvec, const float* __restrict__ contrib, uint32_t n, float* out) {
    float acc = 0.f;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nvec; i += stride) {
        const uint32_t e = (uint32_t)i * 4u;
        acc += __ldg(contrib + mix32(e) % n) + __ldg(contrib + mix32(e + 1) % n) + __ldg(contrib + mix32(e + 2) % n) +
               __ldg(contrib + mix32(e + 3) % n);
    }
    addOut(acc, out);
}

}  // namespace

// kind 0: gbEdgeSum, 1: gbEdgeSmem (h contributions, h * 4 bytes <= 200 KB), 2: gbRandSum.
// Returns the launch's CUDA error code, or -1 for a bad kind or size.
extern "C" int gb_gather_probe(int kind, const uint32_t* col, uint64_t nvec, const float* contrib, uint32_t n,
                               uint32_t h, float* out, int blocks, int threads, cudaStream_t s) {
    if (kind == 0) {
        gbEdgeSum<<<blocks, threads, 0, s>>>(col, nvec, contrib, out);
    } else if (kind == 1) {
        if (h == 0 || h > n || (size_t)h * 4 > 200 * 1024) return -1;
        cudaError_t e = cudaFuncSetAttribute(gbEdgeSmem, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        if (e != cudaSuccess) return (int)e;
        gbEdgeSmem<<<blocks, threads, (size_t)h * 4, s>>>(col, nvec, contrib, out, h);
    } else if (kind == 2) {
        if (n == 0) return -1;
        gbRandSum<<<blocks, threads, 0, s>>>(nvec, contrib, n, out);
    } else {
        return -1;
    }
    return (int)cudaGetLastError();
}
