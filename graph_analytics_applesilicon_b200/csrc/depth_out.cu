// depth_out.cu -- returning BFS depths to host memory.  A depth array is
// 4 bytes per vertex, but a traversal of L levels only needs depths below L:
// when L < 15 (255, 65535) the depths travel over PCIe as 4 bits (1 byte,
// 2 bytes) per vertex, sentinel all ones for unreached, in chunks whose host-side widening to
// uint32 (OpenMP threads) overlaps the copy of the next chunk.  The pack
// kernel also checks every depth against the width, so a wrong level count
// can only cost a plain copy, never a wrong result.
#include <omp.h>

#include <algorithm>
#include <cstring>

#include "bfs.hpp"

namespace gb {
namespace {

constexpr uint64_t kPackMin = 1u << 18;   // smaller arrays go as one plain copy
constexpr uint64_t kPackChunk = 1u << 20;  // vertices per pipelined chunk

template <typename T>
__global__ void packDepthsKernel(const uint32_t* d, uint64_t count, T* out, unsigned* overflow) {
    const uint32_t sentinel = (uint32_t)(T)~0u;
    bool bad = false;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = d[i];
        bad |= v != 0xFFFFFFFFu && v >= sentinel;
        out[i] = v == 0xFFFFFFFFu ? (T)sentinel : (T)v;
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(overflow, 1u);
}

// Two depths per byte (low nibble first), 0xF for unreached; depths must be < 15.
__global__ void packDepths4Kernel(const uint32_t* d, uint64_t count, uint8_t* out, unsigned* overflow) {
    bool bad = false;
    const uint64_t pairs = (count + 1) / 2;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < pairs; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v0 = d[2 * i], v1 = 2 * i + 1 < count ? d[2 * i + 1] : 0xFFFFFFFFu;
        bad |= (v0 != 0xFFFFFFFFu && v0 >= 15u) || (v1 != 0xFFFFFFFFu && v1 >= 15u);
        const uint32_t a = v0 == 0xFFFFFFFFu ? 15u : (v0 & 15u), b = v1 == 0xFFFFFFFFu ? 15u : (v1 & 15u);
        out[i] = (uint8_t)(a | (b << 4));
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(overflow, 1u);
}

void widen4(const uint8_t* in, uint32_t* out, uint64_t count) {  // count even, or the array's tail
    const int threads = std::max(1, std::min(16, omp_get_max_threads()));
    const int64_t pairs = (int64_t)(count / 2);
#pragma omp parallel for num_threads(threads) schedule(static) if (count >= (1u << 16))
    for (int64_t i = 0; i < pairs; ++i) {
        const uint32_t b = in[i], lo = b & 15u, hi = b >> 4;
        out[2 * i] = lo == 15u ? 0xFFFFFFFFu : lo;
        out[2 * i + 1] = hi == 15u ? 0xFFFFFFFFu : hi;
    }
    if (count & 1) {
        const uint32_t lo = in[pairs] & 15u;
        out[count - 1] = lo == 15u ? 0xFFFFFFFFu : lo;
    }
}

template <typename T>
void widen(const T* in, uint32_t* out, uint64_t count) {
    const uint32_t sentinel = (uint32_t)(T)~0u;
    const int threads = std::max(1, std::min(16, omp_get_max_threads()));
#pragma omp parallel for num_threads(threads) schedule(static) if (count >= (1u << 16))
    for (int64_t i = 0; i < (int64_t)count; ++i) {
        const uint32_t v = in[i];
        out[i] = v == sentinel ? 0xFFFFFFFFu : v;
    }
}

template <typename T>
bool packedCopy(gb_bfs* h, const uint32_t* d, uint64_t count, uint32_t* out) {
    cudaStream_t st = h->stream.s;
    h->packDev.ensure(count * sizeof(T));
    h->packHost.ensure(count * sizeof(T));
    h->packFlag.ensure(1);
    h->packFlagHost.ensure(1);
    GB_CUDA(cudaMemsetAsync(h->packFlag.get(), 0, 4, st));
    T* dp = reinterpret_cast<T*>(h->packDev.get());
    T* hp = reinterpret_cast<T*>(h->packHost.p);
    packDepthsKernel<T><<<deviceSmCount() * 8, 256, 0, st>>>(d, count, dp, h->packFlag.get());
    GB_LAUNCH_CHECK();
    const uint64_t chunks = (count + kPackChunk - 1) / kPackChunk;
    while (h->packEv.size() < chunks) {
        cudaEvent_t e;
        GB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        h->packEv.push_back(e);
    }
    for (uint64_t c = 0; c < chunks; ++c) {
        const uint64_t lo = c * kPackChunk, len = std::min(kPackChunk, count - lo);
        GB_CUDA(cudaMemcpyAsync(hp + lo, dp + lo, len * sizeof(T), cudaMemcpyDeviceToHost, st));
        if (c + 1 == chunks)
            GB_CUDA(cudaMemcpyAsync(h->packFlagHost.p, h->packFlag.get(), 4, cudaMemcpyDeviceToHost, st));
        GB_CUDA(cudaEventRecord(h->packEv[c], st));
    }
    for (uint64_t c = 0; c < chunks; ++c) {
        const uint64_t lo = c * kPackChunk, len = std::min(kPackChunk, count - lo);
        GB_CUDA(cudaEventSynchronize(h->packEv[c]));
        widen(hp + lo, out + lo, len);
    }
    return *h->packFlagHost.p == 0;
}

bool packedCopy4(gb_bfs* h, const uint32_t* d, uint64_t count, uint32_t* out) {
    cudaStream_t st = h->stream.s;
    const uint64_t bytes = (count + 1) / 2;
    h->packDev.ensure(bytes);
    h->packHost.ensure(bytes);
    h->packFlag.ensure(1);
    h->packFlagHost.ensure(1);
    GB_CUDA(cudaMemsetAsync(h->packFlag.get(), 0, 4, st));
    uint8_t* dp = h->packDev.get();
    uint8_t* hp = h->packHost.p;
    packDepths4Kernel<<<deviceSmCount() * 8, 256, 0, st>>>(d, count, dp, h->packFlag.get());
    GB_LAUNCH_CHECK();
    const uint64_t chunks = (count + kPackChunk - 1) / kPackChunk;  // kPackChunk is even
    while (h->packEv.size() < chunks) {
        cudaEvent_t e;
        GB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        h->packEv.push_back(e);
    }
    for (uint64_t c = 0; c < chunks; ++c) {
        const uint64_t lo = c * kPackChunk, len = std::min(kPackChunk, count - lo);
        GB_CUDA(cudaMemcpyAsync(hp + lo / 2, dp + lo / 2, (len + 1) / 2, cudaMemcpyDeviceToHost, st));
        if (c + 1 == chunks)
            GB_CUDA(cudaMemcpyAsync(h->packFlagHost.p, h->packFlag.get(), 4, cudaMemcpyDeviceToHost, st));
        GB_CUDA(cudaEventRecord(h->packEv[c], st));
    }
    for (uint64_t c = 0; c < chunks; ++c) {
        const uint64_t lo = c * kPackChunk, len = std::min(kPackChunk, count - lo);
        GB_CUDA(cudaEventSynchronize(h->packEv[c]));
        widen4(hp + lo / 2, out + lo, len);
    }
    return *h->packFlagHost.p == 0;
}

}  // namespace

int packFormat(uint64_t count, uint32_t levels) {
    if (count < kPackMin) return -1;
    if (levels < 15) return 0;
    if (levels < 255) return 1;
    if (levels < 65535) return 2;
    return -1;
}

uint64_t packedBytes(int fmt, uint64_t count) {
    return fmt == 0 ? (count + 1) / 2 : fmt == 1 ? count : 2 * count;
}

void enqueuePack(int fmt, const uint32_t* d, uint64_t count, uint8_t* dev, unsigned* overflow, cudaStream_t st) {
    const int grid = deviceSmCount() * 8;
    if (fmt == 0) packDepths4Kernel<<<grid, 256, 0, st>>>(d, count, dev, overflow);
    else if (fmt == 1) packDepthsKernel<uint8_t><<<grid, 256, 0, st>>>(d, count, dev, overflow);
    else packDepthsKernel<uint16_t><<<grid, 256, 0, st>>>(d, count, reinterpret_cast<uint16_t*>(dev), overflow);
    GB_LAUNCH_CHECK();
}

void widenPacked(int fmt, const uint8_t* in, uint64_t count, uint32_t* out) {
    if (fmt == 0) widen4(in, out, count);
    else if (fmt == 1) widen(in, out, count);
    else widen(reinterpret_cast<const uint16_t*>(in), out, count);
}

void copyDepthsToHost(gb_bfs* h, const uint32_t* d, uint64_t count, uint32_t* out, uint32_t levels) {
    bool done = false;
    if (count >= kPackMin) {
        if (levels < 15) done = packedCopy4(h, d, count, out);
        else if (levels < 255) done = packedCopy<uint8_t>(h, d, count, out);
        else if (levels < 65535) done = packedCopy<uint16_t>(h, d, count, out);
    }
    if (!done) {
        GB_CUDA(cudaMemcpyAsync(out, d, count * 4, cudaMemcpyDeviceToHost, h->stream.s));
        GB_CUDA(cudaStreamSynchronize(h->stream.s));
    }
}

}  // namespace gb
