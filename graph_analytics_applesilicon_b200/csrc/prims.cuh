// prims.cuh -- device-wide primitives on uint32 arrays (the role of the
// reference's src/metal/primitives.{hpp,mm} + src/shaders/primitives.metal).
#pragma once

#include "common.cuh"

namespace gb {

// Scratch the single-pass scan needs; owned by the caller (a handle), reused.
struct ScanScratch {
    DevBuf<unsigned long long> status;  // per-tile (flag << 32 | value)
    DevBuf<unsigned> counters;          // [0] tile ticket, [1] error flag
};

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

// out[i] = in[0] + ... + in[i-1] (mod 2^32); in == out allowed.  If total is
// non-null, *total (device) = sum of all n inputs.  Single pass with
// decoupled look-back; its waits are bounded and set counters[1] on timeout.
void scanExclusive(const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* total, ScanScratch& s,
                   cudaStream_t st);
// *sum / *max (device, may be null) of in[0..n); both must be zeroed by the caller.
void reduceSumMax(const uint32_t* in, uint64_t n, uint32_t* sum, uint32_t* max, cudaStream_t st);
// Zero the bitmap (ceil(n/32) words) then set the bit of each queue entry.
void queueToBitmap(const uint32_t* queue, uint64_t size, uint32_t* bitmap, uint64_t n, cudaStream_t st);
// Append every set vertex v < n to queue (unordered); *count (device, zeroed
// by the caller) = number appended; if row_ptr, deg[i] = degree(queue[i]).
void bitmapToQueue(const uint32_t* bitmap, uint64_t n, uint32_t* queue, uint32_t* count,
                   const uint32_t* row_ptr, uint32_t* deg, cudaStream_t st);
void fillU32(uint32_t* p, uint32_t value, uint64_t n, cudaStream_t st);

}  // namespace gb
