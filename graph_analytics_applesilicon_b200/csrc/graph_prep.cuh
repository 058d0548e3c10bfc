// graph_prep.cuh -- the key-sort pipeline of graph_prep.cu, shared with the
// SNAP edge-list converter (snap_gpu.cu): 64-bit (row << b | column) keys,
// stable LSD radix sort, then keys -> CSR.
#pragma once

#include "graph_b200.h"
#include "prims.cuh"

namespace gb {

// Blocks for a grid-stride loop over `work` items (at most 16 per SM).
uint32_t prepGrid(uint64_t work, uint32_t threads);
// Bits of the largest id below n (at least 1): the column field of a key.
int keyBits(uint64_t n);
// Sorts N keys whose used bits are [0, bits) in place (a holds the result;
// tmp is scratch of N keys).  N < 2^32.
// countsScratch (optional) is reused for the digit histograms across calls.
void radixSortKeys(DevBuf<unsigned long long>& a, DevBuf<unsigned long long>& tmp, uint64_t N, int bits,
                   ScanScratch& sc, cudaStream_t st, DevBuf<uint32_t>* countsScratch = nullptr);
// Sorted keys -> host CSR in *out (n rows, b column bits), dropping repeated
// keys (unique) and self-loops (dropSelf); out->flags = flags.
void keysToCsr(DevBuf<unsigned long long>& keys, uint64_t N, uint64_t n, int b, bool unique, bool dropSelf,
               uint32_t flags, ScanScratch& sc, cudaStream_t st, gb_csr* out);

// Uploads a host CSR and checks it on the device (row_ptr from 0 to m and
// non-decreasing, every column below n); throws GB_ERR_ARG otherwise.
void uploadCheckedCsr(const gb_csr* g, DevBuf<uint32_t>& rp, DevBuf<uint32_t>& ci, cudaStream_t st);
// Checks a device CSR (row_ptr non-decreasing, every column below n); throws
// GB_ERR_ARG otherwise.
void checkDeviceCsr(const uint32_t* rp, const uint32_t* ci, uint64_t n, uint64_t m, cudaStream_t st);
// Connected components of a symmetric device CSR: parent[v] = the smallest
// vertex of v's component.
void connectedComponents(const uint32_t* rp, const uint32_t* ci, uint64_t n, uint32_t* parent, cudaStream_t st);

// Re-sorts every adjacency list of a device CSR (in place) by descending
// neighbour degree, ties by id; row_ptr is unchanged.
void hubFirstAdjacency(const uint32_t* rp, uint32_t* ci, uint64_t n, uint64_t m, cudaStream_t st);

}  // namespace gb
