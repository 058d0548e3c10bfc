// loader.cu -- GGPUCSR1 .bin files into GPU memory (the reference's
// graph::load, src/graph/csr.cpp:54-84, which maps the file and lets the GPU
// read it in place through unified memory).  A discrete GPU cannot do that,
// so the ways in here keep the path from disk to HBM short:
//   gb_csr_load          read by several threads (pread of disjoint slices)
//                        straight into the returned arrays (gb_csr_save
//                        writes the same way);
//   gb_csr_load_pinned   the arrays land in page-locked host memory, read by
//                        several threads at once (pread of disjoint slices);
//                        every later upload of them runs at full PCIe speed.
//   gb_bfs_create_from_file  streams a symmetric graph straight into a BFS
//                        handle: the adjacency is read slice by slice into two
//                        pinned staging buffers in turn, each slice copied to
//                        the device while the next is read; no host copy of
//                        the whole graph is made.
// Files are checked as graph::load checks them (size against header), and the
// device copy is checked (row_ptr non-decreasing, ids below n) before any
// traversal can read it.
#include <fcntl.h>
#include <omp.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_set>

#include "bfs.hpp"
#include "capi_util.hpp"
#include "graph_prep.cuh"

namespace gb {
namespace {

constexpr char kBinMagic[8] = {'G', 'G', 'P', 'U', 'C', 'S', 'R', '1'};
constexpr uint64_t kStage = 64ull << 20;  // bytes per staged slice
constexpr uint64_t kSlice = 8ull << 20;   // bytes per reading thread and slice

std::mutex gPinnedMu;
std::unordered_set<void*> gPinned;  // arrays of gb_csr_load_pinned, released by gb_csr_free

struct BinFile {
    int fd = -1;
    uint64_t n = 0, m = 0;
    uint32_t flags = 0;
    std::string path;
    ~BinFile() {
        if (fd >= 0) close(fd);
    }
};

// Opens and checks a GGPUCSR1 file (src/graph/csr.cpp:54-73).
void openBin(const std::string& path, BinFile& b) {
    b.path = path;
    b.fd = open(path.c_str(), O_RDONLY);
    if (b.fd < 0) throw Error(GB_ERR_IO, "cannot open " + path);
    struct stat st;
    if (fstat(b.fd, &st) != 0) throw Error(GB_ERR_IO, "cannot stat " + path);
    const uint64_t len = (uint64_t)st.st_size;
    unsigned char hdr[32];
    if (len < sizeof hdr || pread(b.fd, hdr, sizeof hdr, 0) != (ssize_t)sizeof hdr) throw Error(GB_ERR_IO, path + ": too small");
    if (std::memcmp(hdr, kBinMagic, 8) != 0) throw Error(GB_ERR_IO, path + ": bad magic");
    uint32_t version;
    std::memcpy(&version, hdr + 8, 4);
    std::memcpy(&b.flags, hdr + 12, 4);
    std::memcpy(&b.n, hdr + 16, 8);
    std::memcpy(&b.m, hdr + 24, 8);
    if (version != 1) throw Error(GB_ERR_IO, path + ": unsupported version");
    if (b.n >= (1ull << 40) || b.m >= (1ull << 40) || 32 + 4 * (b.n + 1) + 4 * b.m != len)
        throw Error(GB_ERR_IO, path + ": size does not match header");
}

// Reads bytes at file offset off into dst with up to 8 threads, each taking
// whole kSlice slices.
void readParallel(const BinFile& b, void* dst, uint64_t bytes, uint64_t off) {
    const int64_t slices = (int64_t)((bytes + kSlice - 1) / kSlice);
    const int threads = (int)std::max<int64_t>(1, std::min<int64_t>({8, slices, omp_get_max_threads()}));
    bool failed = false;
#pragma omp parallel for num_threads(threads) schedule(dynamic, 1) reduction(|| : failed)
    for (int64_t s = 0; s < slices; ++s) {
        const uint64_t lo = (uint64_t)s * kSlice, len = std::min(kSlice, bytes - lo);
        uint64_t got = 0;
        while (got < len) {
            const ssize_t r = pread(b.fd, static_cast<char*>(dst) + lo + got, len - got, (off_t)(off + lo + got));
            if (r <= 0) {
                failed = true;
                break;
            }
            got += (uint64_t)r;
        }
    }
    if (failed) throw Error(GB_ERR_IO, b.path + ": short read");
}

// Writes bytes from src at file offset off with up to 8 threads (pwrite of
// kSlice slices).
bool writeParallel(int fd, const void* src, uint64_t bytes, uint64_t off) {
    const int64_t slices = (int64_t)((bytes + kSlice - 1) / kSlice);
    const int threads = (int)std::max<int64_t>(1, std::min<int64_t>({8, slices, omp_get_max_threads()}));
    bool failed = false;
#pragma omp parallel for num_threads(threads) schedule(dynamic, 1) reduction(|| : failed)
    for (int64_t s = 0; s < slices; ++s) {
        const uint64_t lo = (uint64_t)s * kSlice, len = std::min(kSlice, bytes - lo);
        uint64_t put = 0;
        while (put < len) {
            const ssize_t r = pwrite(fd, static_cast<const char*>(src) + lo + put, len - put, (off_t)(off + lo + put));
            if (r <= 0) {
                failed = true;
                break;
            }
            put += (uint64_t)r;
        }
    }
    return !failed;
}

}  // namespace

bool freePinnedArray(void* p) {
    if (!p) return false;
    {
        std::lock_guard<std::mutex> lk(gPinnedMu);
        if (!gPinned.erase(p)) return false;
    }
    cudaFreeHost(p);
    return true;
}

}  // namespace gb

using namespace gb;

extern "C" {

int gb_csr_load(const char* path, gb_csr* out) {
    return guard([&] {
        GB_REQUIRE(path && out, "null argument");
        BinFile b;
        openBin(path, b);
        uint32_t* rp = static_cast<uint32_t*>(std::malloc((b.n + 1) * 4));
        uint32_t* ci = static_cast<uint32_t*>(std::malloc(std::max<uint64_t>(b.m, 1) * 4));
        try {
            if (!rp || !ci) throw Error(GB_ERR_OOM, "host allocation failed");
            readParallel(b, rp, (b.n + 1) * 4, 32);  // straight into the caller's arrays
            if (b.m) readParallel(b, ci, b.m * 4, 32 + (b.n + 1) * 4);
        } catch (...) {
            std::free(rp);
            std::free(ci);
            throw;
        }
        out->n = b.n;
        out->m = b.m;
        out->flags = b.flags;
        out->row_ptr = rp;
        out->col_idx = ci;
    });
}

// graph::save (src/graph/csr.cpp:30-44): header then row_ptr then col_idx,
// written straight from the caller's arrays by several threads.
int gb_csr_save(const gb_csr* g, const char* path) {
    return guard([&] {
        GB_REQUIRE(path, "null path");
        GB_REQUIRE(g && g->row_ptr && (g->m == 0 || g->col_idx), "null graph");
        const std::string p = path;
        const int fd = open(path, O_WRONLY | O_CREAT | O_TRUNC, 0644);
        if (fd < 0) throw Error(GB_ERR_IO, "cannot write " + p);
        unsigned char hdr[32] = {};
        std::memcpy(hdr, kBinMagic, 8);
        const uint32_t version = 1;
        std::memcpy(hdr + 8, &version, 4);
        std::memcpy(hdr + 12, &g->flags, 4);
        std::memcpy(hdr + 16, &g->n, 8);
        std::memcpy(hdr + 24, &g->m, 8);
        bool ok = writeParallel(fd, hdr, sizeof hdr, 0) && writeParallel(fd, g->row_ptr, (g->n + 1) * 4, 32) &&
                  (g->m == 0 || writeParallel(fd, g->col_idx, g->m * 4, 32 + (g->n + 1) * 4));
        ok = (close(fd) == 0) && ok;
        if (!ok) throw Error(GB_ERR_IO, "short write to " + p);
    });
}

int gb_csr_load_pinned(const char* path, gb_csr* out) {
    return guard([&] {
        GB_REQUIRE(path && out, "null argument");
        BinFile b;
        openBin(path, b);
        void* rp = nullptr;
        void* ci = nullptr;
        GB_CUDA(cudaHostAlloc(&rp, (b.n + 1) * 4, cudaHostAllocDefault));
        if (cudaHostAlloc(&ci, std::max<uint64_t>(b.m, 1) * 4, cudaHostAllocDefault) != cudaSuccess) {
            cudaFreeHost(rp);
            cudaGetLastError();
            throw Error(GB_ERR_OOM, "gb_csr_load_pinned: page-locked allocation failed");
        }
        try {
            readParallel(b, rp, (b.n + 1) * 4, 32);
            if (b.m) readParallel(b, ci, b.m * 4, 32 + (b.n + 1) * 4);
        } catch (...) {
            cudaFreeHost(rp);
            cudaFreeHost(ci);
            throw;
        }
        {
            std::lock_guard<std::mutex> lk(gPinnedMu);
            gPinned.insert(rp);
            gPinned.insert(ci);
        }
        out->n = b.n;
        out->m = b.m;
        out->flags = b.flags;
        out->row_ptr = static_cast<uint32_t*>(rp);
        out->col_idx = static_cast<uint32_t*>(ci);
    });
}

int gb_bfs_create_from_file(const char* path, gb_bfs** out, uint64_t* n_out, uint64_t* m_out) {
    return guard([&] {
        GB_REQUIRE(path && out, "null argument");
        BinFile b;
        openBin(path, b);
        GB_REQUIRE(!(b.flags & 1u), "gb_bfs_create_from_file: the graph is directed; BFS runs on the symmetric "
                                    "graph (gb_csr_symmetrize_gpu, then gb_bfs_create)");
        GB_REQUIRE(b.n >= 1 && b.n < 0xFFFFFFFFull, "GpuBfs: graph too large for uint32 vertex ids");
        GB_REQUIRE(b.m < (1ull << 32), "m must fit in uint32");
        auto h = std::make_unique<gb_bfs>();
        h->n = b.n;
        h->m = b.m;
        h->flags = b.flags;
        h->hostRowPtr.resize(b.n + 1);
        readParallel(b, h->hostRowPtr.data(), (b.n + 1) * 4, 32);
        GB_REQUIRE(h->hostRowPtr[0] == 0 && h->hostRowPtr[b.n] == b.m, "row_ptr must start at 0 and end at m");
        h->rowPtr.ensure(b.n + 1);
        h->colIdx.ensure(b.m + 4);
        h->dist.ensure(b.n + 4);
        cudaStream_t st = h->stream.s;
        GB_CUDA(cudaMemcpyAsync(h->rowPtr.get(), h->hostRowPtr.data(), (b.n + 1) * 4, cudaMemcpyHostToDevice, st));
        if (b.m) {
            HostPinned<char> stage[2];
            stage[0].ensure(kStage);
            stage[1].ensure(kStage);
            cudaEvent_t ev[2];
            GB_CUDA(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
            if (cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming) != cudaSuccess) {
                cudaEventDestroy(ev[0]);
                throw Error(GB_ERR_CUDA, "cudaEventCreate failed");
            }
            struct EvGuard {
                cudaEvent_t* e;
                ~EvGuard() {
                    cudaEventDestroy(e[0]);
                    cudaEventDestroy(e[1]);
                }
            } eg{ev};
            const uint64_t bytes = b.m * 4, base = 32 + (b.n + 1) * 4;
            char* dst = reinterpret_cast<char*>(h->colIdx.get());
            for (uint64_t off = 0, k = 0; off < bytes; off += kStage, ++k) {
                const int s = (int)(k & 1);
                const uint64_t len = std::min(kStage, bytes - off);
                if (k >= 2) GB_CUDA(cudaEventSynchronize(ev[s]));  // this buffer's previous copy is done
                readParallel(b, stage[s].p, len, base + off);
                GB_CUDA(cudaMemcpyAsync(dst + off, stage[s].p, len, cudaMemcpyHostToDevice, st));
                GB_CUDA(cudaEventRecord(ev[s], st));
            }
            GB_CUDA(cudaStreamSynchronize(st));
        }
        checkDeviceCsr(h->rowPtr.get(), h->colIdx.get(), b.n, b.m, st);
        h->stats.ensure(1);
        h->hstats.ensure(1);
        h->hstage.ensure(16);
        GB_CUDA(cudaStreamSynchronize(st));
        if (n_out) *n_out = b.n;
        if (m_out) *m_out = b.m;
        *out = h.release();
    });
}

}  // extern "C"
