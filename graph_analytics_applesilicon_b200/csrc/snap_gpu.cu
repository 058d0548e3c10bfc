// snap_gpu.cu -- SNAP edge-list text (plain or gzip) -> CSR with the parsing,
// relabelling and compaction on the GPU: the reference's graph::convertSnap
// (src/graph/snap.cpp:85-149) and its line reader forEachEdge (:17-81).
//
// The host only moves bytes: it reads (or inflates) the file into two pinned
// staging buffers in turn, cuts each chunk at its last newline (the partial
// line is carried into the next chunk) and copies the chunk to the device
// while it reads the next one.  Per chunk the device
//   1. counts the newlines of each 16 KiB tile and scans the counts,
//   2. writes the position of every newline in file order (nlPos),
//   3. parses one line per thread with the reference's rules and appends the
//      (raw u, raw v) pairs of edge lines; errors record min(line << 2 | kind),
//      so the first failing line in file order wins as in the reference,
//      which stops at the first error.
// After the last chunk: a bitmap of the raw ids that occur, a scan of its
// per-word popcounts (dense id = rank among the occurring raw ids, i.e. the
// reference's relabelling in increasing raw-id order), one 64-bit key
// (dense u << b | dense v, both directions when undirected) per entry, and
// the key sort + unique + self-loop drop of graph_prep.cu, which yields the
// reference's compactAdjacency output exactly.
#include <omp.h>
#include <sys/stat.h>
#include <unistd.h>
#include <zlib.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>

#include "bfs_device.cuh"
#include "capi_util.hpp"
#include "graph_prep.cuh"

namespace gb {
namespace {

constexpr uint32_t kLongLine = 4u << 20;  // a line this long (before '\n') is an error
constexpr uint64_t kDefaultChunk = 64ull << 20;
constexpr uint64_t kMinChunk = (uint64_t)kLongLine + 1;  // holds any legal line and its newline
constexpr int kTileThreads = 256;
constexpr int kVecPerThread = 4;                                 // 16-byte vectors per thread
constexpr uint32_t kTileBytes = kTileThreads * kVecPerThread * 16;  // 16 KiB
constexpr unsigned long long kNoError = ~0ull;
enum : uint32_t { kErrLong = 0, kErrMalformed = 1, kErrTooLarge = 2 };

struct ChunkCounters {
    unsigned long long edges;  // edge lines appended so far (all chunks)
    unsigned long long err;    // min over failing lines of (line << 2 | kind)
    uint32_t lines;            // newlines in the current chunk
    uint32_t maxId;            // largest raw id seen so far
};

// Bit j of the result is set when byte j of the 16-byte vector at txt + off
// (bytes at or past len excluded) is '\n'.
__device__ __forceinline__ uint32_t newlineMask(const uint8_t* txt, uint32_t off, uint32_t len) {
    uint32_t mask = 0;
    if (off + 16 <= len) {
        const uint4 q = *reinterpret_cast<const uint4*>(txt + off);
        const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t eq = __vcmpeq4(w[k], 0x0A0A0A0Au);  // 0xFF in each matching byte
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if ((eq >> (8 * j)) & 1u) mask |= 1u << (4 * k + j);
        }
    } else {
        for (uint32_t j = 0; off + j < len && j < 16; ++j)
            if (txt[off + j] == '\n') mask |= 1u << j;
    }
    return mask;
}

// Byte offset of vector r (round) of thread t in tile `tile`: each round
// reads 256 consecutive vectors, so the loads of a warp are contiguous.
__device__ __forceinline__ uint32_t vecOffset(uint32_t tile, int r, unsigned t) {
    return tile * kTileBytes + ((uint32_t)r * kTileThreads + t) * 16u;
}

__global__ void __launch_bounds__(kTileThreads) nlCountKernel(const uint8_t* txt, uint32_t len, uint32_t* tileCnt) {
    __shared__ uint32_t sm[kTileThreads / 32 + 1];
    uint32_t c = 0;
#pragma unroll
    for (int r = 0; r < kVecPerThread; ++r) {
        const uint32_t off = vecOffset(blockIdx.x, r, threadIdx.x);
        if (off < len) c += __popc(newlineMask(txt, off, len));
    }
    uint32_t total;
    blockScan<kTileThreads>(c, &total, sm);
    if (threadIdx.x == 0) tileCnt[blockIdx.x] = total;
}

// nlPos[k] = offset of the k-th newline of the chunk (file order).
__global__ void __launch_bounds__(kTileThreads) nlPosKernel(const uint8_t* txt, uint32_t len, const uint32_t* tileBase,
                                                            uint32_t* nlPos) {
    __shared__ uint32_t sm[kTileThreads / 32 + 1];
    uint32_t run = tileBase[blockIdx.x];
#pragma unroll
    for (int r = 0; r < kVecPerThread; ++r) {
        const uint32_t off = vecOffset(blockIdx.x, r, threadIdx.x);
        uint32_t mask = off < len ? newlineMask(txt, off, len) : 0u;
        uint32_t total;
        uint32_t pos = run + blockScan<kTileThreads>(__popc(mask), &total, sm);
        while (mask) {
            const int j = __ffs(mask) - 1;
            nlPos[pos++] = off + (uint32_t)j;
            mask &= mask - 1u;
        }
        run += total;
    }
}

__device__ __forceinline__ bool isBlank(uint8_t c) { return c == ' ' || c == '\t'; }
__device__ __forceinline__ bool isDigit(uint8_t c) { return c >= '0' && c <= '9'; }

// One line per lane: txt[start, end) with txt[end] == '\n'.  The rules of
// forEachEdge (src/graph/snap.cpp:45-75): skip ' ', '\t', '\r'; an empty rest
// or '#' / '%' is not an edge; then two ids, each after optional ' ' / '\t',
// each a run of decimal digits accumulated modulo 2^64 and rejected when
// >= 0xFFFFFFFF; whatever follows the second id is ignored.
__global__ void __launch_bounds__(256) parseLinesKernel(const uint8_t* txt, const uint32_t* nlPos,
                                                        unsigned long long lineBase, uint32_t* eu, uint32_t* ev,
                                                        ChunkCounters* cnt) {
    const uint32_t lines = cnt->lines;
    const unsigned lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t w0 = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); w0 < lines; w0 += stride) {
        const uint64_t i = w0 + lane;
        bool edge = false;
        uint32_t ids[2] = {0, 0};
        uint32_t errKind = 0xFFFFFFFFu;
        if (i < lines) {
            uint32_t p = i ? nlPos[i - 1] + 1 : 0u;
            const uint32_t end = nlPos[i];
            if (end - p >= kLongLine) {
                errKind = kErrLong;
            } else {
                while (p < end && (isBlank(txt[p]) || txt[p] == '\r')) ++p;
                if (p < end && txt[p] != '#' && txt[p] != '%') {
                    edge = true;
                    for (int k = 0; k < 2 && edge; ++k) {
                        while (p < end && isBlank(txt[p])) ++p;
                        if (p == end || !isDigit(txt[p])) {
                            errKind = kErrMalformed;
                            edge = false;
                            break;
                        }
                        unsigned long long x = 0;
                        while (p < end && isDigit(txt[p])) x = x * 10ull + (unsigned long long)(txt[p++] - '0');
                        if (x >= 0xFFFFFFFFull) {
                            errKind = kErrTooLarge;
                            edge = false;
                            break;
                        }
                        ids[k] = (uint32_t)x;
                    }
                }
            }
            if (errKind != 0xFFFFFFFFu) atomicMin(&cnt->err, ((lineBase + i + 1) << 2) | errKind);
        }
        const unsigned ballot = __ballot_sync(kFull, edge);
        if (!ballot) continue;
        unsigned long long base = 0;
        const uint32_t mx = __reduce_max_sync(kFull, edge ? max(ids[0], ids[1]) : 0u);
        if (lane == 0) {
            base = atomicAdd(&cnt->edges, (unsigned long long)__popc(ballot));
            atomicMax(&cnt->maxId, mx);
        }
        base = __shfl_sync(kFull, base, 0);
        if (edge) {
            const unsigned long long at = base + __popc(ballot & ((1u << lane) - 1u));
            eu[at] = ids[0];
            ev[at] = ids[1];
        }
    }
}

__global__ void markIdsKernel(const uint32_t* eu, const uint32_t* ev, uint64_t ne, uint32_t* seen) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ne; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t a = eu[i], b = ev[i];
        atomicOr(&seen[a >> 5], 1u << (a & 31));
        atomicOr(&seen[b >> 5], 1u << (b & 31));
    }
}

__global__ void wordPopcKernel(const uint32_t* seen, uint64_t words, uint32_t* cnt) {
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < words; w += (uint64_t)gridDim.x * blockDim.x)
        cnt[w] = __popc(seen[w]);
}

__device__ __forceinline__ unsigned long long denseId(const uint32_t* seen, const uint32_t* wordBase, uint32_t x) {
    return wordBase[x >> 5] + __popc(seen[x >> 5] & ((1u << (x & 31)) - 1u));
}

__global__ void snapKeysKernel(const uint32_t* eu, const uint32_t* ev, uint64_t ne, const uint32_t* seen,
                               const uint32_t* wordBase, int b, bool both, unsigned long long* keys) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ne; i += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned long long u = denseId(seen, wordBase, eu[i]), v = denseId(seen, wordBase, ev[i]);
        keys[i] = (u << b) | v;
        if (both) keys[ne + i] = (v << b) | u;
    }
}

// Plain text of a regular file by several threads at once (pread of 8 MiB
// slices), other plain input through stdio, gzip through zlib (what gzread
// does for all three).
class TextSource {
public:
    explicit TextSource(const std::string& path) : path_(path) {
        FILE* f = std::fopen(path.c_str(), "rb");
        if (!f) throw Error(GB_ERR_IO, "cannot open " + path);
        unsigned char magic[2] = {0, 0};
        const size_t got = std::fread(magic, 1, 2, f);
        if (got == 2 && magic[0] == 0x1f && magic[1] == 0x8b) {
            std::fclose(f);
            gz_ = gzopen(path.c_str(), "rb");
            if (!gz_) throw Error(GB_ERR_IO, "cannot open " + path);
            gzbuffer(gz_, 1 << 20);
            return;
        }
        std::rewind(f);
        struct stat st;
        if (fstat(fileno(f), &st) == 0 && S_ISREG(st.st_mode)) {
            fd_ = dup(fileno(f));
            size_ = (uint64_t)st.st_size;
        }
        if (fd_ >= 0) std::fclose(f);
        else file_ = f;
    }
    ~TextSource() {
        if (gz_) gzclose(gz_);
        if (file_) std::fclose(file_);
        if (fd_ >= 0) close(fd_);
    }
    // Fills dst with up to want bytes; fewer only at the end of the data.
    uint64_t read(char* dst, uint64_t want) {
        if (fd_ >= 0) return readParallel(dst, want);
        uint64_t have = 0;
        while (have < want) {
            const uint64_t ask = std::min<uint64_t>(want - have, 1u << 30);
            if (gz_) {
                const int got = gzread(gz_, dst + have, (unsigned)ask);
                if (got < 0) throw Error(GB_ERR_IO, "gzread failed on " + path_);
                if (got == 0) break;
                have += (uint64_t)got;
            } else {
                const size_t got = std::fread(dst + have, 1, ask, file_);
                if (got == 0) {
                    if (std::ferror(file_)) throw Error(GB_ERR_IO, "read failed on " + path_);
                    break;
                }
                have += got;
            }
        }
        return have;
    }

private:
    uint64_t readParallel(char* dst, uint64_t want) {
        constexpr uint64_t kSlice = 8ull << 20;
        const uint64_t bytes = std::min(want, size_ - std::min(size_, off_));
        const int64_t slices = (int64_t)((bytes + kSlice - 1) / kSlice);
        const int threads = (int)std::max<int64_t>(1, std::min<int64_t>({8, slices, omp_get_max_threads()}));
        bool failed = false;
#pragma omp parallel for num_threads(threads) schedule(dynamic, 1) reduction(|| : failed)
        for (int64_t sl = 0; sl < slices; ++sl) {
            const uint64_t lo = (uint64_t)sl * kSlice, len = std::min(kSlice, bytes - lo);
            uint64_t got = 0;
            while (got < len) {
                const ssize_t r = pread(fd_, dst + lo + got, len - got, (off_t)(off_ + lo + got));
                if (r <= 0) {
                    failed = true;
                    break;
                }
                got += (uint64_t)r;
            }
        }
        if (failed) throw Error(GB_ERR_IO, "read failed on " + path_);
        off_ += bytes;
        return bytes;
    }

    std::string path_;
    gzFile gz_ = nullptr;
    FILE* file_ = nullptr;
    int fd_ = -1;
    uint64_t size_ = 0, off_ = 0;
};

// Device array that keeps its contents when it grows.
void growKeep(DevBuf<uint32_t>& a, uint64_t used, uint64_t need, cudaStream_t st) {
    if (a.n >= need && a.p) return;
    DevBuf<uint32_t> b;
    b.ensure(std::max<uint64_t>(need, 2 * (uint64_t)a.n));
    if (used) GB_CUDA(cudaMemcpyAsync(b.p, a.p, used * 4, cudaMemcpyDeviceToDevice, st));
    GB_CUDA(cudaStreamSynchronize(st));
    std::swap(a.p, b.p);
    std::swap(a.n, b.n);
}

std::string errorText(const std::string& path, unsigned long long key) {
    const unsigned long long line = key >> 2;
    switch ((uint32_t)(key & 3u)) {
        case kErrLong: return "line longer than 4 MB in " + path;
        case kErrMalformed: return path + ": malformed line " + std::to_string(line);
        default: return path + ": vertex ID too large on line " + std::to_string(line);
    }
}

void snapToCsr(const std::string& path, bool directed, uint64_t chunk, gb_csr* out, gb_convert_stats* stats) {
    const auto t0 = std::chrono::steady_clock::now();
    if (chunk == 0) chunk = kDefaultChunk;
    GB_REQUIRE(chunk >= kMinChunk && chunk < (1ull << 32) - 64, "snap: chunk_bytes must be in [4 MiB + 1, 4 GiB)");
    TextSource src(path);
    Stream st;
    ScanScratch sc;
    HostPinned<char> stage[2];
    stage[0].ensure(chunk + 1);
    stage[1].ensure(chunk + 1);
    HostPinned<ChunkCounters> hc;
    hc.ensure(1);
    const uint32_t maxTiles = (uint32_t)((chunk + 1 + kTileBytes - 1) / kTileBytes);
    DevBuf<uint8_t> txt;
    DevBuf<uint32_t> nlPos, tileCnt, eu, ev;
    DevBuf<ChunkCounters> cnt;
    txt.ensure(chunk + 64);
    nlPos.ensure(chunk + 1);
    tileCnt.ensure(maxTiles + 1);
    cnt.ensure(1);
    ChunkCounters init{0ull, kNoError, 0u, 0u};
    GB_CUDA(cudaMemcpyAsync(cnt.get(), &init, sizeof init, cudaMemcpyHostToDevice, st.s));
    cudaEvent_t done;
    GB_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
    struct EventGuard {
        cudaEvent_t e;
        ~EventGuard() { cudaEventDestroy(e); }
    } eg{done};
    const uint32_t parseGrid = (uint32_t)deviceSmCount() * 8;

    unsigned long long lineBase = 0, edges = 0;
    uint32_t maxId = 0;
    uint64_t have = 0;  // carried bytes at the start of stage[cur]
    int cur = 0;
    bool eof = false, inFlight = false;
    std::string error;
    // Waits for the chunk in flight; folds its counters into the totals.
    auto finish = [&]() {
        GB_CUDA(cudaEventSynchronize(done));
        inFlight = false;
        const ChunkCounters c = *hc.p;
        if (c.err != kNoError) {
            error = errorText(path, c.err);
            return;
        }
        lineBase += c.lines;
        edges = c.edges;
        maxId = c.maxId;
    };
    while (!eof && error.empty()) {
        char* buf = stage[cur].p;
        uint64_t got = 0;
        try {
            got = src.read(buf + have, chunk - have);
        } catch (...) {
            if (inFlight) finish();  // an error on an earlier line is reported first
            if (!error.empty()) break;
            throw;
        }
        eof = got == 0;
        uint64_t len = have + got;
        if (eof && len > 0 && buf[len - 1] != '\n') buf[len++] = '\n';  // last line without newline
        uint64_t end = len;
        while (end > 0 && buf[end - 1] != '\n') --end;
        if (inFlight) finish();  // the previous chunk's errors come first in file order
        if (!error.empty()) break;
        if (end == 0) {
            if (len == chunk) error = "line longer than 4 MB in " + path;  // no newline in a full buffer
            have = len;  // else the data ended inside this line: the next read sees eof
            continue;
        }
        // room for this chunk's edges: an edge line has at least 4 bytes
        growKeep(eu, edges, edges + end / 4 + 1, st.s);
        growKeep(ev, edges, edges + end / 4 + 1, st.s);
        const uint32_t L = (uint32_t)end, tiles = (L + kTileBytes - 1) / kTileBytes;
        GB_CUDA(cudaMemcpyAsync(txt.get(), buf, L, cudaMemcpyHostToDevice, st.s));
        nlCountKernel<<<tiles, kTileThreads, 0, st.s>>>(txt.get(), L, tileCnt.get());
        GB_LAUNCH_CHECK();
        scanExclusive(tileCnt.get(), tileCnt.get(), tiles, &cnt.get()->lines, sc, st.s);
        nlPosKernel<<<tiles, kTileThreads, 0, st.s>>>(txt.get(), L, tileCnt.get(), nlPos.get());
        GB_LAUNCH_CHECK();
        parseLinesKernel<<<parseGrid, 256, 0, st.s>>>(txt.get(), nlPos.get(), lineBase, eu.get(), ev.get(), cnt.get());
        GB_LAUNCH_CHECK();
        GB_CUDA(cudaMemcpyAsync(hc.p, cnt.get(), sizeof(ChunkCounters), cudaMemcpyDeviceToHost, st.s));
        GB_CUDA(cudaEventRecord(done, st.s));
        inFlight = true;
        // the partial last line opens the other stage buffer, whose previous
        // chunk has finished copying (finish() above waited for it)
        const int nxt = cur ^ 1;
        have = len - end;
        if (have) std::memcpy(stage[nxt].p, buf + end, have);
        cur = nxt;
    }
    if (inFlight) finish();
    if (!error.empty()) {
        const bool io = error.rfind("cannot open", 0) == 0;
        throw Error(io ? GB_ERR_IO : GB_ERR_ARG, error);
    }
    const uint64_t total = directed ? edges : 2 * edges;
    if (total >= 0xFFFFFFFFull) throw Error(GB_ERR_ARG, "too many edges for uint32 offsets");

    uint64_t n = 0;
    DevBuf<unsigned long long> keys, tmp;
    int b = 1;
    if (edges) {
        const uint64_t words = (uint64_t)maxId / 32 + 1;
        DevBuf<uint32_t> seen, wcnt;
        DevBuf<uint32_t> nDev;
        seen.ensure(words);
        wcnt.ensure(words + 1);
        nDev.ensure(1);
        GB_CUDA(cudaMemsetAsync(seen.get(), 0, words * 4, st.s));
        markIdsKernel<<<prepGrid(edges, 256), 256, 0, st.s>>>(eu.get(), ev.get(), edges, seen.get());
        GB_LAUNCH_CHECK();
        wordPopcKernel<<<prepGrid(words, 256), 256, 0, st.s>>>(seen.get(), words, wcnt.get());
        GB_LAUNCH_CHECK();
        scanExclusive(wcnt.get(), wcnt.get(), words, nDev.get(), sc, st.s);
        uint32_t hn = 0;
        GB_CUDA(cudaMemcpyAsync(&hn, nDev.get(), 4, cudaMemcpyDeviceToHost, st.s));
        GB_CUDA(cudaStreamSynchronize(st.s));
        n = hn;
        b = keyBits(n);
        keys.ensure(total + 1);
        snapKeysKernel<<<prepGrid(edges, 256), 256, 0, st.s>>>(eu.get(), ev.get(), edges, seen.get(), wcnt.get(), b,
                                                               !directed, keys.get());
        GB_LAUNCH_CHECK();
        eu.release();
        ev.release();
        radixSortKeys(keys, tmp, total, 2 * b, sc, st.s);
    }
    constexpr uint32_t kFlagDirected = 1u, kFlagSorted = 2u, kFlagDedup = 4u;
    keysToCsr(keys, total, n, b, true, true, (directed ? kFlagDirected : 0u) | kFlagSorted | kFlagDedup, sc, st.s,
              out);
    if (stats) {
        stats->lines = edges;
        stats->raw_max_id = edges ? maxId : 0;
        stats->n = n;
        stats->m_before = total;
        stats->m = out->m;
        stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
}

}  // namespace
}  // namespace gb

using namespace gb;

extern "C" {

int gb_csr_from_snap_gpu(const char* path, int directed, uint64_t chunk_bytes, gb_csr* out,
                         gb_convert_stats* stats) {
    return guard([&] {
        GB_REQUIRE(path && out, "null argument");
        snapToCsr(path, directed != 0, chunk_bytes, out, stats);
    });
}

int gb_convert_snap_gpu(const char* in_path, const char* out_path, int directed, gb_convert_stats* stats) {
    return guard([&] {
        GB_REQUIRE(in_path && out_path, "null argument");
        const auto t0 = std::chrono::steady_clock::now();
        gb_csr g{};
        snapToCsr(in_path, directed != 0, 0, &g, stats);
        const int rc = gb_csr_save(&g, out_path);
        gb_csr_free(&g);
        if (rc != GB_OK) throw Error((gb_status)rc, gb_last_error());
        if (stats) stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    });
}

}  // extern "C"
