// l2_rates.cu -- the L2 staging rates the blocked PageRank pull is measured against:
//  * TMA bulk copies (cp.async.bulk) of S bytes from an L2-resident 12 MiB array
//    into a ring of D shared-memory stages, one producer thread per block;
//  * 16-byte loads by every thread (ld.global.cg) of the same array.
// (Gather rates are measured on a graph's own in-lists by gather_bound.py.)
// Every wait is bounded (an error flag instead of a hang) and every index is
// reduced into its array.  Build and run on one GPU:
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -o l2_rates \
//       graph_analytics_applesilicon_b200/microbench/l2_rates.cu && ./l2_rates
#include <cstdio>
#include <cstdint>
#include <cuda_runtime.h>
#define CK(x) do { cudaError_t e = (x); if (e != cudaSuccess) { printf("CUDA %s at %d\n", cudaGetErrorString(e), __LINE__); return 1; } } while (0)
__device__ __forceinline__ uint32_t sa(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ bool waitPar(uint64_t* mb, uint32_t par, unsigned long long lim) {
    for (unsigned long long i = 0; i < lim; ++i) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done) : "r"(sa(mb)), "r"(par) : "memory");
        if (done) return true;
    }
    return false;
}
constexpr int MAXD = 8;
__global__ void tmaRing(const char* src, size_t nchunks, uint32_t S, int D, int K, int* err, float* sink) {
    extern __shared__ __align__(128) char buf[];
    __shared__ __align__(8) uint64_t full[MAXD], empty[MAXD];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (threadIdx.x == 0) {
        for (int s = 0; s < D; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sa(&full[s])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sa(&empty[s])), "r"(nw - 1) : "memory");
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const unsigned long long lim = 1ull << 24;
    if (warp == 0) {
        if (lane == 0) {
            for (int t = 0; t < K; ++t) {
                int s = t % D;
                if (!waitPar(&empty[s], ((t / D) & 1) ^ 1, lim)) { atomicOr(err, 1); break; }
                size_t c = ((size_t)blockIdx.x * 977 + t) % nchunks;
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sa(&full[s])), "r"(S) : "memory");
                asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                             ::"r"(sa(buf + (size_t)s * S)), "l"(src + c * S), "r"(S), "r"(sa(&full[s])) : "memory");
            }
            for (int s = 0; s < D && s < K; ++s) {
                int last = K - 1 - ((K - 1 - s) % D);
                waitPar(&full[s], (last / D) & 1, lim);
            }
        }
        __syncwarp();
    } else {
        float acc = 0;
        for (int t = 0; t < K; ++t) {
            int s = t % D;
            if (!waitPar(&full[s], (t / D) & 1, lim)) { atomicOr(err, 2); break; }
            acc += reinterpret_cast<const float*>(buf + (size_t)s * S)[lane + 32 * (warp - 1)];
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(sa(&empty[s])) : "memory");
        }
        if (acc == 12345.f) sink[0] = acc;
    }
}
__global__ void vecLoad(const uint4* src, size_t nchunks, uint32_t S, int K, float* sink) {
    float acc = 0;
    const uint32_t w = S / 16;
    for (int t = 0; t < K; ++t) {
        size_t c = ((size_t)blockIdx.x * 977 + t) % nchunks;
        const uint4* p = src + c * w;
        for (uint32_t i = threadIdx.x; i < w; i += blockDim.x) { uint4 v = __ldcg(p + i); acc += __uint_as_float(v.x ^ v.y ^ v.z ^ v.w); }
    }
    if (acc == 12345.f) sink[0] = acc;
}
int main() {
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0));
    const size_t nbytes = 12u << 20;
    char* src; float* sink; int* err;
    CK(cudaMalloc(&src, nbytes)); CK(cudaMemset(src, 1, nbytes)); CK(cudaMalloc(&sink, 64)); CK(cudaMalloc(&err, 4)); CK(cudaMemset(err, 0, 4));
    cudaEvent_t e0, e1; CK(cudaEventCreate(&e0)); CK(cudaEventCreate(&e1));
    CK(cudaFuncSetAttribute(tmaRing, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    printf("sms %d\n", sms);
    for (uint32_t S : {8192u, 16384u, 32768u, 49152u}) for (int D : {2, 3, 4, 6}) {
        if ((size_t)S * D > 200 * 1024) continue;
        for (int threads : {128, 1024}) {
            int K = (int)((256ull << 20) / S / sms); size_t nchunks = nbytes / S;
            tmaRing<<<sms, threads, S * D>>>(src, nchunks, S, D, K, err, sink); CK(cudaGetLastError());
            CK(cudaEventRecord(e0)); tmaRing<<<sms, threads, S * D>>>(src, nchunks, S, D, K, err, sink); CK(cudaEventRecord(e1));
            CK(cudaEventSynchronize(e1)); float ms; CK(cudaEventElapsedTime(&ms, e0, e1));
            double bytes = (double)K * S * sms; int herr; CK(cudaMemcpy(&herr, err, 4, cudaMemcpyDeviceToHost));
            printf("TMA S=%6u D=%d thr=%4d: %.3f ms, %.2f TB/s, %.1f GB/s/SM, %.3f us/copy%s\n", S, D, threads, ms, bytes / ms / 1e9, bytes / ms / 1e6 / sms, ms * 1e3 / K, herr ? " ERR" : "");
        }
    }
    for (int bps : {1, 2}) for (uint32_t S : {16384u, 65536u}) {
        int K = (int)((256ull << 20) / S / (sms * bps)); size_t nchunks = nbytes / S;
        vecLoad<<<sms * bps, 1024 / bps>>>((const uint4*)src, nchunks, S, K, sink);
        CK(cudaEventRecord(e0)); vecLoad<<<sms * bps, 1024 / bps>>>((const uint4*)src, nchunks, S, K, sink); CK(cudaEventRecord(e1));
        CK(cudaEventSynchronize(e1)); float ms; CK(cudaEventElapsedTime(&ms, e0, e1));
        printf("LDG.128 S=%6u blocks/SM=%d: %.3f ms, %.2f TB/s\n", S, bps, ms, (double)K * S * sms * bps / ms / 1e9);
    }
    int herr; CK(cudaMemcpy(&herr, err, 4, cudaMemcpyDeviceToHost)); printf("err %d\n", herr);
    return 0;
}
