// selector_train.cu -- training kernels of the learned BFS strategy selector.
//
// Model (selector.cuh): out = W3 relu(W2 relu(W1 x + b1) + b2) + b3 with 8
// features, 32 hidden units, one output per strategy (predicted log2 of the
// level's time in microseconds).  Loss: mean squared error over the measured
// (masked) entries.  One warp per sample: lane j owns hidden unit j in the
// forward and backward passes; gradients are accumulated per block in shared
// memory and added to global memory once per block.  Adam updates on the GPU.
// No counterpart in the reference; the CPU check is orc_mlp_loss_grad in the
// test oracle.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#include "capi_util.hpp"
#include "selector.cuh"

namespace gb {
namespace {

constexpr int F = kSelFeatures, H = kSelHidden, O = kSelOutputs, NP = kSelParams;
constexpr int OFF_W1 = 0, OFF_B1 = H * F, OFF_W2 = OFF_B1 + H, OFF_B2 = OFF_W2 + H * H, OFF_W3 = OFF_B2 + H,
              OFF_B3 = OFF_W3 + O * H;

// Per-warp forward of one sample; returns h1, h2 (lane = unit) and out (lane < O).
__device__ __forceinline__ void forward(const float* P, const float* x, unsigned lane, float& h1, float& h2,
                                        float& out) {
    h1 = P[OFF_B1 + lane];
#pragma unroll
    for (int f = 0; f < F; ++f) h1 = fmaf(P[OFF_W1 + lane * F + f], x[f], h1);
    h1 = fmaxf(h1, 0.f);
    h2 = P[OFF_B2 + lane];
#pragma unroll
    for (int k = 0; k < H; ++k) h2 = fmaf(P[OFF_W2 + lane * H + k], __shfl_sync(kFull, h1, k), h2);
    h2 = fmaxf(h2, 0.f);
    const unsigned o = lane < O ? lane : 0;
    out = P[OFF_B3 + o];
#pragma unroll
    for (int k = 0; k < H; ++k) out = fmaf(P[OFF_W3 + o * H + k], __shfl_sync(kFull, h2, k), out);
}

// Gradient (unscaled: d/dout = 2 mask (out - y)) accumulated into g (global),
// plus sum(mask * err^2) and sum(mask) into acc[0], acc[1].  rows selects the
// samples (idx[i] for i < count; idx null = identity).
__global__ void lossGradKernel(const float* __restrict__ P, const float* __restrict__ X, const float* __restrict__ Y,
                               const float* __restrict__ M, const int* __restrict__ idx, int count, float* g,
                               double* acc) {
    __shared__ float sP[NP];
    __shared__ float sG[NP];
    __shared__ double sAcc[2];
    for (int i = threadIdx.x; i < NP; i += blockDim.x) {
        sP[i] = P[i];
        sG[i] = 0.f;
    }
    if (threadIdx.x < 2) sAcc[threadIdx.x] = 0;
    __syncthreads();
    const unsigned lane = laneId();
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < count; i += warpsPerGrid) {
        const int row = idx ? idx[i] : i;
        float x[F];
#pragma unroll
        for (int f = 0; f < F; ++f) x[f] = X[(size_t)row * F + f];
        float h1, h2, out;
        forward(sP, x, lane, h1, h2, out);
        float dout = 0.f;
        if (lane < O) {
            const float mk = M[(size_t)row * O + lane];
            const float e = out - Y[(size_t)row * O + lane];
            dout = 2.f * mk * e;
            atomicAdd(&sAcc[0], (double)(mk * e * e));
            atomicAdd(&sAcc[1], (double)mk);
            atomicAdd(&sG[OFF_B3 + lane], dout);
        }
        // layer 3: gW3[o][k] += dout[o] h2[k]; dh2[k] = sum_o dout[o] W3[o][k]
        float dh2 = 0.f;
#pragma unroll
        for (int o = 0; o < O; ++o) {
            const float d = __shfl_sync(kFull, dout, o);
            atomicAdd(&sG[OFF_W3 + o * H + lane], d * h2);
            dh2 = fmaf(d, sP[OFF_W3 + o * H + lane], dh2);
        }
        dh2 = h2 > 0.f ? dh2 : 0.f;
        atomicAdd(&sG[OFF_B2 + lane], dh2);
        // layer 2: gW2[j][k] += dh2[j] h1[k]; dh1[k] = sum_j dh2[j] W2[j][k]
        float dh1 = 0.f;
#pragma unroll 4
        for (int j = 0; j < H; ++j) {
            const float d = __shfl_sync(kFull, dh2, j);
            atomicAdd(&sG[OFF_W2 + j * H + lane], d * h1);
            dh1 = fmaf(d, sP[OFF_W2 + j * H + lane], dh1);
        }
        dh1 = h1 > 0.f ? dh1 : 0.f;
        atomicAdd(&sG[OFF_B1 + lane], dh1);
#pragma unroll
        for (int f = 0; f < F; ++f) atomicAdd(&sG[OFF_W1 + lane * F + f], dh1 * x[f]);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < NP; i += blockDim.x)
        if (sG[i] != 0.f) atomicAdd(&g[i], sG[i]);
    if (threadIdx.x < 2 && sAcc[threadIdx.x] != 0) atomicAdd(&acc[threadIdx.x], sAcc[threadIdx.x]);
}

__global__ void forwardKernel(const float* __restrict__ P, const float* __restrict__ X, int count, float* Out) {
    __shared__ float sP[NP];
    for (int i = threadIdx.x; i < NP; i += blockDim.x) sP[i] = P[i];
    __syncthreads();
    const unsigned lane = laneId();
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < count; i += warpsPerGrid) {
        float x[F];
#pragma unroll
        for (int f = 0; f < F; ++f) x[f] = X[(size_t)i * F + f];
        float h1, h2, out;
        forward(sP, x, lane, h1, h2, out);
        if (lane < O) Out[(size_t)i * O + lane] = out;
    }
}

// g /= max(1, mask sum) (the mean), then one Adam step (bias-corrected).
__global__ void adamKernel(float* P, float* g, float* m, float* v, const double* acc, float lr, float b1t, float b2t) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NP) return;
    const double ms = acc[1];
    const float scale = ms > 1.0 ? (float)(1.0 / ms) : 1.f;
    const float gi = g[i] * scale;
    const float b1 = 0.9f, b2 = 0.999f;
    m[i] = b1 * m[i] + (1 - b1) * gi;
    v[i] = b2 * v[i] + (1 - b2) * gi * gi;
    const float mh = m[i] / (1 - b1t), vh = v[i] / (1 - b2t);
    P[i] -= lr * mh / (sqrtf(vh) + 1e-8f);
    g[i] = 0.f;
}

uint32_t warpGrid(int count) {
    return (uint32_t)std::max(1, std::min((count + 7) / 8, deviceSmCount() * 4));
}

}  // namespace
}  // namespace gb

using namespace gb;

extern "C" {

int gb_mlp_loss_grad(const float* params, int batch, const float* x, const float* y, const float* mask,
                     float* grads_out, double* loss_out) {
    return guard([&] {
        GB_REQUIRE(params && grads_out && batch >= 0 && (batch == 0 || (x && y && mask)), "null argument");
        DevBuf<float> P, X, Y, M, Gr;
        DevBuf<double> acc;
        P.ensure(NP);
        Gr.ensure(NP);
        acc.ensure(2);
        X.ensure((size_t)batch * F + 1);
        Y.ensure((size_t)batch * O + 1);
        M.ensure((size_t)batch * O + 1);
        GB_CUDA(cudaMemcpy(P.get(), params, NP * 4, cudaMemcpyHostToDevice));
        if (batch) {
            GB_CUDA(cudaMemcpy(X.get(), x, (size_t)batch * F * 4, cudaMemcpyHostToDevice));
            GB_CUDA(cudaMemcpy(Y.get(), y, (size_t)batch * O * 4, cudaMemcpyHostToDevice));
            GB_CUDA(cudaMemcpy(M.get(), mask, (size_t)batch * O * 4, cudaMemcpyHostToDevice));
        }
        GB_CUDA(cudaMemset(Gr.get(), 0, NP * 4));
        GB_CUDA(cudaMemset(acc.get(), 0, 16));
        lossGradKernel<<<warpGrid(batch), 256>>>(P.get(), X.get(), Y.get(), M.get(), nullptr, batch, Gr.get(),
                                                 acc.get());
        GB_LAUNCH_CHECK();
        std::vector<float> g(NP);
        double a[2];
        GB_CUDA(cudaMemcpy(g.data(), Gr.get(), NP * 4, cudaMemcpyDeviceToHost));
        GB_CUDA(cudaMemcpy(a, acc.get(), 16, cudaMemcpyDeviceToHost));
        const double scale = a[1] > 1 ? 1.0 / a[1] : 1.0;
        for (int i = 0; i < NP; ++i) grads_out[i] = (float)(g[i] * scale);
        if (loss_out) *loss_out = a[0] * scale;
    });
}

int gb_mlp_forward(const float* params, int batch, const float* x, float* out) {
    return guard([&] {
        GB_REQUIRE(params && out && (batch == 0 || x), "null argument");
        if (batch == 0) return;
        DevBuf<float> P, X, Out;
        P.ensure(NP);
        X.ensure((size_t)batch * F);
        Out.ensure((size_t)batch * O);
        GB_CUDA(cudaMemcpy(P.get(), params, NP * 4, cudaMemcpyHostToDevice));
        GB_CUDA(cudaMemcpy(X.get(), x, (size_t)batch * F * 4, cudaMemcpyHostToDevice));
        forwardKernel<<<warpGrid(batch), 256>>>(P.get(), X.get(), batch, Out.get());
        GB_LAUNCH_CHECK();
        GB_CUDA(cudaMemcpy(out, Out.get(), (size_t)batch * O * 4, cudaMemcpyDeviceToHost));
    });
}

// Minibatch Adam on the GPU: every epoch a host-shuffled order of the rows is
// uploaded; each minibatch is one gradient kernel and one update kernel.
int gb_mlp_train(float* params_inout, int rows, const float* x, const float* y, const float* mask, int epochs,
                 int batch, float lr, uint64_t seed, float* final_loss) {
    return guard([&] {
        GB_REQUIRE(params_inout && rows > 0 && x && y && mask && epochs >= 0 && batch > 0, "bad training arguments");
        DevBuf<float> P, X, Y, M, Gr, Mo, Vo;
        DevBuf<double> acc;
        DevBuf<int> idx;
        P.ensure(NP);
        Gr.ensure(NP);
        Mo.ensure(NP);
        Vo.ensure(NP);
        acc.ensure(2);
        X.ensure((size_t)rows * F);
        Y.ensure((size_t)rows * O);
        M.ensure((size_t)rows * O);
        idx.ensure(rows);
        Stream st;
        GB_CUDA(cudaMemcpyAsync(P.get(), params_inout, NP * 4, cudaMemcpyHostToDevice, st.s));
        GB_CUDA(cudaMemcpyAsync(X.get(), x, (size_t)rows * F * 4, cudaMemcpyHostToDevice, st.s));
        GB_CUDA(cudaMemcpyAsync(Y.get(), y, (size_t)rows * O * 4, cudaMemcpyHostToDevice, st.s));
        GB_CUDA(cudaMemcpyAsync(M.get(), mask, (size_t)rows * O * 4, cudaMemcpyHostToDevice, st.s));
        GB_CUDA(cudaMemsetAsync(Gr.get(), 0, NP * 4, st.s));
        GB_CUDA(cudaMemsetAsync(Mo.get(), 0, NP * 4, st.s));
        GB_CUDA(cudaMemsetAsync(Vo.get(), 0, NP * 4, st.s));
        std::vector<int> order(rows);
        std::iota(order.begin(), order.end(), 0);
        std::mt19937_64 rng(seed);
        HostPinned<int> hOrder;
        hOrder.ensure(rows);
        int t = 0;
        for (int ep = 0; ep < epochs; ++ep) {
            std::shuffle(order.begin(), order.end(), rng);
            GB_CUDA(cudaStreamSynchronize(st.s));  // hOrder is reused
            std::memcpy(hOrder.p, order.data(), rows * sizeof(int));
            GB_CUDA(cudaMemcpyAsync(idx.get(), hOrder.p, rows * sizeof(int), cudaMemcpyHostToDevice, st.s));
            for (int b0 = 0; b0 < rows; b0 += batch) {
                const int cnt = std::min(batch, rows - b0);
                GB_CUDA(cudaMemsetAsync(acc.get(), 0, 16, st.s));
                lossGradKernel<<<warpGrid(cnt), 256, 0, st.s>>>(P.get(), X.get(), Y.get(), M.get(), idx.get() + b0,
                                                                cnt, Gr.get(), acc.get());
                ++t;
                adamKernel<<<divUp(NP, 256), 256, 0, st.s>>>(P.get(), Gr.get(), Mo.get(), Vo.get(), acc.get(), lr,
                                                              std::pow(0.9f, (float)t), std::pow(0.999f, (float)t));
                GB_LAUNCH_CHECK();
            }
        }
        // full-data loss of the final parameters
        GB_CUDA(cudaMemsetAsync(acc.get(), 0, 16, st.s));
        GB_CUDA(cudaMemsetAsync(Gr.get(), 0, NP * 4, st.s));
        lossGradKernel<<<warpGrid(rows), 256, 0, st.s>>>(P.get(), X.get(), Y.get(), M.get(), nullptr, rows, Gr.get(),
                                                         acc.get());
        GB_LAUNCH_CHECK();
        double a[2];
        GB_CUDA(cudaMemcpyAsync(a, acc.get(), 16, cudaMemcpyDeviceToHost, st.s));
        GB_CUDA(cudaMemcpyAsync(params_inout, P.get(), NP * 4, cudaMemcpyDeviceToHost, st.s));
        GB_CUDA(cudaStreamSynchronize(st.s));
        if (final_loss) *final_loss = (float)(a[1] > 1 ? a[0] / a[1] : a[0]);
    });
}

}  // extern "C"
