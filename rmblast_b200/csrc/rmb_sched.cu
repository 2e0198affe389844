// rmb_sched.cu -- training of the learned schedule's network (rmb_sched.cuh) on the GPU, and the
// C entry points that train it, take its gradients and run its inference on given features.
//
// Training runs the network in FP32 with BF16-rounded weights (the inference kernel's weights):
// forward  Z1 = X W1 + b1, H1 = relu(Z1), Z2 = H1 W2 + b2, H2 = relu(Z2), y = H2 w3 + b3,
// loss     mean((y - t)^2) with t = log1p(cells),
// backward dy = 2 (y - t) / B; dw3 = H2^T dy; dZ2 = (dy w3^T) * [Z2 > 0]; dW2 = H1^T dZ2;
//          dZ1 = (dZ2 W2^T) * [Z1 > 0]; dW1 = X^T dZ1; bias gradients are column sums;
// and Adam on FP32 master weights (rate falling linearly to a tenth), re-rounded to BF16 after
// every step.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/rmb_gpu.h"
#include "rmb_kernels.hpp"
#include "rmb_sched.cuh"

namespace rmb {
static_assert(RMB_SCHED_NET == SCHED_NET && RMB_SCHED_NPARAM == SCHED_NPARAM, "parameter layout");
namespace {

struct SchedError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

void ck(cudaError_t e) {
    if (e != cudaSuccess) throw SchedError(std::string("CUDA: ") + cudaGetErrorString(e));
}

struct Buf {  // device buffer owned by one call
    void* p = nullptr;
    explicit Buf(size_t n) { ck(cudaMalloc(&p, std::max<size_t>(n, 16))); }
    ~Buf() {
        if (p) cudaFree(p);
    }
    Buf(const Buf&) = delete;
    Buf& operator=(const Buf&) = delete;
    float* f() const { return (float*)p; }
    uint32_t* u() const { return (uint32_t*)p; }
};

// C (M x N, ldc) = op(A) (M x K) * op(B) (K x N), 16 x 16 tiles.
template <bool TA, bool TB>
__global__ void k_gemm(int M, int N, int K, const float* __restrict__ A, int lda, const float* __restrict__ B, int ldb,
                       float* __restrict__ C, int ldc) {
    __shared__ float As[16][17], Bs[16][17];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int r = blockIdx.y * 16 + ty, c = blockIdx.x * 16 + tx;
    float acc = 0.0f;
    for (int k0 = 0; k0 < K; k0 += 16) {
        const int ka = k0 + tx, kb = k0 + ty;
        As[ty][tx] = (r < M && ka < K) ? (TA ? A[(size_t)ka * lda + r] : A[(size_t)r * lda + ka]) : 0.0f;
        Bs[ty][tx] = (kb < K && c < N) ? (TB ? B[(size_t)c * ldb + kb] : B[(size_t)kb * ldb + c]) : 0.0f;
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) acc += As[ty][kk] * Bs[kk][tx];
        __syncthreads();
    }
    if (r < M && c < N) C[(size_t)r * ldc + c] = acc;
}

template <bool TA, bool TB>
void gemm(int M, int N, int K, const float* A, int lda, const float* B, int ldb, float* C, int ldc, cudaStream_t st) {
    const dim3 blk(16, 16), grd((N + 15) / 16, (M + 15) / 16);
    k_gemm<TA, TB><<<grd, blk, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc);
    ck(cudaGetLastError());
}

// Z += bias (per column); H = relu(Z) (H may be null: bias only)
__global__ void k_bias_relu(int M, int N, float* __restrict__ Z, const float* __restrict__ bias, float* __restrict__ H) {
    const size_t n = (size_t)M * N;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float z = Z[i] + bias[i % N];
        Z[i] = z;
        if (H) H[i] = fmaxf(z, 0.0f);
    }
}

// D *= [Z > 0]
__global__ void k_relu_bwd(size_t n, float* __restrict__ D, const float* __restrict__ Z) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        if (Z[i] <= 0.0f) D[i] = 0.0f;
}

// out[j] = sum_i X[i][j], one block per column
__global__ void k_colsum(int M, int N, const float* __restrict__ X, float* __restrict__ out) {
    __shared__ float red[256];
    const int j = blockIdx.x;
    float s = 0.0f;
    for (int i = threadIdx.x; i < M; i += blockDim.x) s += X[(size_t)i * N + j];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[j] = red[0];
}

// dy = 2 (y - t) / B (y gets + b3 first); sse += sum (y - t)^2
__global__ void k_mse(int M, float* __restrict__ y, const float* __restrict__ b3, const float* __restrict__ t,
                      float* __restrict__ dy, float scale, double* __restrict__ sse) {
    __shared__ double red[256];
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M; i += gridDim.x * blockDim.x) {
        const float v = y[i] + b3[0];
        y[i] = v;
        const float e = v - t[i];
        if (dy) dy[i] = 2.0f * e * scale;
        s += (double)e * e;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(sse, red[0]);
}

__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// Adam step on the master weights w (n = SCHED_NET), then wq = bf16(w)
__global__ void k_adam(int n, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float c1, float c2, float* __restrict__ wq) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi, vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        wq[i] = bf16_round(wi);
    }
}

__global__ void k_round_bf16(int n, const float* __restrict__ w, float* __restrict__ wq) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) wq[i] = bf16_round(w[i]);
}

// X[i][k] = (raw[i][k] - mean[k]) * istd[k]
__global__ void k_normalize(size_t n, const float* __restrict__ raw, const float* __restrict__ params,
                            float* __restrict__ X) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n * SCHED_NF; i += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(i % SCHED_NF);
        X[i] = (raw[i] - params[SCHED_OFF_MEAN + k]) * params[SCHED_OFF_ISTD + k];
    }
}

// rows perm[0..m) of X and t into Xb, tb
__global__ void k_gather_rows(int m, const uint32_t* __restrict__ perm, const float* __restrict__ X,
                              const float* __restrict__ t, float* __restrict__ Xb, float* __restrict__ tb) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m * SCHED_NF; i += gridDim.x * blockDim.x) {
        const int r = i / SCHED_NF, k = i % SCHED_NF;
        Xb[i] = X[(size_t)perm[r] * SCHED_NF + k];
        if (k == 0) tb[r] = t[perm[r]];
    }
}

int blocks(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 4096); }

// Activations and gradients of one batch of up to B rows.
struct Work {
    int B;
    Buf z1, h1, z2, h2, y, dy, d2, d1, grad;
    Buf sse;
    explicit Work(int b)
        : B(b), z1((size_t)b * SCHED_H * 4), h1((size_t)b * SCHED_H * 4), z2((size_t)b * SCHED_H * 4),
          h2((size_t)b * SCHED_H * 4), y((size_t)b * 4), dy((size_t)b * 4), d2((size_t)b * SCHED_H * 4),
          d1((size_t)b * SCHED_H * 4), grad(SCHED_NET * 4), sse(8) {}
};

// Forward over M rows (Xb normalised, M x 12) with weights wq; with tb: the squared error into
// sse, and with `backward` also the gradient into W.grad.
void forward_backward(Work& W, int M, const float* Xb, const float* tb, const float* wq, bool backward,
                      cudaStream_t st) {
    const float* w1 = wq + SCHED_OFF_W1;
    const float* w2 = wq + SCHED_OFF_W2;
    const float* w3 = wq + SCHED_OFF_W3;
    gemm<false, false>(M, SCHED_H, SCHED_NF, Xb, SCHED_NF, w1, SCHED_H, W.z1.f(), SCHED_H, st);
    k_bias_relu<<<blocks((size_t)M * SCHED_H), 256, 0, st>>>(M, SCHED_H, W.z1.f(), wq + SCHED_OFF_B1, W.h1.f());
    gemm<false, false>(M, SCHED_H, SCHED_H, W.h1.f(), SCHED_H, w2, SCHED_H, W.z2.f(), SCHED_H, st);
    k_bias_relu<<<blocks((size_t)M * SCHED_H), 256, 0, st>>>(M, SCHED_H, W.z2.f(), wq + SCHED_OFF_B2, W.h2.f());
    gemm<false, false>(M, 1, SCHED_H, W.h2.f(), SCHED_H, w3, 1, W.y.f(), 1, st);
    k_mse<<<std::min(blocks(M), 256), 256, 0, st>>>(M, W.y.f(), wq + SCHED_OFF_B3, tb, backward ? W.dy.f() : nullptr,
                                                    1.0f / (float)M, (double*)W.sse.p);
    ck(cudaGetLastError());
    if (!backward) return;
    float* g = W.grad.f();
    gemm<true, false>(SCHED_H, 1, M, W.h2.f(), SCHED_H, W.dy.f(), 1, g + SCHED_OFF_W3, 1, st);
    k_colsum<<<1, 256, 0, st>>>(M, 1, W.dy.f(), g + SCHED_OFF_B3);
    gemm<false, false>(M, SCHED_H, 1, W.dy.f(), 1, w3, SCHED_H, W.d2.f(), SCHED_H, st);
    k_relu_bwd<<<blocks((size_t)M * SCHED_H), 256, 0, st>>>((size_t)M * SCHED_H, W.d2.f(), W.z2.f());
    gemm<true, false>(SCHED_H, SCHED_H, M, W.h1.f(), SCHED_H, W.d2.f(), SCHED_H, g + SCHED_OFF_W2, SCHED_H, st);
    k_colsum<<<SCHED_H, 256, 0, st>>>(M, SCHED_H, W.d2.f(), g + SCHED_OFF_B2);
    gemm<false, true>(M, SCHED_H, SCHED_H, W.d2.f(), SCHED_H, w2, SCHED_H, W.d1.f(), SCHED_H, st);
    k_relu_bwd<<<blocks((size_t)M * SCHED_H), 256, 0, st>>>((size_t)M * SCHED_H, W.d1.f(), W.z1.f());
    gemm<true, false>(SCHED_NF, SCHED_H, M, Xb, SCHED_NF, W.d1.f(), SCHED_H, g + SCHED_OFF_W1, SCHED_H, st);
    k_colsum<<<SCHED_H, 256, 0, st>>>(M, SCHED_H, W.d1.f(), g + SCHED_OFF_B1);
    ck(cudaGetLastError());
}

int fail(const std::exception& e, char* err, size_t errlen, int code) {
    if (err && errlen) snprintf(err, errlen, "%s", e.what());
    return code;
}

}  // namespace
}  // namespace rmb

using namespace rmb;

extern "C" {

int rmb_sched_grad(int32_t device, const float* params, const float* features, const float* targets, uint32_t n,
                   float* grad_out, float* loss_out, char* err, size_t errlen) {
    try {
        if (!params || !features || !targets || !grad_out || !n) throw SchedError("null argument or no rows");
        ck(cudaSetDevice(device));
        cudaStream_t st = 0;
        Buf p(SCHED_NPARAM * 4), wq(SCHED_NPARAM * 4), raw((size_t)n * SCHED_NF * 4), X((size_t)n * SCHED_NF * 4),
            t((size_t)n * 4);
        ck(cudaMemcpy(p.p, params, SCHED_NPARAM * 4, cudaMemcpyHostToDevice));
        ck(cudaMemcpy(raw.p, features, (size_t)n * SCHED_NF * 4, cudaMemcpyHostToDevice));
        ck(cudaMemcpy(t.p, targets, (size_t)n * 4, cudaMemcpyHostToDevice));
        k_round_bf16<<<blocks(SCHED_NET), 256, 0, st>>>(SCHED_NET, p.f(), wq.f());
        k_normalize<<<blocks((size_t)n * SCHED_NF), 256, 0, st>>>(n, raw.f(), p.f(), X.f());
        Work W((int)n);
        ck(cudaMemset(W.sse.p, 0, 8));
        forward_backward(W, (int)n, X.f(), t.f(), wq.f(), true, st);
        double sse = 0;
        ck(cudaMemcpy(grad_out, W.grad.p, SCHED_NET * 4, cudaMemcpyDeviceToHost));
        ck(cudaMemcpy(&sse, W.sse.p, 8, cudaMemcpyDeviceToHost));
        if (loss_out) *loss_out = (float)(sse / n);
        return RMB_OK;
    } catch (const std::exception& e) {
        return fail(e, err, errlen, RMB_ECUDA);
    }
}

int rmb_sched_predict(int32_t device, const float* params, const float* features, uint64_t n, float* pred_out,
                      char* err, size_t errlen) {
    try {
        if (!params || !features || !pred_out) throw SchedError("null argument");
        if (!n) return RMB_OK;
        ck(cudaSetDevice(device));
        int sms = 0;
        ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        Buf p(SCHED_NPARAM * 4), f(n * SCHED_NF * 4), y(n * 4);
        ck(cudaMemcpy(p.p, params, SCHED_NPARAM * 4, cudaMemcpyHostToDevice));
        ck(cudaMemcpy(f.p, features, n * SCHED_NF * 4, cudaMemcpyHostToDevice));
        ck(launch_sched_predict_features(n, f.f(), p.f(), y.f(), sms, 0));
        ck(cudaMemcpy(pred_out, y.p, n * 4, cudaMemcpyDeviceToHost));
        return RMB_OK;
    } catch (const std::exception& e) {
        return fail(e, err, errlen, RMB_ECUDA);
    }
}

int rmb_sched_train(int32_t device, const float* features, const float* targets, uint64_t n, uint32_t epochs,
                    uint32_t batch, float lr, uint64_t seed, float val_fraction, float* params_io, float* stats_out,
                    char* err, size_t errlen) {
    try {
        if (!features || !targets || !params_io || !n || !batch) throw SchedError("null argument or empty input");
        if (!(val_fraction >= 0.0f && val_fraction < 1.0f)) throw SchedError("val_fraction must be in [0, 1)");
        if (n > 0xffffffffull) throw SchedError("at most 2^32 - 1 training rows");
        ck(cudaSetDevice(device));
        cudaStream_t st = 0;
        Buf p(SCHED_NPARAM * 4), wq(SCHED_NPARAM * 4), m(SCHED_NET * 4), v(SCHED_NET * 4);
        Buf raw(n * SCHED_NF * 4), X(n * SCHED_NF * 4), t(n * 4);
        ck(cudaMemcpy(p.p, params_io, SCHED_NPARAM * 4, cudaMemcpyHostToDevice));
        ck(cudaMemcpy(raw.p, features, n * SCHED_NF * 4, cudaMemcpyHostToDevice));
        ck(cudaMemcpy(t.p, targets, n * 4, cudaMemcpyHostToDevice));
        ck(cudaMemset(m.p, 0, SCHED_NET * 4));
        ck(cudaMemset(v.p, 0, SCHED_NET * 4));
        k_normalize<<<blocks(n * SCHED_NF), 256, 0, st>>>(n, raw.f(), p.f(), X.f());
        k_round_bf16<<<blocks(SCHED_NET), 256, 0, st>>>(SCHED_NET, p.f(), wq.f());
        // a seeded split: the last val_fraction of a shuffled index is held out
        std::mt19937_64 rng(seed);
        std::vector<uint32_t> idx(n);
        std::iota(idx.begin(), idx.end(), 0u);
        std::shuffle(idx.begin(), idx.end(), rng);
        const uint64_t n_val = (uint64_t)((double)n * val_fraction);
        const uint64_t n_tr = n - n_val;
        std::vector<uint32_t> tr(idx.begin(), idx.begin() + n_tr);
        Buf perm(n * 4);
        const int B = (int)std::min<uint64_t>(batch, std::max<uint64_t>(n_tr, 1));
        Work W(B);
        Buf Xb((size_t)B * SCHED_NF * 4), tb((size_t)B * 4);
        uint64_t step = 0;
        const uint64_t total_steps = (uint64_t)epochs * ((n_tr + B - 1) / B);
        for (uint32_t e = 0; e < epochs; ++e) {
            std::shuffle(tr.begin(), tr.end(), rng);
            ck(cudaMemcpyAsync(perm.p, tr.data(), n_tr * 4, cudaMemcpyHostToDevice, st));
            ck(cudaMemsetAsync(W.sse.p, 0, 8, st));
            for (uint64_t b0 = 0; b0 < n_tr; b0 += B) {
                const int M = (int)std::min<uint64_t>(B, n_tr - b0);
                k_gather_rows<<<blocks((size_t)M * SCHED_NF), 256, 0, st>>>(M, perm.u() + b0, X.f(), t.f(), Xb.f(),
                                                                           tb.f());
                forward_backward(W, M, Xb.f(), tb.f(), wq.f(), true, st);
                ++step;
                const float c1 = 1.0f - powf(0.9f, (float)step), c2 = 1.0f - powf(0.999f, (float)step);
                // the rate falls linearly to a tenth over the run
                const float lr_t = lr * (1.0f - 0.9f * (float)(step - 1) / (float)std::max<uint64_t>(total_steps, 1));
                k_adam<<<blocks(SCHED_NET), 256, 0, st>>>(SCHED_NET, p.f(), W.grad.f(), m.f(), v.f(), lr_t, c1, c2,
                                                          wq.f());
                ck(cudaGetLastError());
            }
            double sse = 0;
            ck(cudaMemcpyAsync(&sse, W.sse.p, 8, cudaMemcpyDeviceToHost, st));
            ck(cudaStreamSynchronize(st));
            if (stats_out) stats_out[e] = (float)(sse / (double)n_tr);  // mean squared error of the epoch
        }
        // held-out root mean squared error in log-cells, with the trained BF16 weights
        double sse_val = 0;
        if (n_val) {
            std::vector<uint32_t> va(idx.begin() + n_tr, idx.end());
            ck(cudaMemcpyAsync(perm.p, va.data(), n_val * 4, cudaMemcpyHostToDevice, st));
            ck(cudaMemsetAsync(W.sse.p, 0, 8, st));
            for (uint64_t b0 = 0; b0 < n_val; b0 += B) {
                const int M = (int)std::min<uint64_t>(B, n_val - b0);
                k_gather_rows<<<blocks((size_t)M * SCHED_NF), 256, 0, st>>>(M, perm.u() + b0, X.f(), t.f(), Xb.f(),
                                                                           tb.f());
                forward_backward(W, M, Xb.f(), tb.f(), wq.f(), false, st);
            }
            ck(cudaMemcpyAsync(&sse_val, W.sse.p, 8, cudaMemcpyDeviceToHost, st));
        }
        // the trained weights, BF16-rounded as the inference kernel uses them
        ck(cudaMemcpyAsync(params_io, wq.p, SCHED_NET * 4, cudaMemcpyDeviceToHost, st));
        ck(cudaStreamSynchronize(st));
        if (stats_out) stats_out[epochs] = n_val ? (float)std::sqrt(sse_val / (double)n_val) : 0.0f;
        return RMB_OK;
    } catch (const std::exception& e) {
        return fail(e, err, errlen, RMB_ECUDA);
    }
}

}  // extern "C"
