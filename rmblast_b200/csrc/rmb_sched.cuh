#pragma once
// Learned schedule of the preliminary DP: a small MLP predicts each ungapped record's DP cells
// (log1p of the cells of its two X-drop extensions) from features of the record, and the records
// leave the DP queue in descending predicted cost.  The network only orders work: every record
// is still computed by the same kernel, so the output is the same as with the FIFO queue.
//
// Network: 12 features -> 64 -> 64 -> 1, ReLU, BF16 weights, FP32 accumulation.
// Flat parameter layout (floats), shared by the C ABI, the training kernels and the inference
// kernel: W1[12][64] (W1[k * 64 + n]), b1[64], W2[64][64], b2[64], w3[64], b3, then the feature
// normalisation mean[12] and inv_std[12] (x_norm = (x - mean) * inv_std).
#include <cuda_bf16.h>

#include <cstdint>

#include "rmb_device.cuh"

namespace rmb {

constexpr int SCHED_NF = 12, SCHED_H = 64;
constexpr int SCHED_OFF_W1 = 0, SCHED_OFF_B1 = SCHED_NF * SCHED_H, SCHED_OFF_W2 = SCHED_OFF_B1 + SCHED_H,
              SCHED_OFF_B2 = SCHED_OFF_W2 + SCHED_H * SCHED_H, SCHED_OFF_W3 = SCHED_OFF_B2 + SCHED_H,
              SCHED_OFF_B3 = SCHED_OFF_W3 + SCHED_H, SCHED_NET = SCHED_OFF_B3 + 1,
              SCHED_OFF_MEAN = SCHED_NET, SCHED_OFF_ISTD = SCHED_OFF_MEAN + SCHED_NF,
              SCHED_NPARAM = SCHED_OFF_ISTD + SCHED_NF;
// predicted log-cells to a cost bin: 0.25 wide, 64 bins
constexpr int SCHED_BINS = 64;
__host__ __device__ __forceinline__ uint32_t sched_bin(float pred) {
    const float b = pred * 4.0f;
    return b <= 0.0f ? 0u : b >= (float)(SCHED_BINS - 1) ? (uint32_t)(SCHED_BINS - 1) : (uint32_t)b;
}

// The network in shared memory, BF16 weights stored output-major (Wt[n][k]) so that an mma
// B fragment (two consecutive k of one n) is one 32-bit load; k padded to 16 for layer 1 and
// layer 3's single output padded to 8 columns.
struct SchedSmem {
    uint16_t w1t[SCHED_H][16];
    uint16_t w2t[SCHED_H][SCHED_H];
    uint16_t w3t[8][SCHED_H];
    float b1[SCHED_H], b2[SCHED_H], b3;
    float mean[SCHED_NF], istd[SCHED_NF];
};

__device__ __forceinline__ uint16_t sched_bf16(float x) {
    const __nv_bfloat16 h = __float2bfloat16_rn(x);
    return *reinterpret_cast<const uint16_t*>(&h);
}
__device__ __forceinline__ uint32_t sched_pack2(float lo, float hi) {
    return (uint32_t)sched_bf16(lo) | ((uint32_t)sched_bf16(hi) << 16);
}

// Block-wide load of the parameters into shared memory (all threads of the block call it).
__device__ __forceinline__ void sched_load(SchedSmem& S, const float* __restrict__ p) {
    for (int i = threadIdx.x; i < SCHED_H * 16; i += blockDim.x) {
        const int n = i / 16, k = i % 16;
        S.w1t[n][k] = sched_bf16(k < SCHED_NF ? p[SCHED_OFF_W1 + k * SCHED_H + n] : 0.0f);
    }
    for (int i = threadIdx.x; i < SCHED_H * SCHED_H; i += blockDim.x) {
        const int n = i / SCHED_H, k = i % SCHED_H;
        S.w2t[n][k] = sched_bf16(p[SCHED_OFF_W2 + k * SCHED_H + n]);
    }
    for (int i = threadIdx.x; i < 8 * SCHED_H; i += blockDim.x) {
        const int n = i / SCHED_H, k = i % SCHED_H;
        S.w3t[n][k] = sched_bf16(n == 0 ? p[SCHED_OFF_W3 + k] : 0.0f);
    }
    for (int i = threadIdx.x; i < SCHED_H; i += blockDim.x) {
        S.b1[i] = p[SCHED_OFF_B1 + i];
        S.b2[i] = p[SCHED_OFF_B2 + i];
    }
    for (int i = threadIdx.x; i < SCHED_NF; i += blockDim.x) {
        S.mean[i] = p[SCHED_OFF_MEAN + i];
        S.istd[i] = p[SCHED_OFF_ISTD + i];
    }
    if (threadIdx.x == 0) S.b3 = p[SCHED_OFF_B3];
}

// D += A (16x16 bf16, row-major fragment) * B (16x8 bf16, column fragment), FP32 accumulate.
__device__ __forceinline__ void sched_mma(float d[4], const uint32_t a[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// One hidden layer on a 16-row tile: H = relu(A * W + b) for 64 outputs, with A given as the four
// k-tiles of the previous layer (kt k-tiles), returned as the four k-tiles of the next layer's A.
template <int KT>
__device__ __forceinline__ void sched_layer(const uint32_t a[KT][4], const uint16_t* wt, int ldw, const float* bias,
                                            uint32_t out[4][4], int g, int t) {
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        float d[4] = {0.f, 0.f, 0.f, 0.f};
        const uint16_t* row = wt + (nt * 8 + g) * ldw;
#pragma unroll
        for (int kk = 0; kk < KT; ++kk)
            sched_mma(d, a[kk], *reinterpret_cast<const uint32_t*>(row + kk * 16 + 2 * t),
                      *reinterpret_cast<const uint32_t*>(row + kk * 16 + 2 * t + 8));
        const float c0 = bias[nt * 8 + 2 * t], c1 = bias[nt * 8 + 2 * t + 1];
        // C fragment (rows g, g + 8; columns 2t, 2t + 1 of this n-tile) -> A fragment of k-tile nt / 2
        const uint32_t lo = sched_pack2(fmaxf(d[0] + c0, 0.f), fmaxf(d[1] + c1, 0.f));
        const uint32_t hi = sched_pack2(fmaxf(d[2] + c0, 0.f), fmaxf(d[3] + c1, 0.f));
        out[nt >> 1][(nt & 1) * 2 + 0] = lo;
        out[nt >> 1][(nt & 1) * 2 + 1] = hi;
    }
}

// The network on the 32 records of a warp: lane l passes its record's 12 normalised features and
// gets its prediction back.  xs: this warp's 32 x 16 BF16 staging tile in shared memory.  Every
// lane of the warp must call it.
__device__ __forceinline__ float sched_mlp_warp(const SchedSmem& S, uint16_t (*xs)[16], float* ys, const float f[SCHED_NF]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int k = 0; k < 16; ++k) xs[lane][k] = sched_bf16(k < SCHED_NF ? f[k] : 0.0f);
    __syncwarp();
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
        const int r0 = mt * 16 + g, r1 = r0 + 8;
        uint32_t a1[1][4];
        a1[0][0] = *reinterpret_cast<const uint32_t*>(&xs[r0][2 * t]);
        a1[0][1] = *reinterpret_cast<const uint32_t*>(&xs[r1][2 * t]);
        a1[0][2] = *reinterpret_cast<const uint32_t*>(&xs[r0][2 * t + 8]);
        a1[0][3] = *reinterpret_cast<const uint32_t*>(&xs[r1][2 * t + 8]);
        uint32_t a2[4][4], a3[4][4];
        sched_layer<1>(a1, &S.w1t[0][0], 16, S.b1, a2, g, t);
        sched_layer<4>(a2, &S.w2t[0][0], SCHED_H, S.b2, a3, g, t);
        float d[4] = {0.f, 0.f, 0.f, 0.f};
        const uint16_t* row = &S.w3t[g][0];
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)
            sched_mma(d, a3[kk], *reinterpret_cast<const uint32_t*>(row + kk * 16 + 2 * t),
                      *reinterpret_cast<const uint32_t*>(row + kk * 16 + 2 * t + 8));
        if (t == 0) {  // column 0: the output
            ys[r0] = d[0] + S.b3;
            ys[r1] = d[2] + S.b3;
        }
    }
    __syncwarp();
    const float y = ys[lane];
    __syncwarp();
    return y;
}

}  // namespace rmb
