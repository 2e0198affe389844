// rmb_probe.cu -- int32 throughput probe: the denominator of the DP kernels' roofline.
//
// The X-drop DP cell is add / subtract / max / compare on int32 (search/gapped.rs:234-262), so
// its ceiling is the SM integer pipe, not HBM or the tensor cores.  This kernel keeps 8
// independent max-plus chains per thread (one add + one max per step, the DP's mix) at full
// occupancy and reports the sustained int32 operations per second.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/rmb_gpu.h"

namespace {
__global__ void k_int32_probe(int32_t* out, int32_t iters, int32_t a, int32_t b) {
    int32_t x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6,
            x7 = x0 + 7;
    for (int32_t i = 0; i < iters; ++i) {
        x0 = max(x0 + a, x1 - b); x1 = max(x1 + a, x2 - b); x2 = max(x2 + a, x3 - b); x3 = max(x3 + a, x4 - b);
        x4 = max(x4 + a, x5 - b); x5 = max(x5 + a, x6 - b); x6 = max(x6 + a, x7 - b); x7 = max(x7 + a, x0 - b);
    }
    if ((x0 ^ x1 ^ x2 ^ x3 ^ x4 ^ x5 ^ x6 ^ x7) == 0x7fffffff) out[0] = x0;
}
}  // namespace

extern "C" int rmb_probe_int32_peak(int32_t device, double* tops, char* err, size_t errlen) {
    auto bad = [&](cudaError_t e) {
        if (err && errlen) {
            const char* m = cudaGetErrorString(e);
            size_t i = 0;
            for (; m[i] && i + 1 < errlen; ++i) err[i] = m[i];
            err[i] = 0;
        }
        return RMB_ECUDA;
    };
    cudaError_t e;
    if ((e = cudaSetDevice(device)) != cudaSuccess) return bad(e);
    int sms = 0;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess) return bad(e);
    int32_t* out = nullptr;
    if ((e = cudaMalloc(&out, 4)) != cudaSuccess) return bad(e);
    const int block = 256, grid = sms * 8;
    const int32_t iters = 1 << 14;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    k_int32_probe<<<grid, block>>>(out, 256, 3, 5);  // warm-up
    cudaEventRecord(t0);
    k_int32_probe<<<grid, block>>>(out, iters, 3, 5);
    cudaEventRecord(t1);
    e = cudaEventSynchronize(t1);
    float ms = 0;
    cudaEventElapsedTime(&ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    cudaFree(out);
    if (e != cudaSuccess) return bad(e);
    // per step and chain: one add, one subtract, one max
    const double ops = (double)grid * block * iters * 8 * 3;
    *tops = ops / (ms * 1e-3) / 1e12;
    return RMB_OK;
}
