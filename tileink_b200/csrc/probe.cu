// FP32 FMA throughput probe: every thread runs independent register-resident
// FMA chains; the result is the denominator of the fine stage's roofline.
#include <cuda_runtime.h>

#include "kernels.h"

namespace tk {
namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;

__global__ void __launch_bounds__(256) k_fma(float* out, float seed) {
    float a[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = seed + float(threadIdx.x + k);
    const float m = 0.999999f, c = 1e-7f;
    for (int i = 0; i < kIters; ++i) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) a[k] = __fmaf_rn(a[k], m, c);
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += a[k];
    if (s == 1234.5f) out[0] = s;  // keeps the chains live
}

}  // namespace

double probe_fp32_tflops(cudaStream_t st) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    float* out = nullptr;
    cudaMalloc(&out, sizeof(float));
    const int blocks = sms * 8;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    for (int w = 0; w < 3; ++w) k_fma<<<blocks, 256, 0, st>>>(out, 1.0f);
    float best = 1e30f;
    for (int r = 0; r < 10; ++r) {
        cudaEventRecord(a, st);
        k_fma<<<blocks, 256, 0, st>>>(out, 1.0f);
        cudaEventRecord(b, st);
        cudaEventSynchronize(b);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, a, b);
        if (ms < best) best = ms;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    double flops = 2.0 * double(blocks) * 256.0 * kIters * kChains;
    return flops / (double(best) * 1e-3) / 1e12;
}

}  // namespace tk
