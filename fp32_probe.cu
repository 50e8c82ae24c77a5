// FP32 FMA throughput of the device, the denominator of the fine stage's
// roofline in bench.py: every thread runs independent register-resident FMA
// chains, 8 CTAs of 256 threads per SM; the best of 10 timed launches after 3
// warm-up launches (CUDA events on one stream).
//
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -o fp32_probe fp32_probe.cu && ./fp32_probe
//
// Prints one line, `fp32_tflops <value> sm_mhz <clock at launch>`; the measured
// value is committed in profiles/fp32_peak_fma.txt, which bench.py reads.
#include <cstdio>

#include <cuda_runtime.h>

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

int check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        std::fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
        return 1;
    }
    return 0;
}

}  // namespace

int main() {
    int dev = 0, sms = 0, khz = 0;
    if (check(cudaGetDevice(&dev), "device")) return 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, dev);
    float* out = nullptr;
    if (check(cudaMalloc(&out, sizeof(float)), "cudaMalloc")) return 1;
    const int blocks = sms * 8;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    for (int w = 0; w < 3; ++w) k_fma<<<blocks, 256>>>(out, 1.0f);
    float best = 1e30f;
    for (int r = 0; r < 10; ++r) {
        cudaEventRecord(a);
        k_fma<<<blocks, 256>>>(out, 1.0f);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, a, b);
        if (ms < best) best = ms;
    }
    if (check(cudaGetLastError(), "k_fma")) return 1;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    const double flops = 2.0 * double(blocks) * 256.0 * kIters * kChains;
    std::printf("fp32_tflops %.2f sm_mhz %d\n", flops / (double(best) * 1e-3) / 1e12, khz / 1000);
    return 0;
}
