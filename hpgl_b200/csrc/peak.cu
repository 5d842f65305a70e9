// Measured CUDA-core peaks for the roofline of the solve kernels (no
// counterpart in the reference): a kernel of independent fused multiply-add
// chains, timed alone with CUDA events.  The systems are solved on the
// FP32 and FP64 CUDA-core pipes, whose nominal rates depend on the clock
// the part sustains; this measures them on the GPU at hand.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "engine.h"

namespace hpgl_b200 {

namespace {

constexpr int CHAINS = 8;     // independent accumulators per thread
constexpr int UNROLL = 64;    // multiply-adds per chain per loop trip

// FP32: packed two-wide fused multiply-adds (the form the mixed solve uses),
// 2 x CHAINS x UNROLL x iters multiply-adds per thread.
__global__ void __launch_bounds__(256) k_peak_f32(float *out, int iters, float a, float b) {
    float2 acc[CHAINS];
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) acc[c] = make_float2(threadIdx.x * 1e-7f + c, c * 1e-3f);
    const float2 m = make_float2(a, a), k = make_float2(b, b);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < UNROLL; ++u)
#pragma unroll
            for (int c = 0; c < CHAINS; ++c) acc[c] = __ffma2_rn(acc[c], m, k);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) s += acc[c].x + acc[c].y;
    if (s == 1234.5f) out[threadIdx.x] = s;  // keeps the chains live; never true for these inputs
}

__global__ void __launch_bounds__(256) k_peak_f64(double *out, int iters, double a, double b) {
    double acc[CHAINS];
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) acc[c] = threadIdx.x * 1e-9 + c;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < UNROLL; ++u)
#pragma unroll
            for (int c = 0; c < CHAINS; ++c) acc[c] = fma(acc[c], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) s += acc[c];
    if (s == 1234.5) out[threadIdx.x] = s;
}

#define PEAK_CHECK(expr)                                                                       \
    do {                                                                                       \
        cudaError_t e__ = (expr);                                                              \
        if (e__ != cudaSuccess)                                                                \
            throw HpglError{HPGL_E_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e__)}; \
    } while (0)

}  // namespace

// Best of `repeats` timed launches (after one warm-up) of 8 blocks of 256
// threads per SM; returns TFLOP/s (2 flop per multiply-add).
double fma_peak_tflops(int precision, int repeats) {
    int dev = 0, sms = 0;
    PEAK_CHECK(cudaGetDevice(&dev));
    PEAK_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = sms * 8, threads = 256;
    const int iters = precision ? 512 : 256;
    void *out = nullptr;
    PEAK_CHECK(cudaMalloc(&out, threads * sizeof(double)));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    double best = 0.0;
    try {
        PEAK_CHECK(cudaEventCreate(&e0));
        PEAK_CHECK(cudaEventCreate(&e1));
        for (int r = 0; r <= std::max(1, repeats); ++r) {
            PEAK_CHECK(cudaEventRecord(e0));
            if (precision) k_peak_f32<<<blocks, threads>>>((float *)out, iters, 0.999999f, 1e-7f);
            else k_peak_f64<<<blocks, threads>>>((double *)out, iters, 0.999999999, 1e-12);
            PEAK_CHECK(cudaGetLastError());
            PEAK_CHECK(cudaEventRecord(e1));
            PEAK_CHECK(cudaEventSynchronize(e1));
            float ms = 0.f;
            PEAK_CHECK(cudaEventElapsedTime(&ms, e0, e1));
            const double fma_per_thread = (double)iters * UNROLL * CHAINS * (precision ? 2 : 1);
            const double tflops = 2.0 * fma_per_thread * blocks * threads / (ms * 1e-3) / 1e12;
            if (r > 0) best = std::max(best, tflops);
        }
    } catch (...) {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        cudaFree(out);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    return best;
}

}  // namespace hpgl_b200
