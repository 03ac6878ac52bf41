// FMA-pipe throughput microbenchmark: the roofline denominator for the
// polynomial kernels, which are FP64 (FP32 for the mixed leaf level) FMA bound.
//
// Each thread runs 8 independent FMA chains so the pipe, not latency, limits
// throughput; the grid fills every SM.  Reported as FLOP/s (one FMA = 2 flops).
#include <cuda_runtime.h>

#include "../../include/mbx_b200.h"

namespace {

constexpr int CHAINS = 8;

__global__ void __launch_bounds__(256) k_dfma(double* out, int iters, double a, double b) {
    double v[CHAINS];
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) v[c] = threadIdx.x * 1e-9 + c;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < CHAINS; ++c) v[c] = fma(v[c], a, b);
    }
    double s = 0;
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) s += v[c];
    if (s == 1.2345) out[0] = s;  // keeps the chains live
}

__global__ void __launch_bounds__(256) k_ffma(float* out, int iters, float a, float b) {
    float v[CHAINS];
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) v[c] = threadIdx.x * 1e-6f + c;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < CHAINS; ++c) v[c] = fmaf(v[c], a, b);
    }
    float s = 0;
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) s += v[c];
    if (s == 1.2345f) out[0] = s;
}

// Paired FP32 FMA (fma.rn.f32x2, two lanes of FP32 per instruction).
__global__ void __launch_bounds__(256) k_ffma2(float* out, int iters, float a, float b) {
    unsigned long long v[CHAINS];
    const unsigned long long av = ((unsigned long long)__float_as_uint(a) << 32) | __float_as_uint(a);
    const unsigned long long bv = ((unsigned long long)__float_as_uint(b) << 32) | __float_as_uint(b);
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) {
        const float f = threadIdx.x * 1e-6f + c;
        v[c] = ((unsigned long long)__float_as_uint(f) << 32) | __float_as_uint(f + 0.5f);
    }
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < CHAINS; ++c) asm("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(v[c]) : "l"(av), "l"(bv));
    }
    float s = 0;
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) s += __uint_as_float((unsigned)v[c]) + __uint_as_float((unsigned)(v[c] >> 32));
    if (s == 1.2345f) out[0] = s;
}

}  // namespace

// results[0] = FP64 FMA TFLOP/s, results[1] = FP32 FMA TFLOP/s,
// results[2] = FP32 via fma.rn.f32x2 TFLOP/s (device-timed).
extern "C" int mbx_fma_peaks(int device, double* results) {
    if (!results) return MBX_EINVAL;
    if (cudaSetDevice(device) != cudaSuccess) return MBX_ENODEV;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    void* buf = nullptr;
    if (cudaMalloc(&buf, 64) != cudaSuccess) return MBX_ENOMEM;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int block = 256, grid = sms * 8, iters = 1 << 14;
    const double flops = 2.0 * CHAINS * (double)iters * block * grid;
    for (int kind = 0; kind < 3; ++kind) {
        float best = 1e30f;
        for (int rep = 0; rep < 5; ++rep) {
            cudaEventRecord(e0);
            if (kind == 0) k_dfma<<<grid, block>>>((double*)buf, iters, 0.999999, 1e-7);
            else if (kind == 1) k_ffma<<<grid, block>>>((float*)buf, iters, 0.999999f, 1e-7f);
            else k_ffma2<<<grid, block>>>((float*)buf, iters, 0.999999f, 1e-7f);
            cudaEventRecord(e1);
            cudaEventSynchronize(e1);
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0 && ms < best) best = ms;
        }
        results[kind] = (kind == 2 ? 2.0 : 1.0) * flops / (best * 1e-3) / 1e12;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(buf);
    return cudaGetLastError() == cudaSuccess ? MBX_OK : MBX_ECUDA;
}
