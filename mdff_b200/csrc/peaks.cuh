// peaks.cuh -- measured arithmetic-pipe throughput of the device.
//
// The engine's hot kernels are bound by the FP64 or FP32 FMA pipes (no
// tensor-core contraction, working sets in L2), so their roofline denominators
// are FMA throughputs, measured here with long chains of independent FMAs
// (8 chains per thread, every SM filled), timed with CUDA events.
#include "common.cuh"

namespace mdff {

constexpr int PK_ITERS = 4096;

__global__ void __launch_bounds__(256) k_peak_f64(double* out, double seed) {
    double a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = seed + k + threadIdx.x;
    const double b = 0.999999, c = 1e-7;
    for (int it = 0; it < PK_ITERS; ++it) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = fma(a[k], b, c);
    }
    double s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == 1234.5678) out[0] = s;
}

__global__ void __launch_bounds__(256) k_peak_f32(float* out, float seed) {
    float a[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) a[k] = seed + k + threadIdx.x;
    const float b = 0.9999f, c = 1e-7f;
    for (int it = 0; it < PK_ITERS; ++it) {
#pragma unroll
        for (int k = 0; k < 16; ++k) a[k] = fmaf(a[k], b, c);
    }
    float s = 0;
#pragma unroll
    for (int k = 0; k < 16; ++k) s += a[k];
    if (s == 1234.5678f) out[0] = s;
}

__global__ void __launch_bounds__(256) k_peak_f32x2(float* out, float seed) {
    unsigned long long a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        float2 v = make_float2(seed + k, seed - k + threadIdx.x);
        a[k] = *reinterpret_cast<unsigned long long*>(&v);
    }
    float2 bb = make_float2(0.9999f, 0.9998f), cc = make_float2(1e-7f, 2e-7f);
    const unsigned long long b = *reinterpret_cast<unsigned long long*>(&bb);
    const unsigned long long c = *reinterpret_cast<unsigned long long*>(&cc);
    for (int it = 0; it < PK_ITERS; ++it) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = ffma2(a[k], b, c);
    }
    float s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        float2 v = *reinterpret_cast<float2*>(&a[k]);
        s += v.x + v.y;
    }
    if (s == 1234.5678f) out[0] = s;
}

}  // namespace mdff
