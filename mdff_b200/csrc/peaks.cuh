// peaks.cuh -- measured arithmetic-pipe throughput of the device.
//
// Roofline denominators of the engine's kernels: FMA throughputs (FP64,
// FP32, packed FP32x2) measured with long chains of independent FMAs (every
// SM filled), and the tcgen05 kind::i8 tensor-core throughput of the
// reciprocal-space GEMMs, measured with back-to-back MMAs from resident
// shared-memory operands (one CTA per SM); all timed with CUDA events.
#include "common.cuh"
#include "umma.cuh"

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

// tcgen05 kind::i8 throughput: M = 128, N as given, K = 64 bytes per
// iteration (two MMAs), accumulating into tensor memory; every wait bounded.
template <int N>
__global__ void __launch_bounds__(128) k_peak_i8(int niter, int* err) {
    constexpr int KB = 64;
    extern __shared__ __align__(128) uint8_t pk_smem[];
    uint8_t* sm = pk_smem;
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t slot;
    const int tid = threadIdx.x, warp = tid >> 5;
    for (int i = tid; i < (128 + N) * KB / 4; i += 128) reinterpret_cast<uint32_t*>(sm)[i] = 0x01010101u;
    if (warp == 0) umma::tmem_alloc(&slot, 256);
    if (tid == 0) umma::mbar_init(&mbar, 1);
    umma::fence_smem_to_async();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tm = slot;
    if (tid == 0) {
        const uint32_t a0 = umma::smem_u32(sm), b0 = a0 + 128 * KB;
        const uint32_t lboA = 16 * 128, lboB = (N / 8) * 128;
        for (int r = 0; r < niter; ++r)
            for (int s = 0; s < KB / 32; ++s)
                umma::mma_s8(tm, umma::desc_kmajor(a0 + 2 * s * lboA, lboA, 128),
                             umma::desc_kmajor(b0 + 2 * s * lboB, lboB, 128), umma::idesc_s8(128, N), (r | s) != 0);
        umma::commit(&mbar);
    }
    __syncwarp();
    if (!umma::mbar_wait_ns(&mbar, 0, 2000000000ull) && tid == 0) atomicOr(err, 1);
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        umma::fence_after_sync();
        umma::tmem_dealloc(tm, 256);
    }
}

}  // namespace mdff
