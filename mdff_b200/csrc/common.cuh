// common.cuh -- device helpers shared by the engine's kernels.
#pragma once
#include <cuda_runtime.h>
#include "engine_internal.h"

namespace mdff {

// Minimum-image pair vector from direct (fractional) coordinates in exactly the
// operation order of vnlist_pbc (src/tools.f90:323-332): d = si - sj,
// d - NINT(d) (half away from zero: round()), then r = A d row by row, and
// |r|^2 summed x, y, z.  Every multiply and add is a separate IEEE operation
// (no FMA), so the inclusion test matches the reference bit for bit.
__device__ __forceinline__ double pairvec_exact(const CellP& c, double si1, double si2, double si3,
                                                double sj1, double sj2, double sj3,
                                                double& rx, double& ry, double& rz) {
    double dx = __dsub_rn(si1, sj1), dy = __dsub_rn(si2, sj2), dz = __dsub_rn(si3, sj3);
    dx = __dsub_rn(dx, round(dx));
    dy = __dsub_rn(dy, round(dy));
    dz = __dsub_rn(dz, round(dz));
    rx = __dadd_rn(__dadd_rn(__dmul_rn(dx, c.A[0]), __dmul_rn(dy, c.A[1])), __dmul_rn(dz, c.A[2]));
    ry = __dadd_rn(__dadd_rn(__dmul_rn(dx, c.A[3]), __dmul_rn(dy, c.A[4])), __dmul_rn(dz, c.A[5]));
    rz = __dadd_rn(__dadd_rn(__dmul_rn(dx, c.A[6]), __dmul_rn(dy, c.A[7])), __dmul_rn(dz, c.A[8]));
    return __dadd_rn(__dadd_rn(__dmul_rn(rx, rx), __dmul_rn(ry, ry)), __dmul_rn(rz, rz));
}

// errfc (src/functions.f90:28-39): the reference's fitted erfc (Numerical
// Recipes' Chebyshev approximation), selectable for bit-level parity studies.
__device__ __forceinline__ double erfc_fit(double x) {
    double z = fabs(x);
    double t = 1.0 / (1.0 + 0.5 * z);
    double r = t * exp(-z * z - 1.26551223 + t * (1.00002368 + t * (.37409196 + t * (.09678418 +
               t * (-.18628806 + t * (.27886807 + t * (-1.13520398 + t * (1.48851587 +
               t * (-.82215223 + t * .17087277)))))))));
    return x < 0.0 ? 2.0 - r : r;
}

// Inverse factorials 1/m! by the recurrence inv_m = inv_{m-1} / m in IEEE
// double, evaluated at compile time: the values a division loop produces, so
// the damping below is bit-identical to it without a division per term.
struct InvFact {
    double v[17];
    constexpr InvFact() : v() {
        double inv = 1.0;
        v[0] = 1.0;
        for (int m = 1; m < 17; ++m) {
            inv = inv / (double)m;
            v[m] = inv;
        }
    }
};

// Tang-Toennies damping of order k (TT_damping_functions, src/field.f90:3775-3805):
// f = 1 - c e^{-br} sum_{m<=k} (br)^m/m!,  f' = c b e^{-br} (br)^k / k!.
__device__ __forceinline__ void tt_damp_d(double b, double c, double r, int k, double& f, double& fd) {
    constexpr InvFact IF;
    const double br = b * r;
    const double e = exp(-br) * c;
    double term = 1.0, sum = 1.0, inv = 1.0;
    if (k <= 16) {
#pragma unroll
        for (int m = 1; m <= 16; ++m) {
            if (m > k) break;
            inv = IF.v[m];
            term = term * br;
            sum = fma(term, inv, sum);
        }
    } else {
        for (int m = 1; m <= k; ++m) {
            inv = inv / (double)m;
            term = term * br;
            sum = fma(term, inv, sum);
        }
    }
    f = 1.0 - sum * e;
    fd = term * inv * e * b;
}

// Packed two-lane FP32 arithmetic of sm_100 (add / mul / fma .rn.f32x2): a
// 64-bit register holds the pair (lo, hi).
typedef unsigned long long f2p;
__device__ __forceinline__ f2p pk2(float lo, float hi) {
    f2p r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void upk2(f2p v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f2p ffma2(f2p a, f2p b, f2p c) {
    f2p d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ f2p fmul2(f2p a, f2p b) {
    f2p d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2p fadd2(f2p a, f2p b) {
    f2p d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum over a group of G consecutive lanes (G a power of two <= 32); every lane
// of the group receives the group sum.
template <int G>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of K values per thread, written as per-block partials
// out[blockLinear*K + k].  Fixed reduction tree: deterministic.
template <int K>
__device__ __forceinline__ void block_partials(double (&v)[K], double* out) {
    __shared__ double red[32][K];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarp = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = warp_sum(v[k]);
        if (lane == 0) red[warp][k] = s;
    }
    __syncthreads();
    if (warp == 0) {
        const int bl = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double s = lane < nwarp ? red[lane][k] : 0.0;
            s = warp_sum(s);
            if (lane == 0) out[(size_t)bl * K + k] = s;
        }
    }
}

}  // namespace mdff
