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

// erfc(x) = e^{-x^2} erfcx(x) for 0 <= x < 4.5: erfcx from Chebyshev
// interpolants of degree 13 on the intervals [j/2, j/2 + 1/2) in the variable
// t = 4x - (2j + 1), fitted in 50-digit arithmetic to erfc(x) e^{x^2}
// (mdff_b200/csrc/fit_erfcx.py; relative error 2.1e-16 in FP64 Horner; the
// caller's e^{-x^2} from a rounded x^2 adds x^2 2^-53).  The Ewald kernels already hold
// e^{-x^2} for the F1, F2, F3 terms, so erfc costs one short polynomial
// instead of a second exponential; outside the range CUDA's erfc is used.
static __device__ const double c_erfcx[9][14] = {
    {7.70346547730996756e-01, -1.85801473307503545e-01, 3.65340671514658918e-02, -6.21947525650125982e-03, 9.47330996756585606e-04, -1.31803606497923632e-04, 1.69901537299267292e-05, -2.05024020381396702e-06, 2.33436817177143440e-07, -2.52334468554404523e-08, 2.60156149536226003e-09, -2.57085438111745281e-10, 2.51350646707265604e-11, -2.29821709880457116e-12},
    {5.06937650293144859e-01, -9.19931729139488452e-02, 1.44348832219559353e-02, -2.02868846867000109e-03, 2.60900556751622560e-04, -3.11496699608856403e-05, 3.48857387321987062e-06, -3.69356217759792109e-07, 3.71954508963358907e-08, -3.58014382507898332e-09, 3.30604355650140892e-10, -2.94034891475697202e-11, 2.58559936735718299e-12, -2.14632892795784933e-13},
    {3.67822916452361093e-01, -5.22054689911524636e-02, 6.67472321853740305e-03, -7.84660537436054168e-04, 8.59818916052587423e-05, -8.86877698531245982e-06, 8.67458470381664333e-07, -8.09193681174837838e-08, 7.23221894249489450e-09, -6.21643528409241565e-10, 5.15412474490585635e-11, -4.13452607511939099e-12, 3.27926983823084055e-13, -2.47519717076794981e-14},
    {2.84972234737436381e-01, -3.27440863786212996e-02, 3.48522688044295174e-03, -3.47812425646692449e-04, 3.28293719036726057e-05, -2.95017055803526819e-06, 2.53712041346902825e-07, -2.09676118887175310e-08, 1.67091885632935495e-09, -1.28766511175265426e-10, 9.61830013285077280e-12, -6.98001921004776969e-13, 5.01063442740550835e-14, -3.44680733141451377e-15},
    {2.31087258730391876e-01, -2.21216257021872899e-02, 1.99953921316914102e-03, -1.71907199319375708e-04, 1.41367006029679316e-05, -1.11692234731851606e-06, 8.50916557327824941e-08, -6.26959723619244137e-09, 4.47895124260412718e-10, -3.10908701084346323e-11, 2.10079779348219243e-12, -1.38423675468731790e-13, 9.02856510000448546e-15, -5.67644798347723846e-16},
    {1.93662096279068691e-01, -1.58094093901587109e-02, 1.23491206170767902e-03, -9.27240296405933807e-05, 6.71711673941216822e-06, -4.70893637676876642e-07, 3.20268067630822385e-08, -2.11783505684827448e-09, 1.36415975435179089e-10, -8.57305040538626970e-12, 5.26375692093561092e-13, -3.16187314717068093e-14, 1.88160922717910673e-15, -1.08476556603290315e-16},
    {1.66335348426821877e-01, -1.17998505802925941e-02, 8.08580680188634841e-04, -5.36792390766808417e-05, 3.46095538099348485e-06, -2.17170478094227272e-07, 1.32862326187598925e-08, -7.93740250497401040e-10, 4.63689003375204657e-11, -2.65200852373283976e-12, 1.48653925733325675e-13, -8.17503930574837552e-15, 4.45764831070709062e-16, -2.36471931146022244e-17},
    {1.45589721275038553e-01, -9.11406438318088270e-03, 5.54922220457831146e-04, -3.29262948463923468e-05, 1.90711868006086389e-06, -1.07987866137007266e-07, 5.98543099979860756e-09, -3.25114305970638778e-10, 1.73236948280893169e-11, -9.06373617437550905e-13, 4.65997853503172364e-14, -2.35626153976442944e-15, 1.18228113910100869e-16, -5.79197552373421933e-18},
    {1.29345274785987924e-01, -7.23608285365383297e-03, 3.95741642117046835e-04, -2.11864557360015355e-05, 1.11162170640691086e-06, -5.72221681771075831e-08, 2.89260098733738314e-09, -1.43713417692772748e-10, 7.02301408394134694e-12, -3.37808096316975056e-13, 1.60031161014207372e-14, -7.47136752260601365e-16, 3.46405779482777296e-17, -1.57285591596023904e-18}};
__device__ __forceinline__ double erfc_ex2(double x, double ex2) {
    if (!(x >= 0.0 && x < 4.5)) return erfc(x);
    const int j = (int)(x * 2.0);
    const double t = fma(x, 4.0, -(double)(2 * j + 1));
    const double* c = c_erfcx[j];
    double p = __ldg(c + 13);
#pragma unroll
    for (int k = 12; k >= 0; --k) p = fma(p, t, __ldg(c + k));
    return ex2 * p;
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
