// EFG post-processing on the device: efg_stat (src/efg.f90:2057-2440) with
// nmr_convention (:2546-2650) over a batch of configurations in one pass.
// Per site: the Czjzek components U of the tensor and S = |U|, the principal
// values from a cyclic Jacobi iteration in FP64 (ascending, as DSYEV returns
// them), ordered by the NMR convention |Vzz| >= |Vyy| >= |Vxx| with
// eta = (Vxx - Vyy) / Vzz; then, in the same kernel, the site's bins of the
// Vzz, eta, U and S distributions (block-private shared-memory counts flushed
// with integer atomics: exact and order-free) and its contribution to the
// per-type statistics (block partials by a fixed reduction tree, then a second
// kernel that sums the blocks of a configuration in order).  Each tensor is
// read once (48 bytes per site); per-site outputs are written only on request.
#include "common.cuh"

namespace mdff {

// principal values of the symmetric 3x3 (a00 a11 a22 a01 a02 a12), ascending
__device__ __forceinline__ void sym3_eigvals(double a00, double a11, double a22, double a01, double a02, double a12,
                                             double w[3]) {
    double d0 = a00, d1 = a11, d2 = a22, o01 = a01, o02 = a02, o12 = a12;
    const double nrm = fabs(a00) + fabs(a11) + fabs(a22) + fabs(a01) + fabs(a02) + fabs(a12);
    // one Jacobi rotation zeroing (p, q); r is the remaining index: the
    // diagonal pair and the two off-diagonals that touch r change
    auto rot = [](double& dp, double& dq, double& opq, double& orp, double& orq) {
        const double apq = opq;
        if (apq == 0.0) return;
        const double theta = (dq - dp) / (2.0 * apq);
        const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(fma(theta, theta, 1.0)));
        const double c = 1.0 / sqrt(fma(t, t, 1.0)), s = t * c;
        dp -= t * apq;
        dq += t * apq;
        opq = 0.0;
        const double arp = orp, arq = orq;
        orp = c * arp - s * arq;
        orq = s * arp + c * arq;
    };
    for (int sweep = 0; sweep < 32; ++sweep) {
        const double off = fabs(o01) + fabs(o02) + fabs(o12);
        if (!(off > 1e-17 * nrm)) break;
        rot(d0, d1, o01, o02, o12);   // (0,1), r = 2: a[2][0] = o02, a[2][1] = o12
        rot(d0, d2, o02, o01, o12);   // (0,2), r = 1: a[1][0] = o01, a[1][2] = o12
        rot(d1, d2, o12, o01, o02);   // (1,2), r = 0: a[0][1] = o01, a[0][2] = o02
    }
    double x = d0, y = d1, z = d2, t;
    if (x > y) { t = x; x = y; y = t; }
    if (y > z) { t = y; y = z; z = t; }
    if (x > y) { t = x; x = y; y = t; }
    w[0] = x; w[1] = y; w[2] = z;
}

// nmr_convention (src/efg.f90:2546-2650): nmr = (Vxx, Vyy, Vzz, eta)
__device__ __forceinline__ void nmr_convention_d(const double e[3], double nmr[4]) {
    double diso = (e[0] + e[1] + e[2]) / 3.0;
    if (fabs(diso) != 0.0 && fabs(diso) > 1e-3) diso = 0.0;
    const double a0 = fabs(e[0] - diso), a1 = fabs(e[1] - diso), a2 = fabs(e[2] - diso);
    double d11, d22, d33;
    if (a0 >= a1 && a0 >= a2) {
        d11 = e[0];
        if (a1 >= a2) { d22 = e[1]; d33 = e[2]; } else { d22 = e[2]; d33 = e[1]; }
    } else if (a1 >= a0 && a1 >= a2) {
        d11 = e[1];
        if (a0 >= a2) { d22 = e[0]; d33 = e[2]; } else { d22 = e[2]; d33 = e[0]; }
    } else {
        d11 = e[2];
        if (a0 >= a1) { d22 = e[0]; d33 = e[1]; } else { d22 = e[1]; d33 = e[0]; }
    }
    nmr[0] = d33; nmr[1] = d22; nmr[2] = d11;
    nmr[3] = (nmr[0] - nmr[1]) / nmr[2];
    if (nmr[0] == nmr[1]) nmr[3] = 0.0;
    if (nmr[2] == 0.0) nmr[3] = 0.0;
    if (fabs(nmr[0]) < 1.0e-05 && fabs(nmr[1]) < 1.0e-5 && fabs(nmr[2]) < 1.0e-5) nmr[3] = 0.0;
}

constexpr int EFG_NT_MAX = 16;
// statistics accumulated per type row: sum Vzz, sum |Vzz|, sum eta, sum Vzz^2,
// count Vzz >= 0, count, min Vzz, max Vzz, sum U_k (5), sum U_k U_l for k <= l
// (15, row-major upper triangle)
constexpr int EFG_NACC = 28;
constexpr int EFG_THREADS = 256;
constexpr int EFG_SMEM_BINS = 12288;   // block-private histograms up to 48 KB

struct EfgBins {
    double vzzmin, resvzz, reseta, umin, resu;
    int PANvzz, PANeta, PANU, PANS, ntype;
    int ov, oe, ou, os, nbins;   // offsets of the four histograms in one int array
};

// One site per thread; grid (blocks per configuration, configurations).
// efg6 [nconf][6][n] (xx yy zz xy xz yz).  DIST: bins into hist (through shared
// memory when SMEM) and per-block statistics partials part
// [nconf][gridDim.x][(ntype+1)][EFG_NACC]; bad |= 1 (U), 2 (S), 4 (Vzz), 8 (eta)
// for a site outside a range (that bin is skipped).  nmr/U/S (nullable):
// per-site outputs [nconf][4|5|1][n].
template <bool DIST, bool SMEM>
__global__ void __launch_bounds__(EFG_THREADS) k_efg_sites(int n, const double* __restrict__ efg6,
                                                           const int* __restrict__ type, EfgBins b, int* hist,
                                                           double* __restrict__ part, double* __restrict__ nmr_out,
                                                           double* __restrict__ U_out, double* __restrict__ S_out,
                                                           int* bad) {
    extern __shared__ int efg_sh[];
    const int c = blockIdx.y;
    const int i = blockIdx.x * EFG_THREADS + threadIdx.x;
    const bool live = i < n;
    if (DIST && SMEM) {
        for (int k = threadIdx.x; k < b.nbins; k += EFG_THREADS) efg_sh[k] = 0;
        __syncthreads();
    }
    double u[5] = {0, 0, 0, 0, 0}, r[4] = {0, 0, 0, 0};
    int it = 0;
    if (live) {
        const double* t = efg6 + (size_t)c * 6 * n + i;
        const double xx = t[0], yy = t[(size_t)n], zz = t[(size_t)2 * n];
        const double xy = t[(size_t)3 * n], xz = t[(size_t)4 * n], yz = t[(size_t)5 * n];
        double sq3 = sqrt(3.0);
        sq3 = 1.0 / sq3;
        const double sq32 = sq3 * 0.5;
        u[0] = zz * 0.5; u[1] = xz * sq3; u[2] = yz * sq3; u[3] = xy * sq3; u[4] = (xx - yy) * sq32;
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < 5; ++k) s = s + u[k] * u[k];
        s = sqrt(s);
        double w[3];
        sym3_eigvals(xx, yy, zz, xy, xz, yz, w);
        nmr_convention_d(w, r);
        if (nmr_out) {
#pragma unroll
            for (int k = 0; k < 4; ++k) nmr_out[((size_t)c * 4 + k) * n + i] = r[k];
        }
        if (U_out) {
#pragma unroll
            for (int k = 0; k < 5; ++k) U_out[((size_t)c * 5 + k) * n + i] = u[k];
        }
        if (S_out) S_out[(size_t)c * n + i] = s;
        it = type[i] + 1;   // engine types are 0-based, rows 1..ntype
        if (DIST) {
            int* h = SMEM ? efg_sh : hist;
            const int nt1 = b.ntype + 1;
            int flag = 0;
            for (int ui = 0; ui < 5; ++ui) {
                const int ku = (int)((u[ui] - b.umin) / b.resu) + 1;
                if (ku < 0 || ku > b.PANU) { flag |= 1; continue; }
                atomicAdd(&h[b.ou + (ui * nt1 + 0) * (b.PANU + 1) + ku], 1);
                atomicAdd(&h[b.ou + (ui * nt1 + it) * (b.PANU + 1) + ku], 1);
                if (ui != 0) {
                    atomicAdd(&h[b.ou + (5 * nt1 + 0) * (b.PANU + 1) + ku], 1);
                    atomicAdd(&h[b.ou + (5 * nt1 + it) * (b.PANU + 1) + ku], 1);
                }
            }
            const int ks = (int)(s / b.resu) + 1;
            if (ks < 0 || ks > b.PANS) flag |= 2;
            else {
                atomicAdd(&h[b.os + ks], 1);
                atomicAdd(&h[b.os + it * (b.PANS + 1) + ks], 1);
            }
            const int kvzz = (int)((r[2] - b.vzzmin) / b.resvzz) + 1;
            const int keta = (int)(r[3] / b.reseta);
            if (kvzz < 0 || kvzz > b.PANvzz) flag |= 4;
            else {
                atomicAdd(&h[b.ov + kvzz], 1);
                atomicAdd(&h[b.ov + it * (b.PANvzz + 1) + kvzz], 1);
            }
            if (keta < 0 || keta > b.PANeta) flag |= 8;
            else {
                atomicAdd(&h[b.oe + keta], 1);
                atomicAdd(&h[b.oe + it * (b.PANeta + 1) + keta], 1);
            }
            if (flag) atomicOr(bad, flag);
        }
    }
    if (!DIST) return;
    // statistics: for each row, the block's masked sums by a fixed tree
    __shared__ double red[EFG_THREADS / 32][EFG_NACC];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nt1 = b.ntype + 1;
    const double vzz = r[2];
    for (int row = 0; row < nt1; ++row) {
        const bool in = live && (row == 0 || row == it);
        double v[EFG_NACC];
        v[0] = in ? vzz : 0.0;
        v[1] = in ? fabs(vzz) : 0.0;
        v[2] = in ? r[3] : 0.0;
        v[3] = in ? vzz * vzz : 0.0;
        v[4] = in && vzz >= 0.0 ? 1.0 : 0.0;
        v[5] = in ? 1.0 : 0.0;
        v[6] = in ? vzz : INFINITY;
        v[7] = in ? vzz : -INFINITY;
        int m = 8;
#pragma unroll
        for (int k = 0; k < 5; ++k) v[m++] = in ? u[k] : 0.0;
#pragma unroll
        for (int k = 0; k < 5; ++k)
#pragma unroll
            for (int l = k; l < 5; ++l) v[m++] = in ? u[k] * u[l] : 0.0;
#pragma unroll
        for (int k = 0; k < EFG_NACC; ++k) {
            double x = v[k];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double y = __shfl_xor_sync(0xffffffffu, x, o);
                x = k == 6 ? fmin(x, y) : (k == 7 ? fmax(x, y) : x + y);
            }
            if (lane == 0) red[warp][k] = x;
        }
        __syncthreads();
        if (threadIdx.x < EFG_NACC) {
            const int k = threadIdx.x;
            double x = red[0][k];
            for (int w = 1; w < EFG_THREADS / 32; ++w)
                x = k == 6 ? fmin(x, red[w][k]) : (k == 7 ? fmax(x, red[w][k]) : x + red[w][k]);
            part[(((size_t)c * gridDim.x + blockIdx.x) * nt1 + row) * EFG_NACC + k] = x;
        }
        __syncthreads();
    }
    if (SMEM) {
        for (int k = threadIdx.x; k < b.nbins; k += EFG_THREADS) {
            const int v = efg_sh[k];
            if (v) atomicAdd(&hist[k], v);
        }
    }
}

// Sum of a configuration's block partials in block order: grid (ntype+1,
// nconf), one lane per accumulated quantity; out [nconf][(ntype+1)][EFG_NACC].
__global__ void k_efg_stats_fin(int nblk, const double* __restrict__ part, double* __restrict__ out) {
    const int t = blockIdx.x, c = blockIdx.y, nt1 = gridDim.x, k = threadIdx.x;
    if (k >= EFG_NACC) return;
    double x = k == 6 ? INFINITY : (k == 7 ? -INFINITY : 0.0);
    for (int bl = 0; bl < nblk; ++bl) {
        const double y = part[(((size_t)c * nblk + bl) * nt1 + t) * EFG_NACC + k];
        x = k == 6 ? fmin(x, y) : (k == 7 ? fmax(x, y) : x + y);
    }
    out[((size_t)c * nt1 + t) * EFG_NACC + k] = x;
}

}  // namespace mdff
