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
    // diagonal pair and the two off-diagonals that touch r change.  The
    // tangent t = sgn(theta) / (|theta| + sqrt(theta^2 + 1)), theta =
    // h / (2 apq), h = aqq - app, is formed as 2 sgn(theta)|apq| /
    // (|h| + sqrt(h^2 + 4 apq^2)): one division and one square root.
    auto rot = [](double& dp, double& dq, double& opq, double& orp, double& orq) {
        const double apq = opq;
        if (apq == 0.0) return;
        const double h = dq - dp;
        const double num = h > 0.0 ? apq : (h < 0.0 ? -apq : fabs(apq));
        const double t = 2.0 * num / (fabs(h) + sqrt(fma(h, h, 4.0 * apq * apq)));
        const double c = rsqrt(fma(t, t, 1.0)), s = t * c;
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
// statistics accumulated per type row: the 26 sums -- Vzz, |Vzz|, eta, Vzz^2,
// count Vzz >= 0, count, U_k (5), U_k U_l for k <= l (15, row-major upper
// triangle) -- then min Vzz and max Vzz
constexpr int EFG_NSUM = 26;
constexpr int EFG_NACC = 28;
constexpr int EFG_THREADS = 256;
constexpr int EFG_SMEM_BINS = 12288;   // block-private histograms up to 48 KB

struct EfgBins {
    double vzzmin, resvzz, reseta, umin, resu;
    double ivzz, ieta, iu;   // 1 / resvzz, 1 / reseta, 1 / resu
    int PANvzz, PANeta, PANU, PANS, ntype;
    int ov, oe, ou, os, nbins;   // the four histograms in one int array (rows 0..ntype, U1..U5 + U2..U5)
    int cv, ce, cu, cs, ncomp;   // block-private counts: type rows only, U1..U5 only
};

// int(y / res) (truncation toward zero, as the reference's INT of the
// quotient) from the product with the reciprocal: the product is within 3 ulp
// of the quotient, so when it lies farther than 1e-15 of its magnitude from
// the nearest integer both truncate alike; otherwise divide.
__device__ __forceinline__ int bin_trunc(double y, double res, double inv) {
    const double q = y * inv;
    if (fabs(q - rint(q)) > 1e-15 * fabs(q)) return (int)q;
    return (int)(y / res);
}

// Warp sum of 32 values per lane by a butterfly reduce-scatter: after five
// exchange levels lane l holds the sum over the warp of value l (31 shuffles
// instead of 32 x 5; a fixed tree, so the result is deterministic).
__device__ __forceinline__ double warp_reduce_scatter32(double (&v)[32], int lane) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const bool hi = (lane & o) != 0;
#pragma unroll
        for (int j = 0; j < o; ++j) {
            const double send = hi ? v[j] : v[j + o];
            const double keep = hi ? v[j + o] : v[j];
            v[j] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
    return v[0];
}

// Persistent blocks over chunks of EFG_THREADS sites, one site per thread:
// chunk q covers sites (q % nblk) * EFG_THREADS + lane of configuration
// q / nblk.  efg6 [nconf][6][n] (xx yy zz xy xz yz).  DIST: counts into hist
// (SMEM: per type row into block-private shared counts kept over all of the
// block's chunks, the all-sites row and the U2..U5 histogram formed when they
// are flushed once at the end) and per-chunk statistics partials part
// [nconf][nblk][ntype][EFG_NACC] per type; bad |= 1 (U), 2 (S), 4 (Vzz),
// 8 (eta) for a site outside a range (that bin is skipped).  nmr/U/S
// (nullable): per-site outputs [nconf][4|5|1][n].
template <bool DIST, bool SMEM>
__global__ void __launch_bounds__(EFG_THREADS, 3) k_efg_sites(int n, int nblk, int nchunk,
                                                              const double* __restrict__ efg6,
                                                              const int* __restrict__ type, EfgBins b, int* hist,
                                                              double* __restrict__ part, double* __restrict__ nmr_out,
                                                              double* __restrict__ U_out, double* __restrict__ S_out,
                                                              int* bad) {
    extern __shared__ int efg_sh[];
    __shared__ double red[EFG_THREADS / 32][EFG_NACC];
    if (DIST && SMEM) {
        for (int k = threadIdx.x; k < b.ncomp; k += EFG_THREADS) efg_sh[k] = 0;
        __syncthreads();
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int flag = 0;
    for (int q = blockIdx.x; q < nchunk; q += gridDim.x) {
        const int c = q / nblk, bx = q - c * nblk;
        const int i = bx * EFG_THREADS + threadIdx.x;
        const bool live = i < n;
        double u[5] = {0, 0, 0, 0, 0}, r[4] = {0, 0, 0, 0};
        int ty = -1;
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
            ty = type[i];   // 0-based; histogram rows 1..ntype
            if (DIST) {
                const int it = ty + 1, nt1 = b.ntype + 1;
                const int ks = bin_trunc(s, b.resu, b.iu) + 1;
                const int kvzz = bin_trunc(r[2] - b.vzzmin, b.resvzz, b.ivzz) + 1;
                const int keta = bin_trunc(r[3], b.reseta, b.ieta);
                if (SMEM) {
                    for (int ui = 0; ui < 5; ++ui) {
                        const int ku = bin_trunc(u[ui] - b.umin, b.resu, b.iu) + 1;
                        if (ku < 0 || ku > b.PANU) { flag |= 1; continue; }
                        atomicAdd(&efg_sh[b.cu + (ui * b.ntype + ty) * (b.PANU + 1) + ku], 1);
                    }
                    if (ks < 0 || ks > b.PANS) flag |= 2;
                    else atomicAdd(&efg_sh[b.cs + ty * (b.PANS + 1) + ks], 1);
                    if (kvzz < 0 || kvzz > b.PANvzz) flag |= 4;
                    else atomicAdd(&efg_sh[b.cv + ty * (b.PANvzz + 1) + kvzz], 1);
                    if (keta < 0 || keta > b.PANeta) flag |= 8;
                    else atomicAdd(&efg_sh[b.ce + ty * (b.PANeta + 1) + keta], 1);
                } else {
                    for (int ui = 0; ui < 5; ++ui) {
                        const int ku = bin_trunc(u[ui] - b.umin, b.resu, b.iu) + 1;
                        if (ku < 0 || ku > b.PANU) { flag |= 1; continue; }
                        atomicAdd(&hist[b.ou + (ui * nt1 + 0) * (b.PANU + 1) + ku], 1);
                        atomicAdd(&hist[b.ou + (ui * nt1 + it) * (b.PANU + 1) + ku], 1);
                        if (ui != 0) {
                            atomicAdd(&hist[b.ou + (5 * nt1 + 0) * (b.PANU + 1) + ku], 1);
                            atomicAdd(&hist[b.ou + (5 * nt1 + it) * (b.PANU + 1) + ku], 1);
                        }
                    }
                    if (ks < 0 || ks > b.PANS) flag |= 2;
                    else {
                        atomicAdd(&hist[b.os + ks], 1);
                        atomicAdd(&hist[b.os + it * (b.PANS + 1) + ks], 1);
                    }
                    if (kvzz < 0 || kvzz > b.PANvzz) flag |= 4;
                    else {
                        atomicAdd(&hist[b.ov + kvzz], 1);
                        atomicAdd(&hist[b.ov + it * (b.PANvzz + 1) + kvzz], 1);
                    }
                    if (keta < 0 || keta > b.PANeta) flag |= 8;
                    else {
                        atomicAdd(&hist[b.oe + keta], 1);
                        atomicAdd(&hist[b.oe + it * (b.PANeta + 1) + keta], 1);
                    }
                }
            }
        }
        if (!DIST) continue;
        // statistics: per type, the chunk's sums by a fixed tree (types with
        // no site in the chunk write the empty partial without reducing)
        const double vzz = r[2];
        for (int t = 0; t < b.ntype; ++t) {
            const bool in = ty == t;
            double* out = part + (((size_t)c * nblk + bx) * b.ntype + t) * EFG_NACC;
            if (!__syncthreads_or(in)) {
                if (threadIdx.x < EFG_NACC)
                    out[threadIdx.x] = threadIdx.x == 26 ? INFINITY : (threadIdx.x == 27 ? -INFINITY : 0.0);
                continue;
            }
            double v[32];
            v[0] = in ? vzz : 0.0;
            v[1] = in ? fabs(vzz) : 0.0;
            v[2] = in ? r[3] : 0.0;
            v[3] = in ? vzz * vzz : 0.0;
            v[4] = in && vzz >= 0.0 ? 1.0 : 0.0;
            v[5] = in ? 1.0 : 0.0;
            int m = 6;
#pragma unroll
            for (int k = 0; k < 5; ++k) v[m++] = in ? u[k] : 0.0;
#pragma unroll
            for (int k = 0; k < 5; ++k)
#pragma unroll
                for (int l = k; l < 5; ++l) v[m++] = in ? u[k] * u[l] : 0.0;
#pragma unroll
            for (int k = EFG_NSUM; k < 32; ++k) v[k] = 0.0;
            const double sum = warp_reduce_scatter32(v, lane);
            double mn = in ? vzz : INFINITY, mx = in ? vzz : -INFINITY;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
                mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            }
            if (lane < EFG_NSUM) red[warp][lane] = sum;
            if (lane == 0) { red[warp][26] = mn; red[warp][27] = mx; }
            __syncthreads();
            if (threadIdx.x < EFG_NACC) {
                const int k = threadIdx.x;
                double x = red[0][k];
                for (int w = 1; w < EFG_THREADS / 32; ++w)
                    x = k == 26 ? fmin(x, red[w][k]) : (k == 27 ? fmax(x, red[w][k]) : x + red[w][k]);
                out[k] = x;
            }
            __syncthreads();
        }
    }
    if (!DIST) return;
    if (flag) atomicOr(bad, flag);
    if (SMEM) __syncthreads();
    if (SMEM) {
        // flush: global bin k of the full layout from the block's type rows
        const int nt = b.ntype, nt1 = nt + 1;
        for (int k = threadIdx.x; k < b.nbins; k += EFG_THREADS) {
            int base, w, row, hsel = 0;
            if (k < b.oe) { w = b.PANvzz + 1; row = k / w; base = b.cv; }
            else if (k < b.ou) { w = b.PANeta + 1; row = (k - b.oe) / w; base = b.ce; }
            else if (k < b.os) { w = b.PANU + 1; const int q = (k - b.ou) / w; hsel = q / nt1; row = q % nt1; base = b.cu; }
            else { w = b.PANS + 1; row = (k - b.os) / w; base = b.cs; }
            const int bin = (k < b.oe ? k : k < b.ou ? k - b.oe : k < b.os ? k - b.ou : k - b.os) % w;
            int v = 0;
            const int u0 = hsel < 5 ? hsel : 1, u1 = hsel < 5 ? hsel : 4;   // U2..U5 together: histograms 1..4
            for (int uh = u0; uh <= u1; ++uh) {
                const int hb = base + uh * nt * w;   // uh = 0 for the three single histograms
                if (row == 0)
                    for (int t = 0; t < nt; ++t) v += efg_sh[hb + t * w + bin];
                else
                    v += efg_sh[hb + (row - 1) * w + bin];
            }
            if (v) atomicAdd(&hist[k], v);
        }
    }
}

// Sum of a configuration's chunk partials: grid (ntype+1, nconf), one block
// of EFG_THREADS per row; row 0 (all sites) takes every type's partials.
// Thread j sums records j, j + EFG_THREADS, ... of the row's (chunk, type)
// records in order, then a fixed tree (butterfly within warps, warps in order)
// combines the threads: deterministic.  out [nconf][(ntype+1)][EFG_NACC].
__global__ void __launch_bounds__(EFG_THREADS) k_efg_stats_fin(int nblk, int ntype, const double* __restrict__ part,
                                                               double* __restrict__ out) {
    __shared__ double red[EFG_THREADS / 32][EFG_NACC];
    const int row = blockIdx.x, c = blockIdx.y;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int per = row == 0 ? ntype : 1, t0 = row == 0 ? 0 : row - 1;
    const int nrec = nblk * per;
    double v[32];
#pragma unroll
    for (int k = 0; k < 32; ++k) v[k] = 0.0;
    double mn = INFINITY, mx = -INFINITY;
    for (int j = threadIdx.x; j < nrec; j += EFG_THREADS) {
        const int bl = j / per, t = t0 + j % per;
        const double* rec = part + (((size_t)c * nblk + bl) * ntype + t) * EFG_NACC;
#pragma unroll
        for (int k = 0; k < EFG_NSUM; ++k) v[k] += rec[k];
        mn = fmin(mn, rec[26]);
        mx = fmax(mx, rec[27]);
    }
    const double sum = warp_reduce_scatter32(v, lane);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if (lane < EFG_NSUM) red[warp][lane] = sum;
    if (lane == 0) { red[warp][26] = mn; red[warp][27] = mx; }
    __syncthreads();
    if (threadIdx.x < EFG_NACC) {
        const int k = threadIdx.x;
        double x = red[0][k];
        for (int w = 1; w < EFG_THREADS / 32; ++w)
            x = k == 26 ? fmin(x, red[w][k]) : (k == 27 ? fmax(x, red[w][k]) : x + red[w][k]);
        out[((size_t)c * (ntype + 1) + row) * EFG_NACC + k] = x;
    }
}

}  // namespace mdff
