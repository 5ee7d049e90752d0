// EFG post-processing on the device: efg_stat's per-site part (src/efg.f90:
// 2225-2270) and distributions (:2344-2440), with nmr_convention
// (:2546-2650).  Per site: the Czjzek components U of the traceless tensor
// and S = |U|, the principal values (ascending, as DSYEV returns them) from a
// cyclic Jacobi iteration in FP64, ordered by the NMR convention
// |Vzz| >= |Vyy| >= |Vxx| with eta = (Vxx - Vyy) / Vzz; then integer
// histograms of Vzz, eta, U and S per type (atomic integer counts, exact) and
// per-block partial sums and extrema for the per-type statistics.
#include "common.cuh"

namespace mdff {

// principal values of the symmetric 3x3 (a00 a11 a22 a01 a02 a12), ascending
__device__ __forceinline__ void sym3_eigvals(double a00, double a11, double a22, double a01, double a02, double a12,
                                             double w[3]) {
    double a[3][3] = {{a00, a01, a02}, {a01, a11, a12}, {a02, a12, a22}};
    const double nrm = fabs(a00) + fabs(a11) + fabs(a22) + fabs(a01) + fabs(a02) + fabs(a12);
    for (int sweep = 0; sweep < 32; ++sweep) {
        const double off = fabs(a[0][1]) + fabs(a[0][2]) + fabs(a[1][2]);
        if (!(off > 1e-17 * nrm)) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                const double apq = a[p][q];
                if (apq == 0.0) continue;
                const double theta = (a[q][q] - a[p][p]) / (2.0 * apq);
                const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                a[p][p] -= t * apq;
                a[q][q] += t * apq;
                a[p][q] = a[q][p] = 0.0;
                const int r = 3 - p - q;
                const double arp = a[r][p], arq = a[r][q];
                a[r][p] = a[p][r] = c * arp - s * arq;
                a[r][q] = a[q][r] = s * arp + c * arq;
            }
    }
    double x = a[0][0], y = a[1][1], z = a[2][2], t;
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

// per site: nmr[4][n], U[5][n], S[n] from the tensors efg6[6][n] (xx yy zz xy xz yz)
__global__ void k_efg_nmr(int n, const double* __restrict__ efg6, double* __restrict__ nmr, double* __restrict__ U,
                          double* __restrict__ S) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double xx = efg6[i], yy = efg6[(size_t)n + i], zz = efg6[(size_t)2 * n + i];
    const double xy = efg6[(size_t)3 * n + i], xz = efg6[(size_t)4 * n + i], yz = efg6[(size_t)5 * n + i];
    double sq3 = sqrt(3.0);
    sq3 = 1.0 / sq3;
    const double sq32 = sq3 * 0.5;
    const double u[5] = {zz * 0.5, xz * sq3, yz * sq3, xy * sq3, (xx - yy) * sq32};
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        U[(size_t)k * n + i] = u[k];
        s = s + u[k] * u[k];
    }
    S[i] = sqrt(s);
    double w[3], r[4];
    sym3_eigvals(xx, yy, zz, xy, xz, yz, w);
    nmr_convention_d(w, r);
#pragma unroll
    for (int k = 0; k < 4; ++k) nmr[(size_t)k * n + i] = r[k];
}

struct EfgBins {
    double vzzmin, resvzz, reseta, umin, resu;
    int PANvzz, PANeta, PANU, PANS, ntype;
};

// distributions (:2344-2440): counts per type (0 = all sites) -- dib_vzz
// [(ntype+1)][PANvzz+1], dib_eta [(ntype+1)][PANeta+1], dib_u [6][(ntype+1)][PANU+1]
// (U1..U5 and all of U2..U5), dib_s [(ntype+1)][PANS+1]; out-of-range sites set *bad.
__global__ void k_efg_dist(int n, const int* __restrict__ type, const double* __restrict__ nmr,
                           const double* __restrict__ U, const double* __restrict__ S, EfgBins b, int* dib_vzz,
                           int* dib_eta, int* dib_u, int* dib_s, int* bad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int it = type[i] + 1;     // engine types are 0-based, histogram rows 1..ntype
    const int nt1 = b.ntype + 1;
    for (int ui = 0; ui < 5; ++ui) {
        const double uk = (U[(size_t)ui * n + i] - b.umin) / b.resu;
        const int ku = (int)uk + 1;
        if (ku < 0 || ku > b.PANU) { atomicOr(bad, 1); continue; }
        atomicAdd(&dib_u[((size_t)ui * nt1 + 0) * (b.PANU + 1) + ku], 1);
        atomicAdd(&dib_u[((size_t)ui * nt1 + it) * (b.PANU + 1) + ku], 1);
        if (ui != 0) {
            atomicAdd(&dib_u[((size_t)5 * nt1 + 0) * (b.PANU + 1) + ku], 1);
            atomicAdd(&dib_u[((size_t)5 * nt1 + it) * (b.PANU + 1) + ku], 1);
        }
    }
    const int ks = (int)(S[i] / b.resu) + 1;
    if (ks < 0 || ks > b.PANS) atomicOr(bad, 2);
    else {
        atomicAdd(&dib_s[(size_t)0 * (b.PANS + 1) + ks], 1);
        atomicAdd(&dib_s[(size_t)it * (b.PANS + 1) + ks], 1);
    }
    const int kvzz = (int)((nmr[(size_t)2 * n + i] - b.vzzmin) / b.resvzz) + 1;
    const int keta = (int)(nmr[(size_t)3 * n + i] / b.reseta);
    if (kvzz < 0 || kvzz > b.PANvzz) atomicOr(bad, 4);
    else {
        atomicAdd(&dib_vzz[(size_t)0 * (b.PANvzz + 1) + kvzz], 1);
        atomicAdd(&dib_vzz[(size_t)it * (b.PANvzz + 1) + kvzz], 1);
    }
    if (keta < 0 || keta > b.PANeta) atomicOr(bad, 8);
    else {
        atomicAdd(&dib_eta[(size_t)0 * (b.PANeta + 1) + keta], 1);
        atomicAdd(&dib_eta[(size_t)it * (b.PANeta + 1) + keta], 1);
    }
}

// per-block partials of the statistics (:2246-2330): for each type row
// t = 0..ntype: sum Vzz, sum |Vzz|, sum eta, sum Vzz^2, count Vzz >= 0, count,
// min Vzz, max Vzz, then sum U_k (5) and sum U_k U_l for k <= l (15, row-major
// upper triangle); out[block][(ntype+1)][EFG_NACC]
constexpr int EFG_NT_MAX = 16;
constexpr int EFG_NACC = 28;
__global__ void __launch_bounds__(256) k_efg_stats(int n, int ntype, const int* __restrict__ type,
                                                   const double* __restrict__ nmr, const double* __restrict__ U,
                                                   double* __restrict__ out) {
    __shared__ double acc[EFG_NT_MAX + 1][EFG_NACC];
    const int nt1 = ntype + 1;
    for (int t = threadIdx.x; t < nt1 * EFG_NACC; t += blockDim.x) {
        const int k = t % EFG_NACC;
        acc[t / EFG_NACC][k] = k == 6 ? 1e300 : (k == 7 ? -1e300 : 0.0);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        // one thread per block walks its sites in order: a fixed summation order
        const int i0 = blockIdx.x * blockDim.x, i1 = min(n, i0 + (int)blockDim.x);
        for (int i = i0; i < i1; ++i) {
            const double vzz = nmr[(size_t)2 * n + i], eta = nmr[(size_t)3 * n + i];
            double u[5];
            for (int k = 0; k < 5; ++k) u[k] = U[(size_t)k * n + i];
            const int rows[2] = {0, type[i] + 1};
            for (int rr = 0; rr < 2; ++rr) {
                double* a = acc[rows[rr]];
                a[0] += vzz;
                a[1] += fabs(vzz);
                a[2] += eta;
                a[3] += vzz * vzz;
                a[4] += vzz >= 0.0 ? 1.0 : 0.0;
                a[5] += 1.0;
                a[6] = fmin(a[6], vzz);
                a[7] = fmax(a[7], vzz);
                int m = 8;
                for (int k = 0; k < 5; ++k) a[m++] += u[k];
                for (int k = 0; k < 5; ++k)
                    for (int l = k; l < 5; ++l) a[m++] += u[k] * u[l];
            }
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < nt1 * EFG_NACC; t += blockDim.x)
        out[(size_t)blockIdx.x * nt1 * EFG_NACC + t] = acc[t / EFG_NACC][t % EFG_NACC];
}

}  // namespace mdff
