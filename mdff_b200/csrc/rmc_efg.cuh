// The EFG terms of reverse Monte Carlo: rmc_efg (src/rmc.f90:1499-1660) and
// the g(r) change of one trial move.  Each trial configuration's EFG comes
// from the engine's own Ewald evaluation; these kernels turn it into the
// integer histograms of rmc_efg (Vzz, eta, and the Czjzek U1..U5 with the
// U2..U5 row), whose normalisation and chi^2 run on the host in the
// reference's order.
#pragma once
// Included by engine.cu after common.cuh, rmc.cuh and efg_post.cuh
// (rmc_bin, sym3_eigvals, nmr_convention_d).

namespace mdff {

struct RmcEfgSpec {
    int ntype, PANU, PANvzz, PANeta;
    int offeta, offU;          // int offsets of the eta and U blocks in the counts
    double cu;                 // coul_unit: the engine's tensors carry it, rmc_efg's do not
    double umin, resu, vzzmin, resvzz, reseta;
    double sq3, sq32;          // 1/sqrt(3) and half of it, as rmc_efg forms them
};

// counts: vzz [ntype+1][PANvzz+1], then eta [ntype+1][PANeta+1], then
// U [6][ntype+1][PANU+1] (rows 0..4 U1..U5, row 5 the U2..U5 pool).  A site
// whose Vzz or eta bin is out of range is skipped whole (the reference's
// cycle), an out-of-range U bin only for that component.  Fortran's INT
// truncates toward zero, so bin = INT(x) + 1 lies in [0, PAN] exactly when
// x is in (-2, PAN), and INT(x) in [0, PAN] when x is in (-1, PAN + 1).
__global__ void k_rmc_efg_hist(int n, const double* __restrict__ efg6, const int* __restrict__ type, RmcEfgSpec sp,
                               int* __restrict__ cnt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) v[c] = __ddiv_rn(efg6[(size_t)c * n + i], sp.cu);   // xx yy zz xy xz yz
    double w[3], nmr[4];
    sym3_eigvals(v[0], v[1], v[2], v[3], v[4], v[5], w);
    nmr_convention_d(w, nmr);
    const double vzzk = __ddiv_rn(nmr[2] - sp.vzzmin, sp.resvzz);
    const double etak = __ddiv_rn(nmr[3], sp.reseta);
    if (!(vzzk > -2.0 && vzzk < (double)sp.PANvzz)) return;
    if (!(etak > -1.0 && etak < (double)sp.PANeta + 1.0)) return;
    const int kvzz = (int)vzzk + 1, keta = (int)etak;
    const int t = type[i] + 1;
    const int wv = sp.PANvzz + 1, we = sp.PANeta + 1, wu = sp.PANU + 1;
    atomicAdd(&cnt[kvzz], 1);
    atomicAdd(&cnt[t * wv + kvzz], 1);
    atomicAdd(&cnt[sp.offeta + keta], 1);
    atomicAdd(&cnt[sp.offeta + t * we + keta], 1);
    if (sp.PANU < 0) return;   // U terms off
    const double U[5] = {__dmul_rn(v[2], 0.5), __dmul_rn(v[4], sp.sq3), __dmul_rn(v[5], sp.sq3),
                         __dmul_rn(v[3], sp.sq3), __dmul_rn(__dsub_rn(v[0], v[1]), sp.sq32)};
    const int rows = sp.ntype + 1;
#pragma unroll
    for (int ui = 0; ui < 5; ++ui) {
        const double uk = __ddiv_rn(U[ui] - sp.umin, sp.resu);
        if (!(uk > -2.0 && uk < (double)sp.PANU)) continue;
        const int ku = (int)uk + 1;
        atomicAdd(&cnt[sp.offU + (ui * rows) * wu + ku], 1);
        atomicAdd(&cnt[sp.offU + (ui * rows + t) * wu + ku], 1);
        if (ui != 0) {   // the pooled U2..U5 row; the reference's loop covers types 1 and 2
            atomicAdd(&cnt[sp.offU + (5 * rows) * wu + ku], 1);
            if (t <= 2) atomicAdd(&cnt[sp.offU + (5 * rows + t) * wu + ku], 1);
        }
    }
}

// The g(r) count change of moving atom p from sold to its current s: pairs
// (p, j) and (j, p) leave their old bin and enter the new one (row 0 twice,
// the two ordered type rows once each), as gr_main counts ordered pairs
__global__ void k_rmc_grdelta(int n, const double* __restrict__ s, const int* __restrict__ type, CellP c, RmcBin k,
                              int p, double o1, double o2, double o3, int* __restrict__ dh) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n || j == p) return;
    const double sj1 = s[j], sj2 = s[(size_t)n + j], sj3 = s[2 * (size_t)n + j];
    const int bo = rmc_bin(c, k, o1, o2, o3, sj1, sj2, sj3);
    const int bn = rmc_bin(c, k, s[p], s[(size_t)n + p], s[2 * (size_t)n + p], sj1, sj2, sj3);
    if (bo == bn) return;
    const int tp = type[p], tj = type[j];
    const int r1 = 1 + tp * k.ntype + tj, r2 = 1 + tj * k.ntype + tp;
    if (bo >= 0) {
        atomicAdd(&dh[bo], -2);
        atomicAdd(&dh[r1 * k.nbins + bo], -1);
        atomicAdd(&dh[r2 * k.nbins + bo], -1);
    }
    if (bn >= 0) {
        atomicAdd(&dh[bn], 2);
        atomicAdd(&dh[r1 * k.nbins + bn], 1);
        atomicAdd(&dh[r2 * k.nbins + bn], 1);
    }
}

// s[p] = (a, b, d) and its Cartesian position, dirkar as k_rmc_dirkar forms it
__global__ void k_rmc_place(int n, double* s, int p, double a, double b, double d, CellP c, double* x, double* y,
                            double* z) {
    s[p] = a;
    s[(size_t)n + p] = b;
    s[2 * (size_t)n + p] = d;
    x[p] = __dadd_rn(__dadd_rn(__dmul_rn(a, c.A[0]), __dmul_rn(b, c.A[1])), __dmul_rn(d, c.A[2]));
    y[p] = __dadd_rn(__dadd_rn(__dmul_rn(a, c.A[3]), __dmul_rn(b, c.A[4])), __dmul_rn(d, c.A[5]));
    z[p] = __dadd_rn(__dadd_rn(__dmul_rn(a, c.A[6]), __dmul_rn(b, c.A[7])), __dmul_rn(d, c.A[8]));
}

}  // namespace mdff
