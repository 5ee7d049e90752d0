// rmc_var.cuh -- the distance-variance chi^2 of reverse Monte Carlo
// (eval_chisq_var_distance, src/rmc.f90:778-1063) on the device.
//
// The reference, at every trial move, computes for every atom ia and type t
// the distances to all other atoms of type t (minimum image in direct
// coordinates, no cutoff), sorts them, averages the n-th smallest over the
// atoms of each type, and sums (d_n(ia) - <d_n>)^2 / <d_n>^2 -- O(N^2 log N)
// per move.  Here the sorted lists stay resident in device memory between
// moves (one row of Ltot = sum_t natmi(t) doubles per atom, one segment per
// type), and a trial move of atom p changes them incrementally:
//   * p's own segments are recomputed and sorted (one block per segment,
//     bitonic sort in shared memory);
//   * in every other atom's segment of p's type exactly one value changes,
//     d(ja, p_old) -> d(ja, p_new): it is found by binary search and moved to
//     its new rank by shifting the values in between (one warp per atom);
// then the means and chi^2 are formed again from the lists: the means by a
// per-rank sum over 64 ranges of atoms added in order, chi^2 per atom and by
// a fixed tree over the atoms.
#include "common.cuh"

namespace mdff {

constexpr int VAR_MAXSEG = 16384;   // longest segment the block sort handles (128 KB of shared memory)

struct VarSpec {
    int n, ntype, Ltot, nmax;
    int off[MDFF_NTYPE_MAX];     // segment offsets in a row
    int natmi[MDFF_NTYPE_MAX];
};

// segment length of type t in the row of an atom of type ti: natmi(t) - (t == ti)
__device__ __forceinline__ int var_len(const VarSpec& v, int t, int ti) { return v.natmi[t] - (t == ti ? 1 : 0); }

// d(i, j) as the reference forms it: pairvec_exact, then an IEEE sqrt
__device__ __forceinline__ double var_dist(const CellP& c, double a1, double a2, double a3, double b1, double b2,
                                           double b3) {
    double rx, ry, rz;
    return sqrt(pairvec_exact(c, a1, a2, a3, b1, b2, b3, rx, ry, rz));
}

// Distances of every ordered pair into the rows, unsorted: segment t of row
// ia holds the atoms of type t other than ia, in atom order.  rank[ja] = the
// number of atoms of ja's type before ja.  Grid: (ceil(n/256), n); row ia =
// blockIdx.y.
__global__ void k_var_fill(VarSpec v, const double* __restrict__ s, const int* __restrict__ type,
                           const int* __restrict__ rank, CellP c, double* __restrict__ vl) {
    const int ja = blockIdx.x * blockDim.x + threadIdx.x, ia = blockIdx.y;
    const int n = v.n;
    if (ja >= n || ja == ia) return;
    const int tj = type[ja];
    const int pos = rank[ja] - ((type[ia] == tj && ja > ia) ? 1 : 0);
    vl[(size_t)ia * v.Ltot + v.off[tj] + pos] =
        var_dist(c, s[ia], s[n + ia], s[2 * n + ia], s[ja], s[n + ja], s[2 * n + ja]);
}

// Row p only (after p moved): the same values for its own segments.
__global__ void k_var_row(VarSpec v, const double* __restrict__ s, const int* __restrict__ type,
                          const int* __restrict__ rank, CellP c, int p, double* __restrict__ vl) {
    const int ja = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = v.n;
    if (ja >= n || ja == p) return;
    const int tj = type[ja];
    const int pos = rank[ja] - ((type[p] == tj && ja > p) ? 1 : 0);
    vl[(size_t)p * v.Ltot + v.off[tj] + pos] =
        var_dist(c, s[p], s[n + p], s[2 * n + p], s[ja], s[n + ja], s[2 * n + ja]);
}

// Ascending sort of segments, one block (1024 threads) per segment: bitonic
// sort of the segment padded with +inf to P (a power of two, P <= VAR_MAXSEG)
// in shared memory.  Segment b: row = row0 + b / ntype (or the single row
// `one_row` >= 0), type = b % ntype.
__global__ void __launch_bounds__(1024) k_var_sort(VarSpec v, const int* __restrict__ type, int row0, int one_row,
                                                   int P, double* __restrict__ vl) {
    extern __shared__ double sk[];
    const int b = blockIdx.x;
    const int ia = one_row >= 0 ? one_row : row0 + b / v.ntype;
    const int t = b % v.ntype;
    const int len = var_len(v, t, type[ia]);
    double* seg = vl + (size_t)ia * v.Ltot + v.off[t];
    for (int k = threadIdx.x; k < P; k += blockDim.x) sk[k] = k < len ? seg[k] : __longlong_as_double(0x7ff0000000000000ll);
    __syncthreads();
    for (int size = 2; size <= P; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int k = threadIdx.x; k < P / 2; k += blockDim.x) {
                const int lo = 2 * k - (k & (stride - 1));   // index with bit 'stride' clear
                const int hi = lo + stride;
                const bool up = (lo & size) == 0;
                const double a = sk[lo], bb = sk[hi];
                if ((a > bb) == up) { sk[lo] = bb; sk[hi] = a; }
            }
            __syncthreads();
        }
    }
    for (int k = threadIdx.x; k < len; k += blockDim.x) seg[k] = sk[k];
}

// first index in seg[0, len) whose value is >= x
__device__ __forceinline__ int var_lower_bound(const double* seg, int len, double x) {
    int lo = 0, hi = len;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (seg[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// p moved from direct position `from` to `to`: in the segment of p's type of
// every other atom, the value d(ja, from) becomes d(ja, to) and moves to its
// rank.  One warp per atom.  A value that is not found (lists out of step
// with the positions) sets *err.
__global__ void k_var_shift(VarSpec v, const double* __restrict__ s, const int* __restrict__ type, CellP c, int p,
                            double f1, double f2, double f3, double t1, double t2, double t3, double* __restrict__ vl,
                            int* err) {
    const int lane = threadIdx.x & 31;
    const int ja = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int n = v.n;
    if (ja >= n || ja == p) return;
    const int tp = type[p];
    const int len = var_len(v, tp, type[ja]);
    double* seg = vl + (size_t)ja * v.Ltot + v.off[tp];
    const double a1 = s[ja], a2 = s[n + ja], a3 = s[2 * n + ja];
    const double dold = var_dist(c, a1, a2, a3, f1, f2, f3);
    const double dnew = var_dist(c, a1, a2, a3, t1, t2, t3);
    if (dold == dnew) return;
    const int r_old = var_lower_bound(seg, len, dold);
    if (r_old >= len || seg[r_old] != dold) {
        if (lane == 0) atomicOr(err, 1);
        return;
    }
    const int r_ins = var_lower_bound(seg, len, dnew);   // counts the old value when dnew > dold
    if (dnew > dold) {
        // seg[r_old + 1 .. r_ins - 1] one place down, dnew at r_ins - 1
        for (int k = r_old; k < r_ins - 1; k += 32) {
            const int q = k + lane;
            const double val = q < r_ins - 1 ? seg[q + 1] : 0.0;
            __syncwarp();
            if (q < r_ins - 1) seg[q] = val;
            __syncwarp();
        }
        if (lane == 0) seg[r_ins - 1] = dnew;
    } else {
        // seg[r_ins .. r_old - 1] one place up, dnew at r_ins
        for (int k = r_old - 1; k >= r_ins; k -= 32) {
            const int q = k - lane;
            const double val = q >= r_ins ? seg[q] : 0.0;
            __syncwarp();
            if (q >= r_ins) seg[q + 1] = val;
            __syncwarp();
        }
        if (lane == 0) seg[r_ins] = dnew;
    }
}

// dab_aver of the reference: for every list type t2 and rank m, the sum over
// the atoms of each type t1 of their m-th smallest distance to type t2 (zero
// distances left out, as there), divided by natmi(t1).  Pass 1: one thread per
// (t2, m) and range of VAR_NCH atoms (blockIdx.y), atoms in order, partial
// sums psum[(chunk * ntype + t1) * Ltot + off[t2] + m]; pass 2 (k_var_mean_fin)
// adds the chunks in order: mean[(t1 * ntype + t2) * nmax + m].
constexpr int VAR_NCH = 64;
__global__ void k_var_mean(VarSpec v, const int* __restrict__ type, const double* __restrict__ vl,
                           double* __restrict__ psum) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    int t2 = 0, m = g;
    while (t2 < v.ntype && m >= v.natmi[t2]) { m -= v.natmi[t2]; ++t2; }
    if (t2 >= v.ntype) return;
    const int per = (v.n + VAR_NCH - 1) / VAR_NCH;
    const int a0 = blockIdx.y * per, a1 = min(v.n, a0 + per);
    double S[MDFF_NTYPE_MAX];
    for (int t = 0; t < v.ntype; ++t) S[t] = 0.0;
    for (int ia = a0; ia < a1; ++ia) {
        const int t1 = type[ia];
        if (m < var_len(v, t2, t1)) {
            const double d = vl[(size_t)ia * v.Ltot + v.off[t2] + m];
            if (d != 0.0) S[t1] += d;
        }
    }
    for (int t1 = 0; t1 < v.ntype; ++t1) psum[((size_t)blockIdx.y * v.ntype + t1) * v.Ltot + v.off[t2] + m] = S[t1];
}

__global__ void k_var_mean_fin(VarSpec v, const double* __restrict__ psum, double* __restrict__ mean) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    int t2 = 0, m = g;
    while (t2 < v.ntype && m >= v.natmi[t2]) { m -= v.natmi[t2]; ++t2; }
    if (t2 >= v.ntype) return;
    for (int t1 = 0; t1 < v.ntype; ++t1) {
        double S = 0.0;
        for (int ch = 0; ch < VAR_NCH; ++ch) S += psum[((size_t)ch * v.ntype + t1) * v.Ltot + v.off[t2] + m];
        mean[((size_t)t1 * v.ntype + t2) * v.nmax + m] = S / (double)v.natmi[t1];
    }
}

// chi^2 per atom, sum over t2 and ranks with a nonzero mean of
// (d - mean)^2 / mean^2; one warp per atom, block partials for a fixed-order
// tree over the atoms.
__global__ void k_var_chi(VarSpec v, const int* __restrict__ type, const double* __restrict__ vl,
                          const double* __restrict__ mean, double* part) {
    const int lane = threadIdx.x & 31;
    const int ia = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    double acc[1] = {0.0};
    if (ia < v.n) {
        const int t1 = type[ia];
        double c = 0.0;
        for (int t2 = 0; t2 < v.ntype; ++t2) {
            const int len = var_len(v, t2, t1);
            const double* seg = vl + (size_t)ia * v.Ltot + v.off[t2];
            const double* mn = mean + ((size_t)t1 * v.ntype + t2) * v.nmax;
            for (int m = lane; m < len; m += 32) {
                const double a = mn[m];
                if (a != 0.0) {
                    const double dd = seg[m] - a;
                    c += dd * dd / (a * a);
                }
            }
        }
        c = warp_sum(c);
        if (lane == 0) acc[0] = c;
    }
    block_partials<1>(acc, part);
}

}  // namespace mdff
