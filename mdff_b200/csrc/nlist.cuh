// nlist.cu -- Verlet-list construction and the skin check on the GPU.
//
// Replaces vnlist_pbc / vnlistcheck (src/tools.f90:274-535).  The reference
// tests all N^2 pairs; here atoms are binned into cells at least one list
// radius wide and each atom tests only the atoms of its neighbouring cells.
// The inclusion test itself is the reference's FP64 expression evaluated in
// its exact operation order (pairvec_exact), so the lists are bit-identical;
// the cell pruning only skips pairs that are provably farther apart than the
// list radius.
#include "common.cuh"

namespace mdff {

// kardir (src/lattice.f90:183-222), one atom per thread, exact operation order.
__global__ void k_frac(int n, const double* __restrict__ x, const double* __restrict__ y,
                       const double* __restrict__ z, CellP c, double* sx, double* sy, double* sz) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double X = x[i], Y = y[i], Z = z[i];
    sx[i] = __dadd_rn(__dadd_rn(__dmul_rn(X, c.B[0]), __dmul_rn(Y, c.B[3])), __dmul_rn(Z, c.B[6]));
    sy[i] = __dadd_rn(__dadd_rn(__dmul_rn(X, c.B[1]), __dmul_rn(Y, c.B[4])), __dmul_rn(Z, c.B[7]));
    sz[i] = __dadd_rn(__dadd_rn(__dmul_rn(X, c.B[2]), __dmul_rn(Y, c.B[5])), __dmul_rn(Z, c.B[8]));
}

void launch_frac(cudaStream_t st, int n, const double* x, const double* y, const double* z, CellP c,
                 double* sx, double* sy, double* sz) {
    k_frac<<<(n + 255) / 256, 256, 0, st>>>(n, x, y, z, c, sx, sy, sz);
}

// read_pos.f90:148-150: kardir, periodicbc (x - NINT(x)), dirkar, in place.
__global__ void k_wrap(int n, double* x, double* y, double* z, CellP c) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double X = x[i], Y = y[i], Z = z[i];
    double s1 = __dadd_rn(__dadd_rn(__dmul_rn(X, c.B[0]), __dmul_rn(Y, c.B[3])), __dmul_rn(Z, c.B[6]));
    double s2 = __dadd_rn(__dadd_rn(__dmul_rn(X, c.B[1]), __dmul_rn(Y, c.B[4])), __dmul_rn(Z, c.B[7]));
    double s3 = __dadd_rn(__dadd_rn(__dmul_rn(X, c.B[2]), __dmul_rn(Y, c.B[5])), __dmul_rn(Z, c.B[8]));
    s1 = __dsub_rn(s1, round(s1));
    s2 = __dsub_rn(s2, round(s2));
    s3 = __dsub_rn(s3, round(s3));
    x[i] = __dadd_rn(__dadd_rn(__dmul_rn(s1, c.A[0]), __dmul_rn(s2, c.A[1])), __dmul_rn(s3, c.A[2]));
    y[i] = __dadd_rn(__dadd_rn(__dmul_rn(s1, c.A[3]), __dmul_rn(s2, c.A[4])), __dmul_rn(s3, c.A[5]));
    z[i] = __dadd_rn(__dadd_rn(__dmul_rn(s1, c.A[6]), __dmul_rn(s2, c.A[7])), __dmul_rn(s3, c.A[8]));
}

void launch_wrap_positions(cudaStream_t st, int n, double* x, double* y, double* z, CellP c) {
    k_wrap<<<(n + 255) / 256, 256, 0, st>>>(n, x, y, z, c);
}

// ---------------------------------------------------------------- binning --
__device__ __forceinline__ int cell_coord(double s, int nc) {
    double w = s - floor(s);              // [0,1)
    int k = (int)(w * nc);
    return k < 0 ? 0 : (k >= nc ? nc - 1 : k);
}

__global__ void k_bin_count(int n, const double* sx, const double* sy, const double* sz, int nc0, int nc1,
                            int nc2, int* cell_of, int* count) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = (cell_coord(sx[i], nc0) * nc1 + cell_coord(sy[i], nc1)) * nc2 + cell_coord(sz[i], nc2);
    cell_of[i] = c;
    atomicAdd(&count[c], 1);
}

// Exclusive scan of the cell counts in one block (ncell is small: the box
// volume over the list-radius cube).
__global__ void k_scan(int ncell, const int* count, int* start, int* cursor) {
    __shared__ int carry;
    __shared__ int warp_tot[32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < ncell; base += blockDim.x) {
        int i = base + threadIdx.x;
        int v = i < ncell ? count[i] : 0;
        int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += t;
        }
        if (lane == 31) warp_tot[warp] = x;
        __syncthreads();
        if (warp == 0) {
            int w = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0;
            int y = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int t = __shfl_up_sync(0xffffffffu, y, o);
                if (lane >= o) y += t;
            }
            warp_tot[lane] = y - w;
        }
        __syncthreads();
        int excl = carry + warp_tot[warp] + x - v;
        if (i < ncell) { start[i] = excl; cursor[i] = excl; }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) start[ncell] = carry;
}

__global__ void k_bin_fill(int n, const int* cell_of, int* cursor, int* atoms) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int slot = atomicAdd(&cursor[cell_of[i]], 1);
    atoms[slot] = i;
}

// Atomic fill leaves an arbitrary order inside each cell; sort each cell's
// atoms by index so that the list layout is deterministic.  One block per
// cell: the cell's atoms are staged in shared memory and each element is
// written to its rank (the number of smaller indices; indices are distinct).
// A cell of more than SORT_CAP atoms is sorted by one thread (insertion).
constexpr int SORT_CAP = 4096;
__global__ void k_sort_cells(int ncell, const int* __restrict__ start, int* atoms) {
    __shared__ int s_at[SORT_CAP];
    const int c = blockIdx.x;
    if (c >= ncell) return;
    const int b = start[c], e = start[c + 1], m = e - b;
    if (m <= SORT_CAP) {
        for (int t = threadIdx.x; t < m; t += blockDim.x) s_at[t] = atoms[b + t];
        __syncthreads();
        for (int t = threadIdx.x; t < m; t += blockDim.x) {
            const int v = s_at[t];
            int r = 0;
            for (int k = 0; k < m; ++k) r += s_at[k] < v;
            atoms[b + r] = v;
        }
        return;
    }
    if (threadIdx.x != 0) return;
    for (int k = b + 1; k < e; ++k) {
        int v = atoms[k];
        int q = k - 1;
        while (q >= b && atoms[q] > v) { atoms[q + 1] = atoms[q]; --q; }
        atoms[q + 1] = v;
    }
}

// The list kernel's prefilter input, in cell order: the wrapped fractional
// coordinates s - floor(s) rounded to FP32, and the atom index as bits, so a
// warp reads 32 candidates with one coalesced 16-byte load each.
__global__ void k_cell_coords(int n, const double* __restrict__ sx, const double* __restrict__ sy,
                              const double* __restrict__ sz, const int* __restrict__ cell_atoms, float4* cw) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int j = cell_atoms[k];
    const double a = sx[j], b = sy[j], c = sz[j];
    cw[k] = make_float4((float)(a - floor(a)), (float)(b - floor(b)), (float)(c - floor(c)), __int_as_float(j));
}

void launch_bin(cudaStream_t st, int n, const double* sx, const double* sy, const double* sz, CellGrid& g) {
    cudaMemsetAsync(g.cell_count, 0, sizeof(int) * g.ncell, st);
    k_bin_count<<<(n + 255) / 256, 256, 0, st>>>(n, sx, sy, sz, g.nc[0], g.nc[1], g.nc[2], g.cell_of, g.cell_count);
    k_scan<<<1, 1024, 0, st>>>(g.ncell, g.cell_count, g.cell_start, g.cell_cursor);
    k_bin_fill<<<(n + 255) / 256, 256, 0, st>>>(n, g.cell_of, g.cell_cursor, g.cell_atoms);
    k_sort_cells<<<g.ncell, 128, 0, st>>>(g.ncell, g.cell_start, g.cell_atoms);
    k_cell_coords<<<(n + 255) / 256, 256, 0, st>>>(n, sx, sy, sz, g.cell_atoms, g.cell_w);
}

// ------------------------------------------------------------ list build --
// One warp per atom i.  The neighbouring cells are visited in a fixed order;
// along a direction with fewer than three cells every cell is visited once
// (no duplicates).  Candidates j are read 32 at a time from the cell-ordered
// FP32 copy and prefiltered in FP32: a candidate is dropped only when its
// FP32 squared distance exceeds thr, the larger list radius squared plus a
// margin that bounds the FP32 error (set by the host from the cell), so no
// pair inside either radius is ever dropped.  The survivors (about an eighth)
// queue up per warp in shared memory in candidate order and are decided 32 at
// a time by the reference's FP64 expression (pairvec_exact) with full warps;
// the hits are compacted with a ballot, so each row holds the same atoms in
// the same order as an all-FP64 scan.  A fractional offset within 1e-4 of
// +-1/2 (where FP32 and FP64 may pick different periodic images in a skewed
// cell) always goes to the exact test.  Row overflow sets *overflow and stops
// writing (the host grows the capacity and rebuilds).
constexpr int NL_THREADS = 256;
constexpr int NL_QUEUE = 64;   // per warp: below 32 queued before a chunk adds at most 32

// The prefilter's FP32 cell matrix and threshold, passed by value: kernel
// parameters live in the constant bank, so the FP32 products read them as
// operands and nothing is converted inside the candidate loop.
struct NlPre {
    float A[9];
    float thr;
};

__global__ void __launch_bounds__(NL_THREADS)
    k_nlist(int n, const double* __restrict__ sx, const double* __restrict__ sy, const double* __restrict__ sz,
            CellP c, const int* __restrict__ cell_of, const int* __restrict__ cell_start,
            const float4* __restrict__ cell_w, int nc0, int nc1, int nc2, NlPre pre, double rsq_a, int* nbr_a,
            int* cnt_a, int cap_a, double rsq_b, int* nbr_b, int* cnt_b, int cap_b, int* overflow) {
    __shared__ int s_q[NL_THREADS / 32][NL_QUEUE];
    const int lane = threadIdx.x & 31;
    int* q = s_q[threadIdx.x >> 5];
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= n) return;
    const double si1 = sx[i], si2 = sy[i], si3 = sz[i];
    float wi1 = (float)(si1 - floor(si1)), wi2 = (float)(si2 - floor(si2)), wi3 = (float)(si3 - floor(si3));
    // kept in registers: recomputing them from the FP64 coordinates inside the
    // loop would cost conversions on the quarter-rate XU pipe per candidate
    asm volatile("" : "+f"(wi1), "+f"(wi2), "+f"(wi3));
    const float* A = pre.A;
    const int ci = cell_of[i];
    const int cz = ci % nc2, cy = (ci / nc2) % nc1, cx = ci / (nc2 * nc1);
    const int lo0 = nc0 >= 3 ? -1 : 0, hi0 = nc0 >= 3 ? 1 : nc0 - 1;
    const int lo1 = nc1 >= 3 ? -1 : 0, hi1 = nc1 >= 3 ? 1 : nc1 - 1;
    const int lo2 = nc2 >= 3 ? -1 : 0, hi2 = nc2 >= 3 ? 1 : nc2 - 1;
    int na = 0, nb = 0, nq = 0;
    const unsigned lt = (1u << lane) - 1u;
    // exact FP64 test of the first cnt (<= 32) queued candidates, hits appended in queue order
    auto decide = [&](int cnt) {
        bool in_a = false, in_b = false;
        int j = -1;
        if (lane < cnt) {
            j = q[lane];
            double rx, ry, rz;
            const double rsq = pairvec_exact(c, si1, si2, si3, sx[j], sy[j], sz[j], rx, ry, rz);
            in_a = rsq <= rsq_a;
            in_b = rsq <= rsq_b;
        }
        const unsigned ma = __ballot_sync(0xffffffffu, in_a);
        if (in_a) {
            const int pos = na + __popc(ma & lt);
            if (pos < cap_a) nbr_a[(size_t)i * cap_a + pos] = j;
        }
        na += __popc(ma);
        if (nbr_b) {
            const unsigned mb = __ballot_sync(0xffffffffu, in_b);
            if (in_b) {
                const int pos = nb + __popc(mb & lt);
                if (pos < cap_b) nbr_b[(size_t)i * cap_b + pos] = j;
            }
            nb += __popc(mb);
        }
    };
    // periodic neighbour cell along one direction (offset -1, 0, +1), without
    // an integer division
    auto wrap = [](int c0, int off, int nc) {
        if (nc < 3) return off;
        const int v = c0 + off;
        return v < 0 ? v + nc : (v >= nc ? v - nc : v);
    };
    // d - rint(d) for d in [-1, 1] by compare and select (rounding instructions
    // run on the quarter-rate XU pipe); the ties d = +-1/2 are left as they are,
    // as rint leaves them, and go to the exact test anyway
    auto fold = [](float d) { return d > 0.5f ? d - 1.0f : (d < -0.5f ? d + 1.0f : d); };
    for (int a = lo0; a <= hi0; ++a) {
        const int x = wrap(cx, a, nc0);
        for (int b = lo1; b <= hi1; ++b) {
            const int y = wrap(cy, b, nc1);
            for (int d = lo2; d <= hi2; ++d) {
                const int z = wrap(cz, d, nc2);
                int cc = (x * nc1 + y) * nc2 + z;
                int s0 = cell_start[cc], s1 = cell_start[cc + 1];
                for (int base = s0; base < s1; base += 32) {
                    const int k = base + lane;
                    bool keep = false;
                    int j = -1;
                    if (k < s1) {
                        const float4 v = cell_w[k];
                        j = __float_as_int(v.w);
                        if (j != i) {
                            const float d1 = fold(wi1 - v.x), d2 = fold(wi2 - v.y), d3 = fold(wi3 - v.z);
                            const float rx = fmaf(d1, A[0], fmaf(d2, A[1], d3 * A[2]));
                            const float ry = fmaf(d1, A[3], fmaf(d2, A[4], d3 * A[5]));
                            const float rz = fmaf(d1, A[6], fmaf(d2, A[7], d3 * A[8]));
                            const float m = fmaxf(fabsf(d1), fmaxf(fabsf(d2), fabsf(d3)));
                            keep = fmaf(rx, rx, fmaf(ry, ry, rz * rz)) <= pre.thr || m > 0.4999f;
                        }
                    }
                    const unsigned mk = __ballot_sync(0xffffffffu, keep);
                    if (keep) q[nq + __popc(mk & lt)] = j;
                    nq += __popc(mk);
                    __syncwarp();
                    if (nq >= 32) {
                        decide(32);
                        __syncwarp();
                        const int rest = nq - 32;
                        const int moved = lane < rest ? q[32 + lane] : 0;
                        __syncwarp();
                        if (lane < rest) q[lane] = moved;
                        __syncwarp();
                        nq = rest;
                    }
                }
            }
        }
    }
    if (nq > 0) decide(nq);
    if (lane == 0) {
        cnt_a[i] = na < cap_a ? na : cap_a;
        if (na > cap_a) atomicMax(overflow, na);
        if (nbr_b) {
            cnt_b[i] = nb < cap_b ? nb : cap_b;
            if (nb > cap_b) atomicMax(overflow, nb);
        }
    }
}

void launch_nlist(cudaStream_t st, int n, const double* sx, const double* sy, const double* sz, CellP c,
                  const CellGrid& g, double rsq_a, NList& la, double rsq_b, NList* lb, int* overflow) {
    // FP32 error bound of the prefilter's distance: each wrapped fractional
    // coordinate is within 2^-25 of exact, a difference within 2^-24 more, and
    // the Cartesian products add under 2^-23 of |A| |d| (|d| <= 1/2); so a
    // component is off by at most ~2.1e-7 of its row's |A| sum.  Take 5e-7 of
    // the largest row sum, for every component, and pad r^2 accordingly.
    double row = 0.0;
    for (int a = 0; a < 3; ++a) row = std::max(row, std::fabs(c.A[3 * a]) + std::fabs(c.A[3 * a + 1]) + std::fabs(c.A[3 * a + 2]));
    const double del = 5e-7 * row * std::sqrt(3.0);
    const double rmax2 = std::max(rsq_a, lb ? rsq_b : 0.0), rmax = std::sqrt(rmax2);
    NlPre pre;
    for (int e = 0; e < 9; ++e) pre.A[e] = (float)c.A[e];
    pre.thr = std::nextafter((float)(rmax2 + 2.0 * rmax * del + del * del + 1e-6 * rmax2), INFINITY);
    const int blocks = (int)(((size_t)n * 32 + NL_THREADS - 1) / NL_THREADS);
    k_nlist<<<blocks, NL_THREADS, 0, st>>>(n, sx, sy, sz, c, g.cell_of, g.cell_start, g.cell_w, g.nc[0], g.nc[1],
                                           g.nc[2], pre, rsq_a, la.nbr, la.cnt, la.cap, rsq_b, lb ? lb->nbr : nullptr,
                                           lb ? lb->cnt : nullptr, lb ? lb->cap : 0, overflow);
}

// ------------------------------------------------------------ skin check --
// vnlistcheck (src/tools.f90:446-535): displacement of every atom since the
// last build (minimum image, reference operation order), largest and second
// largest over all atoms.  Per-block top-2 partials, merged by one block.
__device__ __forceinline__ void top2_merge(double& a1, double& a2, double b1, double b2) {
    // merge two (max, second max) pairs
    if (b1 > a1) { a2 = fmax(a1, b2); a1 = b1; }
    else a2 = fmax(a2, b1);
}

__global__ void k_skin_partial(int n, const double* sx, const double* sy, const double* sz, const double* xs,
                               const double* ys, const double* zs, CellP c, double* part) {
    double m1 = 0.0, m2 = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double rx, ry, rz;
        double d2 = pairvec_exact(c, sx[i], sy[i], sz[i], xs[i], ys[i], zs[i], rx, ry, rz);
        double d = sqrt(d2);
        if (d > m1) { m2 = m1; m1 = d; }
        else if (d > m2) m2 = d;
    }
    for (int o = 16; o > 0; o >>= 1) {
        double b1 = __shfl_xor_sync(0xffffffffu, m1, o), b2 = __shfl_xor_sync(0xffffffffu, m2, o);
        top2_merge(m1, m2, b1, b2);
    }
    __shared__ double s1[32], s2[32];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { s1[warp] = m1; s2[warp] = m2; }
    __syncthreads();
    if (warp == 0) {
        int nw = blockDim.x >> 5;
        m1 = lane < nw ? s1[lane] : 0.0;
        m2 = lane < nw ? s2[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            double b1 = __shfl_xor_sync(0xffffffffu, m1, o), b2 = __shfl_xor_sync(0xffffffffu, m2, o);
            top2_merge(m1, m2, b1, b2);
        }
        if (lane == 0) { part[2 * blockIdx.x] = m1; part[2 * blockIdx.x + 1] = m2; }
    }
}

__global__ void k_skin_final(int nblocks, const double* part, double skindiff, DevScalars* d) {
    double m1 = 0.0, m2 = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += 32) top2_merge(m1, m2, part[2 * b], part[2 * b + 1]);
    for (int o = 16; o > 0; o >>= 1) {
        double b1 = __shfl_xor_sync(0xffffffffu, m1, o), b2 = __shfl_xor_sync(0xffffffffu, m2, o);
        top2_merge(m1, m2, b1, b2);
    }
    if (threadIdx.x == 0) {
        d->dmax1 = m1;
        d->dmax2 = m2;
        d->rebuild = (m1 + m2 > skindiff) ? 1 : 0;
    }
}

void launch_skin_check(cudaStream_t st, int n, const double* sx, const double* sy, const double* sz,
                       const double* xs, const double* ys, const double* zs, CellP c, double skindiff,
                       Partials& part, DevScalars* d) {
    int blocks = (n + 255) / 256;
    if (blocks > 296) blocks = 296;
    k_skin_partial<<<blocks, 256, 0, st>>>(n, sx, sy, sz, xs, ys, zs, c, part.buf);
    k_skin_final<<<1, 32, 0, st>>>(blocks, part.buf, skindiff, d);
}

}  // namespace mdff
