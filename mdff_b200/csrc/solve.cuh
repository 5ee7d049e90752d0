// solve.cu -- deterministic reductions and the induced-dipole solver's vector
// kernels.
//
// The reference iterates mu <- alpha (E_stat + T mu) (moment_from_pola_scf,
// src/field.f90:3200-3458) and stops on the RMS of mu/alpha - E
// (src/field.f90:3378-3400).  Both that fixed-point iteration and a
// Jacobi-preconditioned conjugate-gradient solve of (1/alpha - T) mu = E_stat
// are driven from the host with these kernels; every dot product is an FP64
// block reduction summed in block order, so runs are bit-reproducible.
#include "common.cuh"

namespace mdff {

// out[k] (+)= sum_b buf[b*K + k]; one warp per k, lanes stride over blocks,
// fixed shuffle tree.
__global__ void k_reduce_partials(const double* __restrict__ buf, int nblocks, int K, double* out, int accumulate) {
    const int k = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    if (k >= K) return;
    double s = 0.0;
    for (int b = lane; b < nblocks; b += 32) s += buf[(size_t)b * K + k];
    s = warp_sum(s);
    if (lane == 0) out[k] = accumulate ? out[k] + s : s;
}

void launch_reduce_partials(cudaStream_t st, const double* buf, int nblocks, int K, double* out, int accumulate) {
    k_reduce_partials<<<1, 32 * K, 0, st>>>(buf, nblocks, K, out, accumulate);
}

// Ad = d/alpha - Eind on polarisable atoms, 0 elsewhere (n3 = 3n, component-major).
__global__ void k_apply_A(int n, const double* __restrict__ d, const double* __restrict__ Eind,
                          const double* __restrict__ inv_alpha, double* Ad) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * n) return;
    int i = t % n;
    double ia = inv_alpha[i];
    Ad[t] = ia != 0.0 ? d[t] * ia - Eind[t] : 0.0;
}

// r = b - Ax on polarisable atoms; z = alpha r; partial sums of r.r and r.z.
__global__ void k_cg_init(int n, const double* __restrict__ b, const double* __restrict__ Ax,
                          const double* __restrict__ alpha, const double* __restrict__ inv_alpha, double* r, double* z,
                          double* dvec, double* part) {
    double v[2] = {0.0, 0.0};
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 3 * n; t += gridDim.x * blockDim.x) {
        int i = t % n;
        double rr = inv_alpha[i] != 0.0 ? b[t] - Ax[t] : 0.0;
        double zz = alpha[i] * rr;
        r[t] = rr;
        z[t] = zz;
        dvec[t] = zz;
        v[0] = fma(rr, rr, v[0]);
        v[1] = fma(rr, zz, v[1]);
    }
    block_partials<2>(v, part);
}

// ---- one PCG iteration in four launches after the operator ------------------
// The sum k_reduce_partials forms for component k of nblocks partials (lanes
// stride over the blocks, then the xor tree), computed by one full warp, so
// a kernel that needs a reduced value forms it itself, bit for bit the same.
__device__ __forceinline__ double warp_reduce_partials(const double* __restrict__ buf, int nblocks, int K, int k) {
    const int lane = threadIdx.x & 31;
    double s = 0.0;
    for (int b = lane; b < nblocks; b += 32) s += buf[(size_t)b * K + k];
    return warp_sum(s);
}

// Ad = d/alpha - (E + 2 selfa2 d) on polarisable atoms, 0 elsewhere, and the
// partial sums of d.Ad: the operator's self term, k_apply_A and the dot
// product in one pass (grid-stride, like the solver's other vector kernels).
__global__ void k_cg_apply(int n, const double* __restrict__ d, const double* __restrict__ E, double two_s,
                           const double* __restrict__ inv_alpha, double* Ad, double* part) {
    double v[1] = {0.0};
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 3 * n; t += gridDim.x * blockDim.x) {
        const int i = t % n;
        const double ia = inv_alpha[i], dt = d[t];
        const double e = fma(two_s, dt, E[t]);
        const double a = ia != 0.0 ? dt * ia - e : 0.0;
        Ad[t] = a;
        v[0] = fma(dt, a, v[0]);
    }
    block_partials<1>(v, part);
}

// x += a d; r -= a Ad; z = alpha r; partial sums of r.r and r.z, with
// a = rz / dAd and d.Ad reduced from k_cg_apply's partials in each block;
// block 0 records d.Ad in the scalars.
__global__ void k_cg_update2(int n, const double* __restrict__ dvec, const double* __restrict__ Ad,
                             const double* __restrict__ alpha, double* x, double* r, double* z, DevScalars* sc,
                             const double* __restrict__ dpart, int ndpart, double* part) {
    __shared__ double sh_a;
    if (threadIdx.x < 32) {
        const double dAd = warp_reduce_partials(dpart, ndpart, 1, 0);
        if (threadIdx.x == 0) {
            sh_a = sc->rz / dAd;
            if (blockIdx.x == 0) sc->dAd = dAd;
        }
    }
    __syncthreads();
    const double a = sh_a;
    double v[2] = {0.0, 0.0};
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 3 * n; t += gridDim.x * blockDim.x) {
        int i = t % n;
        double xx = fma(a, dvec[t], x[t]);
        double rr = fma(-a, Ad[t], r[t]);
        double zz = alpha[i] * rr;
        x[t] = xx;
        r[t] = rr;
        z[t] = zz;
        v[0] = fma(rr, rr, v[0]);
        v[1] = fma(rr, zz, v[1]);
    }
    block_partials<2>(v, part);
}

// d = z + beta d with beta = rz_new / rz, r.r and r.z reduced from
// k_cg_update2's partials in each block; block 0 records them (rz itself
// advances in k_cg_fin / k_cg_fincond, after every block has read it).
__global__ void k_cg_direction2(int n3, const double* __restrict__ z, double* dvec, DevScalars* sc,
                                const double* __restrict__ upart, int nupart) {
    __shared__ double sh_b;
    if (threadIdx.x < 32) {
        const double rr = warp_reduce_partials(upart, nupart, 2, 0);
        const double rzn = warp_reduce_partials(upart, nupart, 2, 1);
        if (threadIdx.x == 0) {
            sh_b = rzn / sc->rz;
            if (blockIdx.x == 0) {
                sc->rr = rr;
                sc->rz_new = rzn;
                sc->beta_cg = sh_b;
            }
        }
    }
    __syncthreads();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n3) dvec[t] = fma(sh_b, dvec[t], z[t]);
}

// the end of an iteration: rz = rz_new; rmsd = sqrt(r.r / npol); count
__device__ __forceinline__ void cg_fin(DevScalars* sc, double inv_npol, double tol) {
    sc->rz = sc->rz_new;
    sc->rmsd = sqrt(sc->rr * inv_npol);
    sc->converged = sc->rmsd <= tol;
    sc->iter += 1;
}
__global__ void k_cg_fin(DevScalars* sc, double inv_npol, double tol) {
    if (threadIdx.x == 0 && blockIdx.x == 0) cg_fin(sc, inv_npol, tol);
}

// Test of the PCG loop when the MD step runs as a CUDA graph (the condition
// of its conditional WHILE node): another iteration while
// (iter < max_it and rmsd > tol) or iter < 1, the host loop's test, and none
// once the residual is not finite (the host reports that after the step).
// The iteration cap makes the loop finite whatever the residuals do.
__global__ void k_cg_cond(const DevScalars* __restrict__ sc, int max_it, double tol, cudaGraphConditionalHandle h) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double r = sc->rmsd;
    const int it = sc->iter;
    const bool go = ((it < max_it && r > tol) || it < 1) && isfinite(r);
    cudaGraphSetConditional(h, go ? 1u : 0u);
}

// The last kernel of the loop body: the end of the iteration, then the test.
__global__ void k_cg_fincond(DevScalars* sc, double inv_npol, double tol, int max_it, cudaGraphConditionalHandle h) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    cg_fin(sc, inv_npol, tol);
    const double r = sc->rmsd;
    const int it = sc->iter;
    const bool go = ((it < max_it && r > tol) || it < 1) && isfinite(r);
    cudaGraphSetConditional(h, go ? 1u : 0u);
}

__global__ void k_cg_first(DevScalars* sc, double inv_npol) {
    if (threadIdx.x != 0) return;
    sc->rz = sc->rz_new;
    sc->rmsd = sqrt(sc->rr * inv_npol);
    sc->iter = 0;
}

// Fixed-point step (induced_moment, src/field.f90:1716-1803): mu = alpha E.
__global__ void k_induced_moment(int n, const double* __restrict__ E, const double* __restrict__ alpha, double* mu) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < 3 * n) mu[t] = alpha[t % n] * E[t];
}

// ASPC corrector (src/field.f90:3986-3991): mu = w alpha (Estat + Eind) + (1-w) mu_p.
__global__ void k_aspc_correct(int n, const double* __restrict__ Estat, const double* __restrict__ Eind,
                               const double* __restrict__ alpha, double w, double* mu) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < 3 * n) mu[t] = w * (alpha[t % n] * (Estat[t] + Eind[t])) + (1.0 - w) * mu[t];
}

// E = Estat + Eind; partial sums of (mu/alpha - E)^2 over polarisable atoms.
__global__ void k_scf_residual(int n, const double* __restrict__ Estat, const double* __restrict__ Eind,
                               const double* __restrict__ mu, const double* __restrict__ inv_alpha, double* E,
                               double* part) {
    double v[1] = {0.0};
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 3 * n; t += gridDim.x * blockDim.x) {
        int i = t % n;
        double e = Estat[t] + Eind[t];
        E[t] = e;
        if (inv_alpha[i] != 0.0) {
            double r = mu[t] * inv_alpha[i] - e;
            v[0] = fma(r, r, v[0]);
        }
    }
    block_partials<1>(v, part);
}

// u_pol = 1/2 sum mu . alpha^-1 mu over polarisable atoms.
__global__ void k_upol(int n, const double* __restrict__ mu, const double* __restrict__ inv_alpha, double* part) {
    double v[1] = {0.0};
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 3 * n; t += gridDim.x * blockDim.x) {
        int i = t % n;
        v[0] = fma(mu[t] * inv_alpha[i], mu[t], v[0]);
    }
    block_partials<1>(v, part);
}

// Sums needed by the self and surface terms (src/field.f90:1869-1880):
// qsq, musq, qtot (sum q r), mutot.
__global__ void k_coul_sums(int n, const double* __restrict__ q, const double* __restrict__ mu,
                            const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
                            double* part) {
    double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double qi = q ? q[i] : 0.0;
        double m0 = mu[i], m1 = mu[n + i], m2 = mu[2 * n + i];
        v[0] += qi * qi;
        v[1] += m0 * m0 + m1 * m1 + m2 * m2;
        v[2] += qi * x[i]; v[3] += qi * y[i]; v[4] += qi * z[i];
        v[5] += m0; v[6] += m1; v[7] += m2;
    }
    block_partials<8>(v, part);
}

// Extrapolation of the induced dipoles from previous steps.
// mode 0: x = sum_k coef[k] hist[k]   (polynomial of order <= 1 and ASPC predictor)
// mode 1: Neville interpolation polint (src/field.f90:3995-4042) at x = 1 from
//         npt points at xa = 0, -1, -2, ...
// The predictor's plan lives in device memory (plan[0..15] the
// coefficients, plan[16] the mode, plan[17] the point count, plan[18] the
// history slots to shift), so one captured step serves every plan.
constexpr int PLAN_LEN = 19;

__global__ void k_extrapolate(int n3, const double* __restrict__ hist, const double* __restrict__ plan, double* x) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n3) return;
    const double* coef = plan;
    const int mode = (int)plan[16], npt = (int)plan[17];
    if (mode == 0) {
        double s = 0.0;
        for (int k = 0; k < npt; ++k) s += coef[k] * hist[(size_t)k * n3 + t];
        x[t] = s;
        return;
    }
    double c[16], d[16];
    int xa[16];
    for (int k = 0; k < npt; ++k) { xa[k] = -k; c[k] = d[k] = hist[(size_t)k * n3 + t]; }
    int ns = 1;
    double dif = fabs(1.0 - xa[0]);
    for (int k = 1; k <= npt; ++k) {
        double dift = fabs(1.0 - xa[k - 1]);
        if (dift < dif) { ns = k; dif = dift; }
    }
    double y = c[ns - 1], dy;
    ns = ns - 1;
    for (int m = 1; m <= npt - 1; ++m) {
        for (int k = 1; k <= npt - m; ++k) {
            double ho = double(xa[k - 1] - 1), hp = double(xa[k] - 1);
            double w = c[k] - d[k - 1];
            double den = w / (ho - hp);
            d[k - 1] = hp * den;
            c[k - 1] = ho * den;
        }
        if (2 * ns < npt - m) dy = c[ns];
        else { dy = d[ns - 1]; ns = ns - 1; }
        y = y + dy;
    }
    x[t] = y;
}

// history slot k <- slot k - 1 for k = plan[18] .. 1 (slot 0 is the newest)
__global__ void k_hist_shift(int n3, double* hist, const double* __restrict__ plan) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n3) return;
    const int s = (int)plan[18];
    for (int k = s; k >= 1; --k) hist[(size_t)k * n3 + t] = hist[(size_t)(k - 1) * n3 + t];
}

}  // namespace mdff
