// Structure optimisation on the device: the vector work of sastry
// (src/opt.f90:452-849) and eforce1d (:864-933).  Every force evaluation is
// the engine's own engforce at trial positions; the line search's scalar
// control flow runs on the host (engine.cu, opt_sastry) from deterministic
// per-atom reductions of these kernels.  Vectors over 3N components are
// component-major ([c * n + i]); per-atom terms are summed per atom first,
// as the reference's loops group them.
#include "common.cuh"

namespace mdff {

// xi = -f; g = -xi; h = g; xi = h (the steepest-descent direction, :496-513),
// with the per-atom terms of |xi|^2.
__global__ void k_opt_steepest(int n, const double* __restrict__ fx, const double* __restrict__ fy,
                               const double* __restrict__ fz, double* __restrict__ xi, double* __restrict__ g,
                               double* __restrict__ h, double* part) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[1] = {0.0};
    if (i < n) {
        const double f[3] = {fx[i], fy[i], fz[i]};
        double s = 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double x = -f[c];
            const double gc = -x;
            g[(size_t)c * n + i] = gc;
            h[(size_t)c * n + i] = gc;
            xi[(size_t)c * n + i] = gc;
            s = s + gc * gc;
        }
        v[0] = s;
    }
    block_partials<1>(v, part);
}

// xi = xi / umag (:508-512)
__global__ void k_opt_div(int n3, double* __restrict__ xi, double umag) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n3) xi[t] = xi[t] / umag;
}

// MODE 0: sum f.xi (the directional derivative, :556-560, :925-929);
// MODE 1: sum f.f (phigrad, :535-538);
// MODE 2: gg = sum g.g and dgg = sum (xi + g).xi with xi = -f (:783-790).
template <int MODE>
__global__ void k_opt_dots(int n, const double* __restrict__ fx, const double* __restrict__ fy,
                           const double* __restrict__ fz, const double* __restrict__ xi, const double* __restrict__ g,
                           double* part) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[2] = {0.0, 0.0};
    if (i < n) {
        const double f[3] = {fx[i], fy[i], fz[i]};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if (MODE == 0) v[0] = v[0] + f[c] * xi[(size_t)c * n + i];
            if (MODE == 1) v[0] = v[0] + f[c] * f[c];
            if (MODE == 2) {
                const double gc = g[(size_t)c * n + i], xc = -f[c];
                v[0] = v[0] + gc * gc;
                v[1] = v[1] + (xc + gc) * xc;
            }
        }
    }
    block_partials<2>(v, part);
}

// trial positions r = r0 + s xi (eforce1d :900-904; the accepted move :705-709)
__global__ void k_opt_move(int n, const double* __restrict__ r0x, const double* __restrict__ r0y,
                           const double* __restrict__ r0z, const double* __restrict__ xi, double s,
                           double* __restrict__ x, double* __restrict__ y, double* __restrict__ z) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    x[i] = r0x[i] + s * xi[i];
    y[i] = r0y[i] + s * xi[(size_t)n + i];
    z[i] = r0z[i] + s * xi[(size_t)2 * n + i];
}

// conjugate-gradient direction (:799-811): xi = -f; g = -xi; h = g + gam h;
// xi = h, with the per-atom terms of |xi|^2.
__global__ void k_opt_cg(int n, const double* __restrict__ fx, const double* __restrict__ fy,
                         const double* __restrict__ fz, double* __restrict__ xi, double* __restrict__ g,
                         double* __restrict__ h, double gam, double* part) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[1] = {0.0};
    if (i < n) {
        const double f[3] = {fx[i], fy[i], fz[i]};
        double s = 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const size_t k = (size_t)c * n + i;
            const double x = -f[c];
            const double gc = -x;
            g[k] = gc;
            const double hc = gc + gam * h[k];
            h[k] = hc;
            xi[k] = hc;
            s = s + hc * hc;
        }
        v[0] = s;
    }
    block_partials<1>(v, part);
}

}  // namespace mdff
