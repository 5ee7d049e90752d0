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

namespace mdff {

// ---- L-BFGS (lbfgs_driver, src/opt.f90:972-1194, over LBFGS/MCSRCH of
// src/lbfgs.f90:243-957) ----------------------------------------------------
// The optimisation vector is X = (rx, ry, rz) and G = -(fx, fy, fz) as the
// driver packs them.  A V3 names the three component arrays of one 3N vector
// (the engine's SoA positions and forces, or a component-major buffer) and a
// sign applied on reading, so G is read straight from the forces.
struct V3 {
    const double* c[3];
    double sgn;
};

__device__ __forceinline__ double v3(const V3& v, int c, int i) { return v.sgn * v.c[c][i]; }

// K = 1 or 2 dot products a0.b0 (and a1.b1), per-atom terms first
template <int K>
__global__ void k_lb_dots(int n, V3 a0, V3 b0, V3 a1, V3 b1, double* part) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[K];
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = 0.0;
    if (i < n) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            v[0] = v[0] + v3(a0, c, i) * v3(b0, c, i);
            if (K > 1) v[K - 1] = v[K - 1] + v3(a1, c, i) * v3(b1, c, i);
        }
    }
    block_partials<K>(v, part);
}

// One step of the two-loop recursion (Nocedal 1980; LBFGS :326-358) with its
// coefficient taken from the device scalar sc[0], the dot product just
// reduced there, so the recursion needs no host round trip.
//   FIRST:  alpha_cp = rho sq, kept in sc[1 + cp];  w = w - alpha_cp y_cp
//   second: beta = alpha_cp - rho yr;               w = w + beta s_cp
template <bool FIRST>
__global__ void k_lb_twoloop(int n3, double* __restrict__ w, const double* __restrict__ v, double* sc, double rho,
                             int cp) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (FIRST) {
        const double alpha = rho * sc[0];
        if (t == 0) sc[1 + cp] = alpha;
        if (t < n3) w[t] = w[t] + (-alpha) * v[t];
    } else {
        double beta = rho * sc[0];
        beta = sc[1 + cp] - beta;
        if (t < n3) w[t] = w[t] + beta * v[t];
    }
}

// w = -G (= f), optionally times a uniform diagonal d (the first direction
// -G DIAG with DIAG = 1, :293-294); g0 = G kept for the gradient change
__global__ void k_lb_negg(int n, const double* __restrict__ fx, const double* __restrict__ fy,
                          const double* __restrict__ fz, double d, double* __restrict__ w) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double f[3] = {fx[i], fy[i], fz[i]};
#pragma unroll
    for (int c = 0; c < 3; ++c) w[(size_t)c * n + i] = (-(-f[c])) * d;
}

__global__ void k_lb_scale(int n3, double* __restrict__ w, double d) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n3) w[t] = d * w[t];
}

// G kept before the line search (W(I) = G(I), :370-371)
__global__ void k_lb_keepg(int n, const double* __restrict__ fx, const double* __restrict__ fy,
                           const double* __restrict__ fz, double* __restrict__ g0) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    g0[i] = -fx[i];
    g0[(size_t)n + i] = -fy[i];
    g0[(size_t)2 * n + i] = -fz[i];
}

// trial point X = WA + stp S (MCSRCH :40)
__global__ void k_lb_place(int n, const double* __restrict__ wa, const double* __restrict__ s, double stp,
                           double* __restrict__ x, double* __restrict__ y, double* __restrict__ z) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    x[i] = wa[i] + stp * s[i];
    y[i] = wa[(size_t)n + i] + stp * s[(size_t)n + i];
    z[i] = wa[(size_t)2 * n + i] + stp * s[(size_t)2 * n + i];
}

// the accepted step and gradient change: S = stp S, Y = G - g0 (:391-393)
__global__ void k_lb_pair(int n, const double* __restrict__ fx, const double* __restrict__ fy,
                          const double* __restrict__ fz, const double* __restrict__ g0, double stp,
                          double* __restrict__ s, double* __restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double f[3] = {fx[i], fy[i], fz[i]};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const size_t k = (size_t)c * n + i;
        s[k] = stp * s[k];
        y[k] = (-f[c]) - g0[k];
    }
}

}  // namespace mdff

namespace mdff {

// ---- M1QN3 in diagonal-initial-scaling mode (m1qn3_driver,
// src/opt.f90:1203-1330, over m1qn3a/dd/mlis3 of src/m1qn3.f90) ------------

// d = -G precos = f precos (the cold start's Fletcher scaling, :477-481)
__global__ void k_m1_start(int n, const double* __restrict__ fx, const double* __restrict__ fy,
                           const double* __restrict__ fz, double precos, double* __restrict__ d,
                           double* __restrict__ diag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double f[3] = {fx[i], fy[i], fz[i]};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        d[(size_t)c * n + i] = (-(-f[c])) * precos;
        diag[(size_t)c * n + i] = 1.0;
    }
}

// max_i |d_i| (tmin = dxmin / max |d_i|, :522-526): non-negative doubles
// order as their bit patterns, so an integer atomicMax is exact; *out must
// be zero before the launch
__global__ void k_m1_absmax(int n3, const double* __restrict__ d, unsigned long long* out) {
    double m = 0.0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n3; t += gridDim.x * blockDim.x) m = fmax(m, fabs(d[t]));
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// the pair of the accepted step: sbar = t d, ybar = G - gg (:637-640)
__global__ void k_m1_pair(int n, const double* __restrict__ fx, const double* __restrict__ fy,
                          const double* __restrict__ fz, const double* __restrict__ gg, const double* __restrict__ d,
                          double t, double* __restrict__ sbar, double* __restrict__ ybar) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double f[3] = {fx[i], fy[i], fz[i]};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const size_t k = (size_t)c * n + i;
        sbar[k] = t * d[k];
        ybar[k] = (-f[c]) - gg[k];
    }
}

// MODE 0: sum diag y^2 (:667-670); MODE 1: sum s^2 / diag (:677-680)
template <int MODE>
__global__ void k_m1_diagsum(int n, const double* __restrict__ diag, const double* __restrict__ v, double* part) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[1] = {0.0};
    if (i < n) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const size_t k = (size_t)c * n + i;
            if (MODE == 0) acc[0] = acc[0] + diag[k] * v[k] * v[k];
            else acc[0] = acc[0] + v[k] * v[k] / diag[k];
        }
    }
    block_partials<1>(acc, part);
}

// the diagonal's BFGS update (:681-687): diag = 1 / (1/diag + y^2 - (s/diag)^2 / den),
// rmin where that is not positive
__global__ void k_m1_diagupd(int n3, double* __restrict__ diag, const double* __restrict__ y,
                             const double* __restrict__ s, double den, double rmin) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n3) return;
    const double q = s[t] / diag[t];
    double v = 1.0 / (1.0 / diag[t] + y[t] * y[t] - (q * q) / den);
    if (v <= 0.0) v = rmin;
    diag[t] = v;
}

// w = w diag (dd's diagonal preconditioning, :895-899)
__global__ void k_m1_mul(int n3, double* __restrict__ w, const double* __restrict__ diag) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n3) w[t] = w[t] * diag[t];
}

// mlis3's machine-precision test (:1270-1274): is xn + t d different from
// both xn and the last trial x in some component?  *flag set to 1 if so.
__global__ void k_m1_moves(int n, const double* __restrict__ xn, const double* __restrict__ d, double t,
                           const double* __restrict__ x, const double* __restrict__ y,
                           const double* __restrict__ z, int* flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* cur[3] = {x, y, z};
    bool moves = false;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const size_t k = (size_t)c * n + i;
        const double zz = xn[k] + t * d[k];
        moves = moves || (zz != xn[k] && zz != cur[c][i]);
    }
    if (moves) *flag = 1;
}

}  // namespace mdff
