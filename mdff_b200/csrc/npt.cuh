// Constant pressure: nhcnp (src/integration.f90:966-1042) -- isotropic
// Martyna-Tobias-Klein barostat (Mol. Phys. 87, 1117 (1996)) with
// Nose-Hoover chains on the particles (chain xi, Q) and on the barostat
// (chain xib, Qb), barostat mass W, log-volume coordinate xe and momentum ve.
//
// The particle updates run on the device (prop_pos_vel_verlet_npt,
// src/integration.f90:1049-1160); the chains act on a handful of scalars and
// run on the host between the kinetic-energy reductions.  Four corrections
// to the reference make the step a time-reversible MTK step whose conserved
// quantity is the reference's own e_npt + e_tot:
//   D14  the k mesh and the tail corrections follow the cell (the reference
//        computes both once at start-up and keeps them while the cell moves);
//   D15  the barostat momentum gets both half kicks, ve += Ge dt/2 after the
//        first chain half and before the second (the reference's calls with
//        trotter orders -1 and +1 give one half kick per step);
//   D16  chain forces G_{k+1} = p_k^2 / Q_k - kT and Gb_1 = ve^2 / W - kT (the
//        reference halves them);
//   D17  kinetic pressure (1 + 3/Nf) 2K / 3V with K = sum m v^2 / 2 (the
//        reference uses K in place of 2K).
#pragma once
#include <cmath>

#include "common.cuh"

namespace mdff {

// v = v AA2 + f BB / m, kinetic-energy partials (sum m v^2)
__global__ void k_npt_kick(int n, double* vx, double* vy, double* vz, const double* fx, const double* fy,
                           const double* fz, const double* mass, double AA2, double BB, double* part) {
    double v[1] = {0.0};
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const double m = mass[i];
        const double a = vx[i] * AA2 + fx[i] * BB / m;
        const double b = vy[i] * AA2 + fy[i] * BB / m;
        const double c = vz[i] * AA2 + fz[i] * BB / m;
        vx[i] = a; vy[i] = b; vz[i] = c;
        v[0] = (a * a + b * b + c * c) * m;
    }
    block_partials<1>(v, part);
}

// r = r AA2 + v BB
__global__ void k_npt_drift(int n, double* x, double* y, double* z, const double* vx, const double* vy,
                            const double* vz, double AA2, double BB) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    x[i] = x[i] * AA2 + vx[i] * BB;
    y[i] = y[i] * AA2 + vy[i] * BB;
    z[i] = z[i] * AA2 + vz[i] * BB;
}

// Refresh of the k tables for a new cell of the same rectangle, membership
// fixed at set-up (mask bit 1: a k of the half space, bit 2: of the mixed
// path's FP32 set): A_k = exp(-k^2 / 4 alpha^2) / k^2 and the stress
// coefficient 2 (1/k^2 + 1/4 alpha^2), as kpoint_sum_init
// (src/kspace.f90:142-207) computes them.
__global__ void k_kgrid_refresh(int nrect, int nzl, int kmax1, int kmax2, CellP c, double a2,
                                const unsigned char* __restrict__ mask, double* Ak, double* kcoe, double* Ak_hi) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrect) return;
    const int col = r / nzl, m = r - col * nzl;
    const int nx = col / (2 * kmax1 + 1), ny = col % (2 * kmax1 + 1) - kmax1, nz = m - kmax2;
    const unsigned char mk = mask[r];
    double ak = 0.0, kc = 0.0;
    if (mk & 1) {
        const double kx = 2.0 * PI * ((double)nx * c.B[0] + (double)ny * c.B[1] + (double)nz * c.B[2]);
        const double ky = 2.0 * PI * ((double)nx * c.B[3] + (double)ny * c.B[4] + (double)nz * c.B[5]);
        const double kz = 2.0 * PI * ((double)nx * c.B[6] + (double)ny * c.B[7] + (double)nz * c.B[8]);
        const double kk = kx * kx + ky * ky + kz * kz;
        ak = exp(-kk * 0.25 / a2) / kk;
        kc = 2.0 * (1.0 / kk + 1.0 / a2 / 4.0);
    }
    Ak[r] = ak;
    kcoe[r] = kc;
    if (Ak_hi) Ak_hi[r] = (mk & 2) ? ak : 0.0;
}

// The same for the mixed path's FP64 low set: column q = (nx, ny, nzlo, nzn).
__global__ void k_lowk_refresh(int ncol, int nzmax, CellP c, double a2, const int* __restrict__ col, double* Ak,
                               double* kcoe) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ncol * nzmax) return;
    const int q = t / nzmax, m = t - q * nzmax;
    const int nx = col[4 * q], ny = col[4 * q + 1], nz = col[4 * q + 2] + m, nn = col[4 * q + 3];
    double ak = 0.0, kc = 0.0;
    if (m < nn) {
        const double kx = 2.0 * PI * ((double)nx * c.B[0] + (double)ny * c.B[1] + (double)nz * c.B[2]);
        const double ky = 2.0 * PI * ((double)nx * c.B[3] + (double)ny * c.B[4] + (double)nz * c.B[5]);
        const double kz = 2.0 * PI * ((double)nx * c.B[6] + (double)ny * c.B[7] + (double)nz * c.B[8]);
        const double kk = kx * kx + ky * ky + kz * kz;
        ak = exp(-kk * 0.25 / a2) / kk;
        kc = 2.0 * (1.0 / kk + 1.0 / a2 / 4.0);
    }
    Ak[t] = ak;
    kcoe[t] = kc;
}

// Barostat and thermostat state (md module: xi, vxi, xib, vxib, xe, ve, xe0).
struct NptState {
    double xi[16] = {0}, vxi[16] = {0}, xib[16] = {0}, vxib[16] = {0};
    double xe = 0.0, ve = 0.0, xe0 = 0.0;
    double e_npt = 0.0;
    double scale = 1.0, scale_build = 1.0;   // linear cell scale now / at the last list build
    double A_build[9] = {0};                 // the cell (column-major) of the last list build
};

struct NptConst {
    int nhc_n, yosh, mults, literal;
    double dt, temp, L, W, press;
    double Q[16], Qb[16];
    double w[9];
};

// One half of chain_nhcnp (src/integration.f90:724-964): first = true runs the
// barostat chain then the particle chain (trotter order -1), false the
// particle chain then the barostat chain (+1).  kin = sum m v^2 / 2 on entry;
// returns the particle velocity scale s and the barostat momentum scale sb.
inline void npt_chain_half(const NptConst& c, NptState& st, double kin, bool first, double& s_out,
                           double& sb_out) {
    const int nh = c.nhc_n;
    double G[16] = {0}, Gb[16] = {0};
    double s = 1.0, sb = 1.0;
    const double temp = c.temp;
    G[0] = 2.0 * kin - c.L * temp;
    Gb[0] = st.ve * st.ve / c.W - temp;   // D16
    auto chain = [&](double* vx, double* x, const double* Q, double* Gv, double& sc, bool baro, double dts) {
        const double dts2 = dts * 0.5, dts4 = dts2 * 0.5, dts8 = dts4 * 0.5;
        Gv[nh - 1] = vx[nh - 2] * vx[nh - 2] / Q[nh - 2] - temp;   // D16
        if (!c.literal)   // inner forces current before the downward pass (D13 of the NVT chain)
            for (int k = 1; k < nh - 1; ++k) Gv[k] = vx[k - 1] * vx[k - 1] / Q[k - 1] - temp;
        vx[nh - 1] = vx[nh - 1] + Gv[nh - 1] * dts4;
        for (int k = nh - 2; k >= 0; --k) {
            vx[k] = vx[k] * std::exp(-vx[k + 1] * dts8 / Q[k + 1]);
            vx[k] = vx[k] + Gv[k] * dts4;
            vx[k] = vx[k] * std::exp(-vx[k + 1] * dts8 / Q[k + 1]);
        }
        sc = sc * std::exp(-vx[0] * dts2 / Q[0]);
        for (int k = 0; k < nh; ++k) x[k] = x[k] + vx[k] * dts2 / Q[k];
        Gv[0] = baro ? st.ve * st.ve * sc * sc / c.W - temp : 2.0 * kin * sc * sc - c.L * temp;
        for (int k = 0; k < nh - 1; ++k) {
            vx[k] = vx[k] * std::exp(-vx[k + 1] * dts8 / Q[k + 1]);
            vx[k] = vx[k] + Gv[k] * dts4;
            vx[k] = vx[k] * std::exp(-vx[k + 1] * dts8 / Q[k + 1]);
            Gv[k + 1] = vx[k] * vx[k] / Q[k] - temp;
        }
        vx[nh - 1] = vx[nh - 1] + Gv[nh - 1] * dts4;
    };
    for (int k = 0; k < c.mults; ++k)
        for (int j = 0; j < c.yosh; ++j) {
            const double dts = c.w[j] * c.dt / (double)c.mults;
            if (first) {
                chain(st.vxib, st.xib, c.Qb, Gb, sb, true, dts);
                chain(st.vxi, st.xi, c.Q, G, s, false, dts);
            } else {
                chain(st.vxi, st.xi, c.Q, G, s, false, dts);
                chain(st.vxib, st.xib, c.Qb, Gb, sb, true, dts);
            }
        }
    s_out = s;
    sb_out = sb;
}

// e_npt of nhcnp (src/integration.f90:1017-1034)
inline double npt_energy(const NptConst& c, const NptState& st, double omega) {
    double e = c.press * omega + st.ve * st.ve * 0.5 / c.W + c.L * c.temp * st.xi[0] + c.temp * st.xib[0] +
               st.vxi[0] * st.vxi[0] * 0.5 / c.Q[0] + st.vxib[0] * st.vxib[0] * 0.5 / c.Qb[0];
    for (int k = 1; k < c.nhc_n; ++k) {
        e += st.vxi[k] * st.vxi[k] * 0.5 / c.Q[k];
        e += st.vxib[k] * st.vxib[k] * 0.5 / c.Qb[k];
        e += c.temp * st.xi[k];
        e += c.temp * st.xib[k];
    }
    return e;
}

// sinh(x)/x by its series to x^8, as prop_pos_vel_verlet_npt evaluates it
inline double npt_poly(double arg) {
    const double e2 = 1.0 / 6.0, e4 = e2 / 20.0, e6 = e4 / 42.0, e8 = e6 / 72.0;
    const double a2 = arg * arg;
    return (((e8 * a2 + e6) * a2 + e4) * a2 + e2) * a2 + 1.0;
}

}  // namespace mdff
