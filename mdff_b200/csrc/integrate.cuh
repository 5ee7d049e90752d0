// integrate.cu -- velocity Verlet and the Nose-Hoover chain on the GPU.
//
// prop_velocity_verlet (src/integration.f90:131-194), prop_pos_vel_verlet
// (src/integration.f90:333-385), chain_nhcn (src/integration.f90:564-713) and
// the conserved thermostat energy of nhcn (src/integration.f90:520-545).
// Per-atom updates are one thread per atom; the kinetic energy is an FP64
// block reduction summed in block order; the thermostat chain is a handful of
// FP64 scalars advanced by a single thread.
#include "common.cuh"

namespace mdff {

constexpr int IB = 256;

// r += v dt + f dt^2/2 / m ; fold = f
__global__ void k_vv_positions(int n, double* x, double* y, double* z, const double* vx, const double* vy,
                               const double* vz, const double* fx, const double* fy, const double* fz,
                               double* fox, double* foy, double* foz, const double* mass, double dt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double dtsq2 = dt * dt * 0.5, m = mass[i];
    x[i] = x[i] + vx[i] * dt + (fx[i] * dtsq2) / m;
    y[i] = y[i] + vy[i] * dt + (fy[i] * dtsq2) / m;
    z[i] = z[i] + vz[i] * dt + (fz[i] * dtsq2) / m;
    fox[i] = fx[i]; foy[i] = fy[i]; foz[i] = fz[i];
}

// v += (fold + f) dt/2 / m ; kinetic-energy partials
__global__ void k_vv_velocities(int n, double* vx, double* vy, double* vz, const double* fx, const double* fy,
                                const double* fz, const double* fox, const double* foy, const double* foz,
                                const double* mass, double dt, double* part) {
    double v[1] = {0.0};
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        double dt2 = dt * 0.5, m = mass[i];
        double a = vx[i] + (fox[i] + fx[i]) * dt2 / m;
        double b = vy[i] + (foy[i] + fy[i]) * dt2 / m;
        double c = vz[i] + (foz[i] + fz[i]) * dt2 / m;
        vx[i] = a; vy[i] = b; vz[i] = c;
        v[0] = (a * a + b * b + c * c) * m;
    }
    block_partials<1>(v, part);
}

// v += f dt/2 / m ; r += v dt   (first half of prop_pos_vel_verlet)
__global__ void k_kick_drift(int n, double* x, double* y, double* z, double* vx, double* vy, double* vz,
                             const double* fx, const double* fy, const double* fz, const double* mass, double dt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double dt2 = dt * 0.5, m = mass[i];
    double a = vx[i] + fx[i] * dt2 / m;
    double b = vy[i] + fy[i] * dt2 / m;
    double c = vz[i] + fz[i] * dt2 / m;
    vx[i] = a; vy[i] = b; vz[i] = c;
    x[i] = x[i] + a * dt;
    y[i] = y[i] + b * dt;
    z[i] = z[i] + c * dt;
}

// v += f dt/2 / m ; kinetic-energy partials
__global__ void k_kick(int n, double* vx, double* vy, double* vz, const double* fx, const double* fy,
                       const double* fz, const double* mass, double dt, double* part) {
    double v[1] = {0.0};
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        double dt2 = dt * 0.5, m = mass[i];
        double a = vx[i] + fx[i] * dt2 / m;
        double b = vy[i] + fy[i] * dt2 / m;
        double c = vz[i] + fz[i] * dt2 / m;
        vx[i] = a; vy[i] = b; vz[i] = c;
        v[0] = (a * a + b * b + c * c) * m;
    }
    block_partials<1>(v, part);
}

// v *= s (s read from the device scalars; s = 1 gives a plain kinetic-energy
// reduction, as calc_temp, src/kinetic.f90:531-560)
__global__ void k_scale_ke(int n, double* vx, double* vy, double* vz, const double* mass, const DevScalars* sc,
                           int apply, double* part) {
    double v[1] = {0.0};
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        double a = vx[i], b = vy[i], c = vz[i];
        if (apply) {
            double s = sc->s_scale;
            a = s * a; b = s * b; c = s * c;
            vx[i] = a; vy[i] = b; vz[i] = c;
        }
        v[0] = (a * a + b * b + c * c) * mass[i];
    }
    block_partials<1>(v, part);
}

struct NhcConst {
    int nhc_n, yosh, mults, literal;
    double dt, temp, L;
    double Q[16];
    double w[9];
};

// chain_nhcn, trotter_order = -1 branch (src/integration.f90:617-649); kin is
// 2*e_kin stored by the preceding reduction (sum m v^2); writes s_scale.
__global__ void k_nhc_chain(DevScalars* sc, NhcConst c, const double* ke2) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int nh = c.nhc_n;
    double G[16];
    for (int k = 0; k < nh; ++k) G[k] = 0.0;
    double* vxi = sc->vxi;
    double* xi = sc->xi;
    const double kin = 0.5 * ke2[0];
    const double temp = c.temp;
    double s = 1.0;
    G[0] = 2.0 * kin - c.L * temp;
    for (int k = 0; k < c.mults; ++k) {
        for (int j = 0; j < c.yosh; ++j) {
            double dts = c.w[j] * c.dt / (double)c.mults;
            double dts2 = dts * 0.5, dts4 = dts2 * 0.5, dts8 = dts4 * 0.5;
            G[nh - 1] = (vxi[nh - 2] * vxi[nh - 2] / c.Q[nh - 2] - temp);
            // The reference leaves G(2..M-1) at 0 / stale on this downward pass,
            // which breaks conservation of the extended energy for M > 2; they
            // are refreshed here unless the literal order is requested.
            if (!c.literal)
                for (int inh = 1; inh < nh - 1; ++inh) G[inh] = vxi[inh - 1] * vxi[inh - 1] / c.Q[inh - 1] - temp;
            vxi[nh - 1] = vxi[nh - 1] + G[nh - 1] * dts4;
            for (int inh = nh - 2; inh >= 0; --inh) {
                vxi[inh] = vxi[inh] * exp(-vxi[inh + 1] * dts8 / c.Q[inh + 1]);
                vxi[inh] = vxi[inh] + G[inh] * dts4;
                vxi[inh] = vxi[inh] * exp(-vxi[inh + 1] * dts8 / c.Q[inh + 1]);
            }
            s = s * exp(-vxi[0] * dts2 / c.Q[0]);
            for (int inh = 0; inh < nh; ++inh) xi[inh] = xi[inh] + vxi[inh] * dts2 / c.Q[inh];
            G[0] = 2.0 * kin * s * s - c.L * temp;
            for (int inh = 0; inh < nh - 1; ++inh) {
                vxi[inh] = vxi[inh] * exp(-vxi[inh + 1] * dts8 / c.Q[inh + 1]);
                vxi[inh] = vxi[inh] + G[inh] * dts4;
                vxi[inh] = vxi[inh] * exp(-vxi[inh + 1] * dts8 / c.Q[inh + 1]);
                G[inh + 1] = (vxi[inh] * vxi[inh] / c.Q[inh] - temp);
            }
            vxi[nh - 1] = vxi[nh - 1] + G[nh - 1] * dts4;
        }
    }
    sc->s_scale = s;
}

// chain_nhc2 (src/integration.f90:265-324): the two-thermostat chain of
// Frenkel and Smit, one quarter/half-step sequence per call (no Suzuki-Yoshida
// splitting).  Here vxi(1), vxi(2) are thermostat VELOCITIES (the chain
// forces are divided by Q and the scaling is exp(-vxi dt)), unlike
// chain_nhcn's momenta.  kin is 2*e_kin from the preceding reduction; the
// chain's own kin -> s^2 kin update feeds its second G1; writes s_scale.
__global__ void k_nhc2_chain(DevScalars* sc, NhcConst c, const double* ke2) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double* vxi = sc->vxi;
    double* xi = sc->xi;
    const double temp = c.temp, L = c.L, Q1 = c.Q[0], Q2 = c.Q[1];
    const double dt2 = c.dt * 0.5, dt4 = dt2 * 0.5, dt8 = dt4 * 0.5;
    double kin = 0.5 * ke2[0];
    double s = 1.0;
    double G1 = (2.0 * kin - L * temp) / Q1;
    double G2 = (Q1 * vxi[0] * vxi[0] - temp) / Q2;
    vxi[1] = vxi[1] + G2 * dt4;
    vxi[0] = vxi[0] * exp(-vxi[1] * dt8);
    vxi[0] = vxi[0] + G1 * dt4;
    vxi[0] = vxi[0] * exp(-vxi[1] * dt8);
    s = s * exp(-vxi[0] * dt2);
    kin = s * s * kin;
    xi[0] = xi[0] + vxi[0] * dt2;
    xi[1] = xi[1] + vxi[1] * dt2;
    G1 = (2.0 * kin - L * temp) / Q1;
    vxi[0] = vxi[0] * exp(-vxi[1] * dt8);
    vxi[0] = vxi[0] + G1 * dt4;
    vxi[0] = vxi[0] * exp(-vxi[1] * dt8);
    G2 = (Q1 * vxi[0] * vxi[0] - temp) / Q2;
    vxi[1] = vxi[1] + G2 * dt4;
    sc->s_scale = s;
}

// Thermostat energy of nhc2 (src/integration.f90:243-250).  The reference
// writes vxi^2 / (2 Q), the momentum form of nhcn, although nhc2's vxi are
// velocities; the conserved quantity of the Frenkel-Smit chain has the
// kinetic terms Q vxi^2 / 2, used here (deviation D23).  With c.literal the
// reference's expression is returned instead.
__global__ void k_nhc2_energy(DevScalars* sc, NhcConst c) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double* v = sc->vxi;
    const double* x = sc->xi;
    double e = c.L * c.temp * x[0];
    e = e + (c.literal ? v[0] * v[0] * 0.5 / c.Q[0] : c.Q[0] * v[0] * v[0] * 0.5);
    e = e + (c.literal ? v[1] * v[1] * 0.5 / c.Q[1] : c.Q[1] * v[1] * v[1] * 0.5);
    e = e + c.temp * x[1];
    sc->e_nvt = e;
}

// Conserved thermostat energy (src/integration.f90:531-544).
__global__ void k_nhc_energy(DevScalars* sc, NhcConst c) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double e = c.L * c.temp * sc->xi[0] + sc->vxi[0] * sc->vxi[0] * 0.5 / c.Q[0];
    double a = 0.0, b = 0.0;
    for (int k = 1; k < c.nhc_n; ++k) {
        a = a + sc->vxi[k] * sc->vxi[k] * 0.5 / c.Q[k];
        b = b + c.temp * sc->xi[k];
    }
    sc->e_nvt = e + a + b;
}

}  // namespace mdff
