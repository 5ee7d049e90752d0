// batch.cu -- many configurations of uneven size in one set of launches:
// forces and stress of every configuration, the force-matching loss and its
// gradient with respect to the force-field parameters.
//
// The reference evaluates one configuration at a time and has no
// derivatives.  Here every phase is ONE launch over all configurations of
// the batch: per-atom kernels index their configuration through cfg_of[],
// the reciprocal-space kernels run over a work list of (configuration,
// chunk of atoms) blocks, and every per-configuration sum is a fixed-order
// block reduction (deterministic).  The induced-dipole systems of all
// configurations are solved by one lockstep preconditioned conjugate
// gradient; a configuration that has converged is frozen and its blocks
// return at once.
//
// Physics per configuration is the engine's FP64 path: BMH / BMHFTD with
// Tang-Toennies dispersion damping and Morse (engforce_bmhftd_pbc,
// src/field.f90:2876-3026; engforce_morse_pbc, :3039-3185), and the multipole
// Ewald sum for charges and induced dipoles with Tang-Toennies charge-dipole
// damping (multipole_ES_dir / _rec, src/field.f90:2057-2873).
//
// Gradient (adjoint method).  With R_i = dL/dF_i and S = dL/dtau fixed,
// dL/dtheta = dJ/dtheta for J = sum_i R_i.F_i + S:tau.  The induced dipoles
// solve A mu = b, A = 1/alpha - T (T: the undamped dipole field operator,
// symmetric), b: the damped static field.  One adjoint solve A lambda = dJ/dmu
// gives dL/dtheta = dJ/dtheta|_mu + lambda.(db/dtheta - dA/dtheta mu).
// dJ/dmu has a real-space part (k_b_dir_adj, the mu-derivatives of the pair
// force expressions weighted by W_ij = cu R_i + cu/(2 omega press) S r_ij) and a
// reciprocal part (a structure factor of the amplitudes (k.R_i)(q_i + i k.mu_i)
// and the field gradient, k_b_sfac MODE 3 and k_b_sfac_reduce ADJ).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "engine_internal.h"
#include "common.cuh"

using namespace mdff;

namespace {

constexpr int CHUNK = 128;     // atoms per reciprocal-space block
constexpr int NZC = 8;         // nz values per thread in the structure factor
constexpr int KT = 128;        // threads of the reciprocal-space blocks
constexpr int CT = 16;         // k-columns staged per tile in the field kernel
constexpr int KF_LPA = 4;      // lanes per atom in the field kernel (columns interleaved)
constexpr int NTYB = 2;        // types supported by the gradient kernels


struct BCfg {
    CellP cell;
    int off, n;            // atoms [off, off+n)
    int roff;              // first k-rectangle entry
    int kmax[3];
    int ncol, nzl, nrect;
    int cs, ce;            // chunks [cs, ce)
    int npol;
    double rc2, alpha, selfa, selfa2;
    double cF, cS;         // loss weights
};

struct BChunk { int c, a0, na; long poff; };

struct BPair {
    double A, B, C, D, BD;
    double eps, rho, sig, rs;
    double db_i, dc_i, db_j, dc_j;
    int dk_i, dk_j, ldamp, pad;
};

struct BFlags {
    int bmh, bmhftd, morse, coul, erfc_ref;
    double cu, press;
};

inline int nblk(long n, int t) { return (int)((n + t - 1) / t); }

// --------------------------------------------------------------------------
// positions
// --------------------------------------------------------------------------

// read_pos.f90:148-150 (kardir, periodicbc, dirkar) and kardir, per atom with
// its configuration's cell; the engine's exact operation order.
__global__ void k_b_wrap_frac(int N, const int* __restrict__ cfg_of, const BCfg* __restrict__ cf, double* x, double* y,
                              double* z, double* sx, double* sy, double* sz) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const CellP& c = cf[cfg_of[i]].cell;
    double X = x[i], Y = y[i], Z = z[i];
    double s1 = __dadd_rn(__dadd_rn(__dmul_rn(X, c.B[0]), __dmul_rn(Y, c.B[3])), __dmul_rn(Z, c.B[6]));
    double s2 = __dadd_rn(__dadd_rn(__dmul_rn(X, c.B[1]), __dmul_rn(Y, c.B[4])), __dmul_rn(Z, c.B[7]));
    double s3 = __dadd_rn(__dadd_rn(__dmul_rn(X, c.B[2]), __dmul_rn(Y, c.B[5])), __dmul_rn(Z, c.B[8]));
    s1 = __dsub_rn(s1, round(s1));
    s2 = __dsub_rn(s2, round(s2));
    s3 = __dsub_rn(s3, round(s3));
    X = __dadd_rn(__dadd_rn(__dmul_rn(s1, c.A[0]), __dmul_rn(s2, c.A[1])), __dmul_rn(s3, c.A[2]));
    Y = __dadd_rn(__dadd_rn(__dmul_rn(s1, c.A[3]), __dmul_rn(s2, c.A[4])), __dmul_rn(s3, c.A[5]));
    Z = __dadd_rn(__dadd_rn(__dmul_rn(s1, c.A[6]), __dmul_rn(s2, c.A[7])), __dmul_rn(s3, c.A[8]));
    x[i] = X; y[i] = Y; z[i] = Z;
    sx[i] = __dadd_rn(__dadd_rn(__dmul_rn(X, c.B[0]), __dmul_rn(Y, c.B[3])), __dmul_rn(Z, c.B[6]));
    sy[i] = __dadd_rn(__dadd_rn(__dmul_rn(X, c.B[1]), __dmul_rn(Y, c.B[4])), __dmul_rn(Z, c.B[7]));
    sz[i] = __dadd_rn(__dadd_rn(__dmul_rn(X, c.B[2]), __dmul_rn(Y, c.B[5])), __dmul_rn(Z, c.B[8]));
}

// Full neighbour rows within rc of each configuration (all pairs of the
// configuration, ascending j, reference inclusion test and operation order);
// one warp per atom, hits compacted with a ballot.
__global__ void k_b_nlist(int N, const int* __restrict__ cfg_of, const BCfg* __restrict__ cf,
                          const double* __restrict__ sx, const double* __restrict__ sy, const double* __restrict__ sz,
                          int* nbr, int* cnt, int cap, int* overflow) {
    const int lane = threadIdx.x & 31;
    const int i = (int)(((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (i >= N) return;
    const BCfg& C = cf[cfg_of[i]];
    const double si1 = sx[i], si2 = sy[i], si3 = sz[i];
    const unsigned lt = (1u << lane) - 1u;
    int na = 0;
    for (int base = C.off; base < C.off + C.n; base += 32) {
        int j = base + lane;
        bool in = false;
        if (j < C.off + C.n && j != i) {
            double rx, ry, rz;
            double rsq = pairvec_exact(C.cell, si1, si2, si3, sx[j], sy[j], sz[j], rx, ry, rz);
            in = rsq <= C.rc2;
        }
        unsigned m = __ballot_sync(0xffffffffu, in);
        if (in) {
            int pos = na + __popc(m & lt);
            if (pos < cap) nbr[(size_t)i * cap + pos] = j;
        }
        na += __popc(m);
    }
    if (lane == 0) {
        cnt[i] = na < cap ? na : cap;
        if (na > cap) atomicMax(overflow, na);
    }
}

// --------------------------------------------------------------------------
// short-range pairs
// --------------------------------------------------------------------------

__device__ __forceinline__ void tt_fd(double b, double r, int k, double& f, double& fd) { tt_damp_d(b, 1.0, r, k, f, fd); }

// Tang-Toennies pieces and their derivatives with respect to b and c:
// g = 1 - f = c e^{-x} sum_{m<=k} x^m/m!, gd = f' = c b e^{-x} x^k/k!, x = b r.
struct TTD { double g, gd, g_b, g_c, gd_b, gd_c; };
__device__ __forceinline__ TTD tt_deriv(double b, double c, double r, int k) {
    const double x = b * r, e = exp(-x);
    double term = 1.0, sum = 1.0, inv = 1.0;
    for (int m = 1; m <= k; ++m) {
        inv = inv / (double)m;
        term = term * x;
        sum = fma(term, inv, sum);
    }
    const double tk = term * inv;
    TTD t;
    t.g = c * e * sum;
    t.gd = c * b * e * tk;
    t.g_c = e * sum;
    t.g_b = -c * r * e * tk;
    t.gd_c = b * e * tk;
    t.gd_b = c * e * tk * (1.0 + k - x);
    return t;
}

// Forces (written), per-atom energy and stress sums (half per ordered pair).
template <int G>
__global__ void __launch_bounds__(256) k_b_pair(int N, const int* __restrict__ cfg_of, const BCfg* __restrict__ cf,
                                                const double* __restrict__ sx, const double* __restrict__ sy,
                                                const double* __restrict__ sz, const int* __restrict__ type,
                                                const int* __restrict__ nbr, const int* __restrict__ cnt, int cap,
                                                const BPair* __restrict__ pc, BFlags fl, double* __restrict__ f,
                                                double* __restrict__ e_atom, double* __restrict__ s_atom) {
    const int gid = (int)(((long)blockIdx.x * blockDim.x + threadIdx.x) / G);
    const int sub = threadIdx.x & (G - 1);
    const bool active = gid < N;
    const int i = active ? gid : 0;
    const BCfg& C = cf[cfg_of[i]];
    double F[3] = {0, 0, 0}, u = 0.0, S[6] = {0, 0, 0, 0, 0, 0};
    if (active) {
        const double si1 = sx[i], si2 = sy[i], si3 = sz[i];
        const int ti = type[i];
        const int m = cnt[i];
        const int* row = nbr + (size_t)i * cap;
        for (int k = sub; k < m; k += G) {
            const int j = row[k];
            double rx, ry, rz;
            const double rsq = pairvec_exact(C.cell, si1, si2, si3, sx[j], sy[j], sz[j], rx, ry, rz);
            if (!(rsq < C.rc2)) continue;
            const BPair& P = pc[ti * NT + type[j]];
            double w = 0.0;
            const double d = sqrt(rsq);
            if ((fl.bmh || fl.bmhftd) && P.A != 0.0) {
                const double ir2 = 1.0 / rsq;
                const double erh = P.A * exp(-P.B * d);
                double ir6 = ir2 * ir2 * ir2;
                double ir8 = ir6 * ir2;
                ir6 *= P.C;
                ir8 *= P.D;
                double ir6d = ir6, ir8d = ir8, fd6 = 0.0, fd8 = 0.0;
                if (fl.bmhftd) {
                    double f6, f8;
                    tt_fd(P.BD, d, 6, f6, fd6);
                    tt_fd(P.BD, d, 8, f8, fd8);
                    ir6d = ir6 * f6;
                    ir8d = ir8 * f8;
                }
                w += (P.B * erh - 6.0 * ir6d / d - 8.0 * ir8d / d + ir6 * fd6 + ir8 * fd8) / d;
                u += 0.5 * (erh - ir6d - ir8d);
            }
            if (fl.morse) {
                const double e = exp(-d * P.rho) * P.rs;
                const double em1 = e - 1.0;
                u += 0.5 * P.eps * (em1 * em1 - 1.0);
                w += 2.0 * P.eps * P.rho * e * em1 / d;
            }
            F[0] += w * rx; F[1] += w * ry; F[2] += w * rz;
            const double hw = 0.5 * w;
            S[0] += hw * rx * rx; S[1] += hw * ry * ry; S[2] += hw * rz * rz;
            S[3] += hw * rx * ry; S[4] += hw * rx * rz; S[5] += hw * ry * rz;
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) F[k] = group_sum<G>(F[k]);
#pragma unroll
    for (int k = 0; k < 6; ++k) S[k] = group_sum<G>(S[k]);
    u = group_sum<G>(u);
    if (active && sub == 0) {
        for (int k = 0; k < 3; ++k) f[(size_t)k * N + i] = F[k];
        e_atom[i] = u;
        for (int k = 0; k < 6; ++k) s_atom[(size_t)k * N + i] = S[k];
    }
}

// --------------------------------------------------------------------------
// real-space Ewald
// --------------------------------------------------------------------------

struct PairG { double d, A1, B2, C3, F0; };

__device__ __forceinline__ PairG ewald_radial(double d2, double a, int erfc_ref) {
    const double rsqpi = 0.56418958354775628695;
    const double a2 = a * a, a3 = a2 * a, a5 = a3 * a2;
    PairG g;
    const double d = sqrt(d2);
    const double dm1 = 1.0 / d, dm2 = dm1 * dm1, dm3 = dm1 * dm2, dm5 = dm3 * dm2, dm7 = dm5 * dm2;
    const double ex2 = exp(-a2 * d2), expon = ex2 * rsqpi;
    const double F0 = erfc_ref ? erfc_fit(a * d) : erfc_ex2(a * d, ex2);
    const double F1 = F0 + 2.0 * a * d * expon;
    const double F2 = F1 + (4.0 * a3 / 3.0) * d2 * d * expon;
    const double F3 = F2 + (8.0 * a5 / 15.0) * d2 * d2 * d * expon;
    g.d = d;
    g.F0 = F0 * dm1;
    g.A1 = F1 * dm3;
    g.B2 = 3.0 * F2 * dm5;
    g.C3 = 15.0 * F3 * dm7;
    return g;
}

// The dipole operator from a pair table.  A batch's positions never move, so
// for every neighbour within rc the pair vector and the radial factors
// A1 = F1/r^3, B2 = 3 F2/r^5 of the undamped dipole field are computed once
// (k_b_ddtab_build) and every application of the operator in the forward and
// adjoint solves is a gather: E_i = sum_j r (r.mu_j) B2 - mu_j A1.  Entries are
// stored per quantity ([5][N cap]: rx ry rz A1 B2), FP64, or FP32 when the
// batch runs mixed (the products then in FP32, the sums in FP64).  Rows are
// compacted to the neighbours within rc in list order.
template <int G, typename T>
__global__ void __launch_bounds__(256) k_b_ddtab_build(int N, const int* __restrict__ cfg_of,
                                                       const BCfg* __restrict__ cf, const double* __restrict__ sx,
                                                       const double* __restrict__ sy, const double* __restrict__ sz,
                                                       const int* __restrict__ nbr, const int* __restrict__ cnt,
                                                       int cap, int erfc_ref, int* __restrict__ dnbr,
                                                       int* __restrict__ dcnt, T* __restrict__ tab) {
    const int gid = (int)(((long)blockIdx.x * blockDim.x + threadIdx.x) / G);
    const int sub = threadIdx.x & (G - 1);
    const bool active = gid < N;
    const int i = active ? gid : 0;
    const BCfg& C = cf[cfg_of[i]];
    const size_t NC = (size_t)N * cap;
    const int g0 = (threadIdx.x & 31) & ~(G - 1);
    const unsigned gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << g0);
    const int m = active ? cnt[i] : 0;
    int base = 0;
    for (int k0 = 0; k0 < m; k0 += G) {   // m is the same for the G lanes of an atom
        const int k = k0 + sub;
        const bool valid = k < m;
        const int j = valid ? nbr[(size_t)i * cap + k] : i;
        double rx = 0, ry = 0, rz = 0, d2 = 0;
        if (valid) d2 = pairvec_exact(C.cell, sx[i], sy[i], sz[i], sx[j], sy[j], sz[j], rx, ry, rz);
        const bool in = valid && d2 <= C.rc2;
        const unsigned bal = (__ballot_sync(gmask, in) & gmask) >> g0;
        const int pos = base + __popc(bal & ((1u << sub) - 1u));
        if (in) {
            const PairG g = ewald_radial(d2, C.alpha, erfc_ref);
            const size_t e = (size_t)i * cap + pos;
            dnbr[e] = j;
            tab[e] = (T)rx;
            tab[NC + e] = (T)ry;
            tab[2 * NC + e] = (T)rz;
            tab[3 * NC + e] = (T)g.A1;
            tab[4 * NC + e] = (T)g.B2;
        }
        base += __popc(bal);
    }
    if (active && sub == 0) dcnt[i] = base;
}

template <int G, typename T>
__global__ void __launch_bounds__(256) k_b_ddtab(int N, const int* __restrict__ cfg_of, const int* __restrict__ conv,
                                                 const int* __restrict__ dnbr, const int* __restrict__ dcnt, int cap,
                                                 const T* __restrict__ tab, const double* __restrict__ v,
                                                 double* __restrict__ E) {
    const int gid = (int)(((long)blockIdx.x * blockDim.x + threadIdx.x) / G);
    const int sub = threadIdx.x & (G - 1);
    bool active = gid < N;
    const int i = active ? gid : 0;
    if (conv && conv[cfg_of[i]]) active = false;
    const size_t NC = (size_t)N * cap;
    double V0 = 0.0, V1 = 0.0, V2 = 0.0;
    if (active) {
        const int m = dcnt[i];
        for (int k = sub; k < m; k += G) {
            const size_t e = (size_t)i * cap + k;
            const int j = dnbr[e];
            const T rx = tab[e], ry = tab[NC + e], rz = tab[2 * NC + e], A1 = tab[3 * NC + e], B2 = tab[4 * NC + e];
            const T mj0 = (T)v[j], mj1 = (T)v[N + j], mj2 = (T)v[2 * N + j];
            const T rb = (rx * mj0 + ry * mj1 + rz * mj2) * B2;
            V0 += (double)(rx * rb - mj0 * A1);
            V1 += (double)(ry * rb - mj1 * A1);
            V2 += (double)(rz * rb - mj2 * A1);
        }
    }
    V0 = group_sum<G>(V0);
    V1 = group_sum<G>(V1);
    V2 = group_sum<G>(V2);
    if (active && sub == 0) { E[i] = V0; E[N + i] = V1; E[2 * N + i] = V2; }
}

// MODE 0: damped field of the charges (static field b of the dipole solve,
//         src/field.f90:3270-3272).
// MODE 1: field of the dipoles mu, undamped (the operator T, src/field.f90:3354).
// MODE 2: forces, energy and stress of charges + dipoles with the damped
//         charge-dipole terms (the final multipole_ES call).
template <int G, int MODE>
__global__ void __launch_bounds__(256) k_b_dir(int N, const int* __restrict__ cfg_of, const BCfg* __restrict__ cf,
                                               const int* __restrict__ conv, const double* __restrict__ sx,
                                               const double* __restrict__ sy, const double* __restrict__ sz,
                                               const int* __restrict__ type, const double* __restrict__ q,
                                               const double* __restrict__ mu, const int* __restrict__ nbr,
                                               const int* __restrict__ cnt, int cap, const BPair* __restrict__ pc,
                                               BFlags fl, double* __restrict__ out, double* __restrict__ e_atom,
                                               double* __restrict__ s_atom) {
    const int gid = (int)(((long)blockIdx.x * blockDim.x + threadIdx.x) / G);
    const int sub = threadIdx.x & (G - 1);
    bool active = gid < N;
    const int i = active ? gid : 0;
    const int c = cfg_of[i];
    if (conv && conv[c]) active = false;
    const BCfg& C = cf[c];
    double V[3] = {0, 0, 0}, u = 0.0, S[6] = {0, 0, 0, 0, 0, 0};
    if (active) {
        const double si1 = sx[i], si2 = sy[i], si3 = sz[i];
        const int ti = type[i];
        const double qi = MODE == 1 ? 0.0 : q[i];
        const double mi0 = MODE == 0 ? 0.0 : mu[i], mi1 = MODE == 0 ? 0.0 : mu[N + i], mi2 = MODE == 0 ? 0.0 : mu[2 * N + i];
        const int m = cnt[i];
        const int* row = nbr + (size_t)i * cap;
        for (int k = sub; k < m; k += G) {
            const int j = row[k];
            double rx, ry, rz;
            const double d2 = pairvec_exact(C.cell, si1, si2, si3, sx[j], sy[j], sz[j], rx, ry, rz);
            if (d2 > C.rc2) continue;
            const PairG g = ewald_radial(d2, C.alpha, fl.erfc_ref);
            if (MODE == 1) {
                const double mj0 = mu[j], mj1 = mu[N + j], mj2 = mu[2 * N + j];
                const double rmj = rx * mj0 + ry * mj1 + rz * mj2;
                V[0] += rx * rmj * g.B2 - mj0 * g.A1;
                V[1] += ry * rmj * g.B2 - mj1 * g.A1;
                V[2] += rz * rmj * g.B2 - mj2 * g.A1;
                continue;
            }
            const int tj = type[j];
            const double qj = q[j];
            const BPair& P = pc[ti * NT + tj];
            double gi = 0.0, gdi = 0.0, gj = 0.0, gdj = 0.0;
            if (P.ldamp) {
                double f1, f2;
                tt_damp_d(P.db_i, P.dc_i, g.d, P.dk_i, f1, gdi);
                tt_damp_d(P.db_j, P.dc_j, g.d, P.dk_j, f2, gdj);
                gi = 1.0 - f1;
                gj = 1.0 - f2;
            }
            if (MODE == 0) {
                const double s = qj * (g.A1 - gi / (g.d * d2));
                V[0] += s * rx; V[1] += s * ry; V[2] += s * rz;
                continue;
            }
            const double mj0 = mu[j], mj1 = mu[N + j], mj2 = mu[2 * N + j];
            const double rmj = rx * mj0 + ry * mj1 + rz * mj2;
            const double rmi = rx * mi0 + ry * mi1 + rz * mi2;
            const double mimj = mi0 * mj0 + mi1 * mj1 + mi2 * mj2;
            double fi[3];
            // charge-charge
            u += 0.5 * qi * qj * g.F0;
            const double sq = qi * qj * g.A1;
            fi[0] = sq * rx; fi[1] = sq * ry; fi[2] = sq * rz;
            // dipole-dipole
            u -= 0.5 * (rmi * rmj * g.B2 - mimj * g.A1);
            const double t3 = -rmi * rmj * g.C3 + mimj * g.B2;
            fi[0] += t3 * rx + (mi0 * rmj + mj0 * rmi) * g.B2;
            fi[1] += t3 * ry + (mi1 * rmj + mj1 * rmi) * g.B2;
            fi[2] += t3 * rz + (mi2 * rmj + mj2 * rmi) * g.B2;
            // charge-dipole
            u += 0.5 * (qi * g.A1 * rmj - qj * g.A1 * rmi);
            const double s = (qi * rmj - qj * rmi) * g.B2;
            fi[0] += rx * s - (qi * mj0 - qj * mi0) * g.A1;
            fi[1] += ry * s - (qi * mj1 - qj * mi1) * g.A1;
            fi[2] += rz * s - (qi * mj2 - qj * mi2) * g.A1;
            if (P.ldamp) {
                const double dm3 = 1.0 / (g.d * d2), dm5 = dm3 / d2;
                u += 0.5 * (-qi * gj * dm3 * rmj + qj * gi * dm3 * rmi);
                const double Bi = 3.0 * (gi + (g.d / 3.0) * gdi) * dm5, Ai = gi * dm3;
                const double Bj = 3.0 * (gj + (g.d / 3.0) * gdj) * dm5, Aj = gj * dm3;
                fi[0] += qj * (rx * rmi * Bi - mi0 * Ai) - qi * (rx * rmj * Bj - mj0 * Aj);
                fi[1] += qj * (ry * rmi * Bi - mi1 * Ai) - qi * (ry * rmj * Bj - mj1 * Aj);
                fi[2] += qj * (rz * rmi * Bi - mi2 * Ai) - qi * (rz * rmj * Bj - mj2 * Aj);
            }
            V[0] += fi[0]; V[1] += fi[1]; V[2] += fi[2];
            S[0] += 2.0 * rx * fi[0]; S[1] += 2.0 * ry * fi[1]; S[2] += 2.0 * rz * fi[2];
            S[3] += rx * fi[1] + ry * fi[0]; S[4] += rx * fi[2] + rz * fi[0]; S[5] += ry * fi[2] + rz * fi[1];
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) V[k] = group_sum<G>(V[k]);
    if (MODE == 2) {
        u = group_sum<G>(u);
#pragma unroll
        for (int k = 0; k < 6; ++k) S[k] = group_sum<G>(S[k]);
    }
    if (active && sub == 0) {
        for (int k = 0; k < 3; ++k) out[(size_t)k * N + i] = V[k];
        if (MODE == 2) {
            e_atom[i] = u;
            for (int k = 0; k < 6; ++k) s_atom[(size_t)k * N + i] = S[k];
        }
    }
}

// mu-derivatives of W . f(i,j), f the force on the first atom of a pair
// evaluation (charge-charge carries no mu): dW/dmu_first (hf) and
// dW/dmu_second (hs).  Bf/Af and Bs/As are the damped radial factors at the
// first and second atom (zero without damping).
__device__ __forceinline__ void force_mu_grad(const double r[3], const double W[3], double qf, double qs,
                                              const double mf[3], const double ms[3], const PairG& g, double Bf,
                                              double Af, double Bs, double As, double hf[3], double hs[3]) {
    const double wr = W[0] * r[0] + W[1] * r[1] + W[2] * r[2];
    const double rmf = r[0] * mf[0] + r[1] * mf[1] + r[2] * mf[2];
    const double rms = r[0] * ms[0] + r[1] * ms[1] + r[2] * ms[2];
    const double Wmf = W[0] * mf[0] + W[1] * mf[1] + W[2] * mf[2];
    const double Wms = W[0] * ms[0] + W[1] * ms[1] + W[2] * ms[2];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        hf[c] = wr * (-r[c] * rms * g.C3 + ms[c] * g.B2) + W[c] * rms * g.B2 + Wms * r[c] * g.B2
              - wr * qs * r[c] * g.B2 + qs * W[c] * g.A1 + qs * (wr * r[c] * Bf - W[c] * Af);
        hs[c] = wr * (-r[c] * rmf * g.C3 + mf[c] * g.B2) + Wmf * r[c] * g.B2 + W[c] * rmf * g.B2
              + wr * qf * r[c] * g.B2 - qf * W[c] * g.A1 - qf * (wr * r[c] * Bs - W[c] * As);
    }
}

// Adjoint right-hand side, real space: h_i = d/dmu_i of sum over ordered pair
// evaluations W.f, for the evaluations of row i (derivative w.r.t. the first
// atom) and those of the rows j that hold i (w.r.t. the second atom, rebuilt
// here from row i by symmetry of the full list).  Also the derivative of the
// damped charge-dipole force w.r.t. the damping b and c at fixed mu (slots
// G_DI_*, G_DJ_* of the ordered pair (ti,tj)).
template <int G>
__global__ void __launch_bounds__(256) k_b_dir_adj(int N, const int* __restrict__ cfg_of, const BCfg* __restrict__ cf,
                                                   const double* __restrict__ sx, const double* __restrict__ sy,
                                                   const double* __restrict__ sz, const int* __restrict__ type,
                                                   const double* __restrict__ q, const double* __restrict__ mu,
                                                   const double* __restrict__ R, const double* __restrict__ Sres,
                                                   const int* __restrict__ nbr, const int* __restrict__ cnt, int cap,
                                                   const BPair* __restrict__ pc, BFlags fl, double* __restrict__ h,
                                                   double* part) {
    const int gid = (int)(((long)blockIdx.x * blockDim.x + threadIdx.x) / G);
    const int sub = threadIdx.x & (G - 1);
    const bool active = gid < N;
    const int i = active ? gid : 0;
    const int c = cfg_of[i];
    const BCfg& C = cf[c];
    double H[3] = {0, 0, 0};
    double acc[NTYB][4];
#pragma unroll
    for (int t = 0; t < NTYB; ++t) acc[t][0] = acc[t][1] = acc[t][2] = acc[t][3] = 0.0;
    const int ti = type[i];
    if (active) {
        const double si1 = sx[i], si2 = sy[i], si3 = sz[i];
        const double qi = q[i];
        const double mi[3] = {mu[i], mu[N + i], mu[2 * N + i]};
        const double Ri[3] = {R[i], R[N + i], R[2 * N + i]};
        double Sm[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) Sm[k] = Sres[c * 9 + k];
        const double sw = 0.5 * fl.cu / (C.cell.omega * fl.press);
        const int m = cnt[i];
        const int* row = nbr + (size_t)i * cap;
        for (int k = sub; k < m; k += G) {
            const int j = row[k];
            double r[3];
            const double d2 = pairvec_exact(C.cell, si1, si2, si3, sx[j], sy[j], sz[j], r[0], r[1], r[2]);
            if (d2 > C.rc2) continue;
            const PairG g = ewald_radial(d2, C.alpha, fl.erfc_ref);
            const int tj = type[j];
            const double qj = q[j];
            const double mj[3] = {mu[j], mu[N + j], mu[2 * N + j]};
            const double Rj[3] = {R[j], R[N + j], R[2 * N + j]};
            double Sr[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) Sr[a] = Sm[a * 3] * r[0] + Sm[a * 3 + 1] * r[1] + Sm[a * 3 + 2] * r[2];
            const double dm3 = 1.0 / (g.d * d2), dm5 = dm3 / d2;
            // evaluation (i,j): W_ij = cu R_i + sw S r
            double W[3], hf[3], hs[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) W[a] = fl.cu * Ri[a] + sw * Sr[a];
            const BPair& P = pc[ti * NT + tj];
            double Bi = 0, Ai = 0, Bj = 0, Aj = 0;
            TTD Ti{}, Tj{};
            if (P.ldamp) {
                Ti = tt_deriv(P.db_i, P.dc_i, g.d, P.dk_i);
                Tj = tt_deriv(P.db_j, P.dc_j, g.d, P.dk_j);
                Ai = Ti.g * dm3; Bi = 3.0 * (Ti.g + g.d / 3.0 * Ti.gd) * dm5;
                Aj = Tj.g * dm3; Bj = 3.0 * (Tj.g + g.d / 3.0 * Tj.gd) * dm5;
            }
            force_mu_grad(r, W, qi, qj, mi, mj, g, Bi, Ai, Bj, Aj, hf, hs);
            H[0] += hf[0]; H[1] += hf[1]; H[2] += hf[2];
            if (P.ldamp) {
                const double wr = W[0] * r[0] + W[1] * r[1] + W[2] * r[2];
                const double rmi = r[0] * mi[0] + r[1] * mi[1] + r[2] * mi[2];
                const double rmj = r[0] * mj[0] + r[1] * mj[1] + r[2] * mj[2];
                const double Wmi = W[0] * mi[0] + W[1] * mi[1] + W[2] * mi[2];
                const double Wmj = W[0] * mj[0] + W[1] * mj[1] + W[2] * mj[2];
                const double dAi_b = Ti.g_b * dm3, dBi_b = (3.0 * Ti.g_b + g.d * Ti.gd_b) * dm5;
                const double dAi_c = Ti.g_c * dm3, dBi_c = (3.0 * Ti.g_c + g.d * Ti.gd_c) * dm5;
                const double dAj_b = Tj.g_b * dm3, dBj_b = (3.0 * Tj.g_b + g.d * Tj.gd_b) * dm5;
                const double dAj_c = Tj.g_c * dm3, dBj_c = (3.0 * Tj.g_c + g.d * Tj.gd_c) * dm5;
                const double v0 = qj * (wr * rmi * dBi_b - Wmi * dAi_b);
                const double v1 = qj * (wr * rmi * dBi_c - Wmi * dAi_c);
                const double v2 = -qi * (wr * rmj * dBj_b - Wmj * dAj_b);
                const double v3 = -qi * (wr * rmj * dBj_c - Wmj * dAj_c);
#pragma unroll
                for (int t = 0; t < NTYB; ++t)
                    if (t == tj) { acc[t][0] += v0; acc[t][1] += v1; acc[t][2] += v2; acc[t][3] += v3; }
            }
            // evaluation (j,i) (row j): first atom j, second atom i, r_ji = -r,
            // W_ji = cu R_j - sw S r, damping from the pair constants (tj,ti)
            double rn[3] = {-r[0], -r[1], -r[2]};
#pragma unroll
            for (int a = 0; a < 3; ++a) W[a] = fl.cu * Rj[a] - sw * Sr[a];
            const BPair& Q = pc[tj * NT + ti];
            double Bf = 0, Af = 0, Bs = 0, As = 0;
            if (Q.ldamp) {
                double f1, gd1, f2, gd2;
                tt_damp_d(Q.db_i, Q.dc_i, g.d, Q.dk_i, f1, gd1);
                tt_damp_d(Q.db_j, Q.dc_j, g.d, Q.dk_j, f2, gd2);
                const double g1 = 1.0 - f1, g2 = 1.0 - f2;
                Af = g1 * dm3; Bf = 3.0 * (g1 + g.d / 3.0 * gd1) * dm5;
                As = g2 * dm3; Bs = 3.0 * (g2 + g.d / 3.0 * gd2) * dm5;
            }
            force_mu_grad(rn, W, qj, qi, mj, mi, g, Bf, Af, Bs, As, hf, hs);
            H[0] += hs[0]; H[1] += hs[1]; H[2] += hs[2];
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) H[k] = group_sum<G>(H[k]);
    if (active && sub == 0)
        for (int k = 0; k < 3; ++k) h[(size_t)k * N + i] = H[k];
    double v[NTYB * NTYB * 4];
#pragma unroll
    for (int a = 0; a < NTYB; ++a)
#pragma unroll
        for (int t = 0; t < NTYB; ++t)
#pragma unroll
            for (int s = 0; s < 4; ++s) v[(a * NTYB + t) * 4 + s] = (active && a == ti) ? acc[t][s] : 0.0;
    block_partials<NTYB * NTYB * 4>(v, part);
}

// Gradient terms gathered over rows after the adjoint solve: the short-range
// parameters (dw/dtheta [R_i.r + r.S.r/(2 omega press)] per ordered pair) and
// the damping of the static field (-q_j lambda_i.r/d^3 dg_i/dtheta).
template <int G>
__global__ void __launch_bounds__(256) k_b_grad_rows(int N, const int* __restrict__ cfg_of, const BCfg* __restrict__ cf,
                                                     const double* __restrict__ sx, const double* __restrict__ sy,
                                                     const double* __restrict__ sz, const int* __restrict__ type,
                                                     const double* __restrict__ q, const double* __restrict__ R,
                                                     const double* __restrict__ Sres, const double* __restrict__ lam,
                                                     const int* __restrict__ nbr, const int* __restrict__ cnt, int cap,
                                                     const BPair* __restrict__ pc, BFlags fl, double* part) {
    const int gid = (int)(((long)blockIdx.x * blockDim.x + threadIdx.x) / G);
    const int sub = threadIdx.x & (G - 1);
    const bool active = gid < N;
    const int i = active ? gid : 0;
    const int c = cfg_of[i];
    const BCfg& C = cf[c];
    constexpr int NS = 10;   // A B C D BD eps rho sig, lambda-b, lambda-c
    double acc[NTYB][NS];
#pragma unroll
    for (int t = 0; t < NTYB; ++t)
#pragma unroll
        for (int s = 0; s < NS; ++s) acc[t][s] = 0.0;
    const int ti = type[i];
    if (active) {
        const double si1 = sx[i], si2 = sy[i], si3 = sz[i];
        const double Ri[3] = {R[i], R[N + i], R[2 * N + i]};
        const double li[3] = {lam[i], lam[N + i], lam[2 * N + i]};
        double Sm[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) Sm[k] = Sres[c * 9 + k];
        const double so2 = 0.5 / (C.cell.omega * fl.press);
        const int m = cnt[i];
        const int* row = nbr + (size_t)i * cap;
        for (int k = sub; k < m; k += G) {
            const int j = row[k];
            double r[3];
            const double d2 = pairvec_exact(C.cell, si1, si2, si3, sx[j], sy[j], sz[j], r[0], r[1], r[2]);
            if (d2 > C.rc2) continue;
            const int tj = type[j];
            const BPair& P = pc[ti * NT + tj];
            const double d = sqrt(d2);
            double v[NS];
#pragma unroll
            for (int s = 0; s < NS; ++s) v[s] = 0.0;
            if (d2 < C.rc2) {
                double rSr = 0.0;
#pragma unroll
                for (int a = 0; a < 3; ++a) rSr += r[a] * (Sm[a * 3] * r[0] + Sm[a * 3 + 1] * r[1] + Sm[a * 3 + 2] * r[2]);
                const double geo = Ri[0] * r[0] + Ri[1] * r[1] + Ri[2] * r[2] + so2 * rSr;
                if ((fl.bmh || fl.bmhftd) && P.A != 0.0) {
                    const double e1 = exp(-P.B * d), erh = P.A * e1;
                    const double d6 = 1.0 / (d2 * d2 * d2), d8 = d6 / d2;
                    double f6 = 1.0, f8 = 1.0, fd6 = 0.0, fd8 = 0.0, df6 = 0.0, df8 = 0.0, dfd6 = 0.0, dfd8 = 0.0;
                    if (fl.bmhftd) {
                        const TTD a6 = tt_deriv(P.BD, 1.0, d, 6), a8 = tt_deriv(P.BD, 1.0, d, 8);
                        f6 = 1.0 - a6.g; fd6 = a6.gd; df6 = -a6.g_b; dfd6 = a6.gd_b;
                        f8 = 1.0 - a8.g; fd8 = a8.gd; df8 = -a8.g_b; dfd8 = a8.gd_b;
                    }
                    v[0] = geo * P.B * e1 / d;
                    v[1] = geo * erh * (1.0 - P.B * d) / d;
                    v[2] = geo * (-6.0 * f6 * d6 / d + fd6 * d6) / d;
                    v[3] = geo * (-8.0 * f8 * d8 / d + fd8 * d8) / d;
                    if (fl.bmhftd)
                        v[4] = geo * (-6.0 * P.C * d6 / d * df6 - 8.0 * P.D * d8 / d * df8 + P.C * d6 * dfd6 + P.D * d8 * dfd8) / d;
                }
                if (fl.morse) {
                    const double e = exp(-d * P.rho) * P.rs;
                    v[5] = geo * 2.0 * P.rho * e * (e - 1.0) / d;
                    v[6] = geo * 2.0 * P.eps / d * (e * (e - 1.0) + P.rho * (P.sig - d) * e * (2.0 * e - 1.0));
                    v[7] = geo * 2.0 * P.eps * P.rho / d * P.rho * e * (2.0 * e - 1.0);
                }
            }
            if (fl.coul && P.ldamp) {
                const TTD Ti = tt_deriv(P.db_i, P.dc_i, d, P.dk_i);
                const double lr = (li[0] * r[0] + li[1] * r[1] + li[2] * r[2]) / (d * d2);
                v[8] = -q[j] * lr * Ti.g_b;
                v[9] = -q[j] * lr * Ti.g_c;
            }
#pragma unroll
            for (int t = 0; t < NTYB; ++t)
                if (t == tj)
#pragma unroll
                    for (int s = 0; s < NS; ++s) acc[t][s] += v[s];
        }
    }
    double v[NTYB * NTYB * NS];
#pragma unroll
    for (int a = 0; a < NTYB; ++a)
#pragma unroll
        for (int t = 0; t < NTYB; ++t)
#pragma unroll
            for (int s = 0; s < NS; ++s) v[(a * NTYB + t) * NS + s] = (active && a == ti) ? acc[t][s] : 0.0;
    block_partials<NTYB * NTYB * NS>(v, part);
}

// --------------------------------------------------------------------------
// reciprocal space
// --------------------------------------------------------------------------

// Pass 1: structure-factor partials of one chunk of atoms over its
// configuration's k rectangle.  One thread per (k-column, run of NZC nz);
// the phase e^{2 pi i n.s} of a run's first nz is the product X[nx] Y[ny]
// Z0[run] of per-atom tables in shared memory (one sincospi per atom and
// table entry, built by the block), then a rotation by e^{2 pi i s_z} per
// further nz.  Amplitudes:
//   MODE 0: q            MODE 1: i k.mu          MODE 2: q + i k.mu
//   MODE 3: (k.R)(q + i k.mu)   (the adjoint structure factor)
// Dynamic shared memory: CHUNK x phw_max double2 (the tables of the block's
// atoms, one row per atom: X[0..kx], Y[-ky..ky], Z0[run]).
template <int MODE>
__global__ void __launch_bounds__(KT) k_b_sfac(const BChunk* __restrict__ chunks, const BCfg* __restrict__ cf,
                                               const int* __restrict__ conv, int N, const double* __restrict__ sx,
                                               const double* __restrict__ sy, const double* __restrict__ sz,
                                               const double* __restrict__ q, const double* __restrict__ mu,
                                               const double* __restrict__ R, double* __restrict__ part_re,
                                               double* __restrict__ part_im) {
    __shared__ double t_q[CHUNK], t_cz[CHUNK], t_sn[CHUNK];
    __shared__ double t_u[3][CHUNK], t_v[3][CHUNK];
    extern __shared__ double2 t_ph[];
    const BChunk ch = chunks[blockIdx.x];
    if (conv && conv[ch.c]) return;
    const BCfg& C = cf[ch.c];
    const int kx = C.kmax[0], ky = C.kmax[1], kz = C.kmax[2];
    const int nzch = (C.nzl + NZC - 1) / NZC;
    const int W = (kx + 1) + (2 * ky + 1) + nzch;
    for (int a = threadIdx.x; a < ch.na; a += blockDim.x) {
        const int ia = ch.a0 + a;
        double sn, cs;
        sincospi(2.0 * sz[ia], &sn, &cs);
        t_cz[a] = cs; t_sn[a] = sn;
        t_q[a] = (MODE == 1) ? 0.0 : q[ia];
        double m0 = 0, m1 = 0, m2 = 0, r0 = 0, r1 = 0, r2 = 0;
        if (MODE != 0) { m0 = mu[ia]; m1 = mu[N + ia]; m2 = mu[2 * N + ia]; }
        if (MODE == 3) { r0 = R[ia]; r1 = R[N + ia]; r2 = R[2 * N + ia]; }
        // 2 pi b_d . v with b_d = column d of B: k.v = nx u0 + ny u1 + nz u2
        for (int dcol = 0; dcol < 3; ++dcol) {
            t_u[dcol][a] = 2.0 * PI * (C.cell.B[dcol] * m0 + C.cell.B[3 + dcol] * m1 + C.cell.B[6 + dcol] * m2);
            t_v[dcol][a] = 2.0 * PI * (C.cell.B[dcol] * r0 + C.cell.B[3 + dcol] * r1 + C.cell.B[6 + dcol] * r2);
        }
    }
    for (int t = threadIdx.x; t < ch.na * W; t += blockDim.x) {
        const int a = t / W, e = t % W, ia = ch.a0 + a;
        double arg;
        if (e <= kx) arg = (double)e * sx[ia];
        else if (e <= kx + 1 + 2 * ky) arg = (double)(e - (kx + 1) - ky) * sy[ia];
        else arg = (double)(-kz + (e - (kx + 2 + 2 * ky)) * NZC) * sz[ia];
        double sn, cs;
        sincospi(2.0 * arg, &sn, &cs);
        t_ph[t] = make_double2(cs, sn);
    }
    __syncthreads();
    const int items = C.ncol * nzch;
    double* pre = part_re + ch.poff;
    double* pim = part_im + ch.poff;
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
        const int col = it / nzch, zc = it % nzch;
        const int ix = col / (2 * ky + 1), iy = col % (2 * ky + 1);
        const double nx = (double)ix;
        const double ny = (double)(iy - ky);
        const int m0 = zc * NZC;
        const double nz0 = (double)(-kz + m0);
        const int ex = ix, ey = kx + 1 + iy, ez = kx + 2 + 2 * ky + zc;
        double are[NZC], aim[NZC];
#pragma unroll
        for (int m = 0; m < NZC; ++m) { are[m] = 0.0; aim[m] = 0.0; }
        for (int a = 0; a < ch.na; ++a) {
            const double2 X = t_ph[a * W + ex], Y = t_ph[a * W + ey], Z = t_ph[a * W + ez];
            const double xr = fma(X.x, Y.x, -X.y * Y.y), xi = fma(X.x, Y.y, X.y * Y.x);
            double er = fma(xr, Z.x, -xi * Z.y), ei = fma(xr, Z.y, xi * Z.x);
            const double rc = t_cz[a], rs = t_sn[a];
            const double qa = t_q[a];
            double km = nx * t_u[0][a] + ny * t_u[1][a] + nz0 * t_u[2][a];
            double kr = nx * t_v[0][a] + ny * t_v[1][a] + nz0 * t_v[2][a];
            const double du = t_u[2][a], dv = t_v[2][a];
#pragma unroll
            for (int m = 0; m < NZC; ++m) {
                double ar = qa, ai = km;
                if (MODE == 3) { ar *= kr; ai *= kr; }
                are[m] += ar * er - ai * ei;
                aim[m] += ar * ei + ai * er;
                const double t = er * rc - ei * rs;
                ei = er * rs + ei * rc;
                er = t;
                km += du;
                kr += dv;
            }
        }
        const int mlim = min(NZC, C.nzl - m0);
        for (int m = 0; m < mlim; ++m) {
            pre[(size_t)col * C.nzl + m0 + m] = are[m];
            pim[(size_t)col * C.nzl + m0 + m] = aim[m];
        }
    }
}

template <int MODE>
__global__ void k_b_sfac_reduce(int nrect_tot, const int* __restrict__ rcfg, const BCfg* __restrict__ cf,
                                const BChunk* __restrict__ chunks, const int* __restrict__ conv,
                                const double* __restrict__ part_re, const double* __restrict__ part_im,
                                const double* __restrict__ Ak, const double* __restrict__ kcoe,
                                const double* __restrict__ Sres, BFlags fl, double* rho_re, double* rho_im,
                                double* C_re, double* C_im) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nrect_tot) return;
    const int c = rcfg[e];
    if (conv && conv[c]) return;
    const BCfg& Cf = cf[c];
    const int l = e - Cf.roff;
    double sr = 0.0, si = 0.0;
    for (int ch = Cf.cs; ch < Cf.ce; ++ch) {
        const long o = chunks[ch].poff + l;
        sr += part_re[o];
        si += part_im[o];
    }
    const double A = Ak[e];
    if (MODE == 1) { rho_re[e] = sr; rho_im[e] = si; }
    if (MODE != 2) {
        C_re[e] = A * sr;
        C_im[e] = -A * si;
        return;
    }
    const int nzl = Cf.nzl, ky = Cf.kmax[1], kz = Cf.kmax[2];
    const int col = l / nzl;
    const double nx = (double)(col / (2 * ky + 1)), ny = (double)(col % (2 * ky + 1) - ky);
    const double nz = (double)(l % nzl - kz);
    const double* B = Cf.cell.B;
    const double k0 = 2.0 * PI * (nx * B[0] + ny * B[1] + nz * B[2]);
    const double k1 = 2.0 * PI * (nx * B[3] + ny * B[4] + nz * B[5]);
    const double k2 = 2.0 * PI * (nx * B[6] + ny * B[7] + nz * B[8]);
    const double* S = Sres + c * 9;
    const double kSk = k0 * (S[0] * k0 + S[1] * k1 + S[2] * k2) + k1 * (S[3] * k0 + S[4] * k1 + S[5] * k2) +
                       k2 * (S[6] * k0 + S[7] * k1 + S[8] * k2);
    const double sk = (S[0] + S[4] + S[8]) - kcoe[e] * kSk;
    const double tpi_V = 2.0 * PI / Cf.cell.omega;
    const double a1 = -2.0 * fl.cu * 2.0 * tpi_V;           // -2 cu fpi_V
    const double a2 = -2.0 * fl.cu / fl.press * 2.0 * tpi_V / Cf.cell.omega * sk;   // -2 c_s s_k
    // a1 i conj(sigma) = a1 (si + i sr);  a2 conj(rho)
    C_re[e] = A * (a1 * si + a2 * rho_re[e]);
    C_im[e] = A * (a1 * sr - a2 * rho_im[e]);
}

// Energy and stress sums of the final structure factor per configuration:
// out[c*8] = sum_k A|rho|^2, out[c*8+1..6] = sum_k (delta - kcoe k k) A |rho|^2
// (xx yy zz xy xz yz), over the half mesh.
__global__ void k_b_rec_sums(const BCfg* __restrict__ cf, const double* __restrict__ rho_re,
                             const double* __restrict__ rho_im, const double* __restrict__ Ak,
                             const double* __restrict__ kcoe, double* out) {
    const BCfg& Cf = cf[blockIdx.x];
    double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const int ky = Cf.kmax[1], kz = Cf.kmax[2];
    const double* B = Cf.cell.B;
    for (int l = threadIdx.x; l < Cf.nrect; l += blockDim.x) {
        const int e = Cf.roff + l;
        const double str = Ak[e] * (rho_re[e] * rho_re[e] + rho_im[e] * rho_im[e]);
        if (str == 0.0) continue;
        const int col = l / Cf.nzl;
        const double nx = (double)(col / (2 * ky + 1)), ny = (double)(col % (2 * ky + 1) - ky);
        const double nz = (double)(l % Cf.nzl - kz);
        const double k[3] = {2.0 * PI * (nx * B[0] + ny * B[1] + nz * B[2]), 2.0 * PI * (nx * B[3] + ny * B[4] + nz * B[5]),
                             2.0 * PI * (nx * B[6] + ny * B[7] + nz * B[8])};
        const double kc = kcoe[e];
        v[0] += str;
        v[1] += (1.0 - kc * k[0] * k[0]) * str;
        v[2] += (1.0 - kc * k[1] * k[1]) * str;
        v[3] += (1.0 - kc * k[2] * k[2]) * str;
        v[4] += -kc * k[0] * k[1] * str;
        v[5] += -kc * k[0] * k[2] * str;
        v[6] += -kc * k[1] * k[2] * str;
    }
    // block sum in fixed order (block = configuration)
    __shared__ double red[32][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        double s = warp_sum(v[k]);
        if (lane == 0) red[warp][k] = s;
    }
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            double s = lane < nw ? red[lane][k] : 0.0;
            s = warp_sum(s);
            if (lane == 0) out[blockIdx.x * 8 + k] = s;
        }
    }
}

// Pass 2: per atom of the chunk, V = scale sum_k k Im(C_k e^{ik.r}) and, with
// GRAD, G = scale sum_k k k^T Re(C_k e^{ik.r}) (xx yy zz xy xz yz).  scale is
// 2 fpi_V of the configuration when SCALE_FPI, else 1.  V is written, or added
// with ADD.
template <int GRAD, int ADD, int SCALE_FPI>
__global__ void __launch_bounds__(KT * KF_LPA) k_b_kfield(const BChunk* __restrict__ chunks, const BCfg* __restrict__ cf,
                                                 const int* __restrict__ conv, int N, const double* __restrict__ sx,
                                                 const double* __restrict__ sy, const double* __restrict__ sz,
                                                 const double* __restrict__ C_re, const double* __restrict__ C_im,
                                                 double* __restrict__ V, double* __restrict__ Gout) {
    extern __shared__ double smem[];
    const BChunk ch = chunks[blockIdx.x];
    if (conv && conv[ch.c]) return;
    const BCfg& C = cf[ch.c];
    const int nzl = C.nzl, ky = C.kmax[1], kz = C.kmax[2];
    double* t_re = smem;
    double* t_im = smem + CT * nzl;
    const int t = threadIdx.x / KF_LPA, sub = threadIdx.x % KF_LPA;   // atom, lane among the atom's
    const bool active = t < ch.na;
    const int ia = ch.a0 + (active ? t : 0);
    const double s1 = sx[ia], s2 = sy[ia], s3 = sz[ia];
    double rs, rc;
    sincospi(2.0 * s3, &rs, &rc);
    const double* B = C.cell.B;
    const double bz0 = 2.0 * PI * B[2], bz1 = 2.0 * PI * B[5], bz2 = 2.0 * PI * B[8];
    double E0 = 0, E1 = 0, E2 = 0, G[6] = {0, 0, 0, 0, 0, 0};
    for (int c0 = 0; c0 < C.ncol; c0 += CT) {
        const int nc = min(CT, C.ncol - c0);
        __syncthreads();
        for (int k = threadIdx.x; k < nc * nzl; k += blockDim.x) {
            const int e = C.roff + c0 * nzl + k;
            t_re[k] = C_re[e];
            t_im[k] = C_im[e];
        }
        __syncthreads();
        if (!active) continue;
        for (int cc = sub; cc < nc; cc += KF_LPA) {
            const int col = c0 + cc;
            const double nx = (double)(col / (2 * ky + 1)), ny = (double)(col % (2 * ky + 1) - ky);
            double sn, cs;
            sincospi(2.0 * (nx * s1 + ny * s2 - (double)kz * s3), &sn, &cs);
            double er = cs, ei = sn;
            double k0 = 2.0 * PI * (nx * B[0] + ny * B[1]) - (double)kz * bz0;
            double k1 = 2.0 * PI * (nx * B[3] + ny * B[4]) - (double)kz * bz1;
            double k2 = 2.0 * PI * (nx * B[6] + ny * B[7]) - (double)kz * bz2;
            const double* cr = t_re + cc * nzl;
            const double* ci = t_im + cc * nzl;
            for (int m = 0; m < nzl; ++m) {
                const double zr = cr[m] * er - ci[m] * ei;
                const double zi = cr[m] * ei + ci[m] * er;
                E0 += k0 * zi; E1 += k1 * zi; E2 += k2 * zi;
                if (GRAD) {
                    G[0] += k0 * k0 * zr; G[1] += k1 * k1 * zr; G[2] += k2 * k2 * zr;
                    G[3] += k0 * k1 * zr; G[4] += k0 * k2 * zr; G[5] += k1 * k2 * zr;
                }
                const double tt = er * rc - ei * rs;
                ei = er * rs + ei * rc;
                er = tt;
                k0 += bz0; k1 += bz1; k2 += bz2;
            }
        }
    }
    // the atom's lanes are adjacent: sum them by a fixed xor tree
#pragma unroll
    for (int o = 1; o < KF_LPA; o <<= 1) {
        E0 += __shfl_xor_sync(0xffffffffu, E0, o);
        E1 += __shfl_xor_sync(0xffffffffu, E1, o);
        E2 += __shfl_xor_sync(0xffffffffu, E2, o);
        if (GRAD)
            for (int k = 0; k < 6; ++k) G[k] += __shfl_xor_sync(0xffffffffu, G[k], o);
    }
    if (!active || sub != 0) return;
    const double sc = SCALE_FPI ? 2.0 * (4.0 * PI / C.cell.omega) : 1.0;
    if (ADD) {
        V[ia] += sc * E0; V[N + ia] += sc * E1; V[2 * N + ia] += sc * E2;
    } else {
        V[ia] = sc * E0; V[N + ia] = sc * E1; V[2 * N + ia] = sc * E2;
    }
    if (GRAD)
        for (int k = 0; k < 6; ++k) Gout[(size_t)k * N + ia] = sc * G[k];
}

// --------------------------------------------------------------------------
// vectors, per-configuration sums
// --------------------------------------------------------------------------

struct SegTerm { const double* a; const double* b; int ncomp; };
struct SegSpec { SegTerm t[8]; };

// out[c*K + k] = sum over atoms of configuration c (and components) of
// a*b (or a); one block per configuration, fixed reduction order.
template <int K>
__global__ void k_b_segsum(SegSpec sp, const BCfg* __restrict__ cf, int N, double* out) {
    const BCfg& C = cf[blockIdx.x];
    double v[K];
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = 0.0;
    for (int a = threadIdx.x; a < C.n; a += blockDim.x) {
        const int i = C.off + a;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const SegTerm& T = sp.t[k];
            for (int cmp = 0; cmp < T.ncomp; ++cmp) {
                const size_t o = (size_t)cmp * N + i;
                v[k] += T.b ? T.a[o] * T.b[o] : T.a[o];
            }
        }
    }
    __shared__ double red[32][K];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = warp_sum(v[k]);
        if (lane == 0) red[warp][k] = s;
    }
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double s = lane < nw ? red[lane][k] : 0.0;
            s = warp_sum(s);
            if (lane == 0) out[blockIdx.x * K + k] = s;
        }
    }
}

// PCG (Jacobi preconditioner M^-1 = alpha) on every configuration at once.
// x0 = alpha b on polarisable atoms.
__global__ void k_b_cg_x0(int N, const double* __restrict__ b, const double* __restrict__ alpha, double* x) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * N) return;
    x[t] = alpha[t % N] * b[t];
}

// Ad = v/alpha - (E + 2 selfa2 v) on polarisable atoms, 0 elsewhere.
__global__ void k_b_apply_A(int N, const int* __restrict__ cfg_of, const BCfg* __restrict__ cf,
                            const int* __restrict__ conv, const double* __restrict__ v, const double* __restrict__ E,
                            const double* __restrict__ inv_alpha, double* Ad) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * N) return;
    const int i = t % N;
    const int c = cfg_of[i];
    if (conv && conv[c]) return;
    const double ia = inv_alpha[i];
    Ad[t] = ia != 0.0 ? v[t] * ia - (E[t] + 2.0 * cf[c].selfa2 * v[t]) : 0.0;
}

// r = b - Ax, z = alpha r, d = z on polarisable atoms.
__global__ void k_b_cg_init(int N, const double* __restrict__ b, const double* __restrict__ Ax,
                            const double* __restrict__ alpha, const double* __restrict__ inv_alpha, double* r,
                            double* z, double* d) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * N) return;
    const int i = t % N;
    const double rr = inv_alpha[i] != 0.0 ? b[t] - Ax[t] : 0.0;
    r[t] = rr;
    z[t] = alpha[i] * rr;
    d[t] = alpha[i] * rr;
}

struct BScal {
    double rr, rz, rz_new, dAd, beta, rmsd;
    int iter, pad;
};

// After the first reduction: rmsd and the convergence flag.
__global__ void k_b_cg_first(int nconf, const BCfg* __restrict__ cf, const double* __restrict__ red2, BScal* sc,
                             int* conv, double tol) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nconf) return;
    BScal& s = sc[c];
    s.rr = red2[2 * c];
    s.rz = red2[2 * c + 1];
    s.iter = 0;
    s.rmsd = cf[c].npol > 0 ? sqrt(s.rr / cf[c].npol) : 0.0;
    conv[c] = !(s.rmsd > tol);
}

// x += a d, r -= a Ad, z = alpha r with a = rz/dAd of the configuration.
__global__ void k_b_cg_update(int N, const int* __restrict__ cfg_of, const int* __restrict__ conv,
                              const BScal* __restrict__ sc, const double* __restrict__ dAd, const double* __restrict__ d,
                              const double* __restrict__ Ad, const double* __restrict__ alpha, double* x, double* r,
                              double* z) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * N) return;
    const int i = t % N;
    const int c = cfg_of[i];
    if (conv[c]) return;
    const double a = sc[c].rz / dAd[c];
    x[t] = fma(a, d[t], x[t]);
    const double rr = fma(-a, Ad[t], r[t]);
    r[t] = rr;
    z[t] = alpha[i] * rr;
}

__global__ void k_b_cg_scalars(int nconf, const BCfg* __restrict__ cf, const double* __restrict__ red2, BScal* sc,
                               int* conv, double tol) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nconf || conv[c]) return;
    BScal& s = sc[c];
    s.rr = red2[2 * c];
    s.rz_new = red2[2 * c + 1];
    s.beta = s.rz_new / s.rz;
    s.rz = s.rz_new;
    s.rmsd = sqrt(s.rr / cf[c].npol);
    s.iter += 1;
    conv[c] = !(s.rmsd > tol);
}

__global__ void k_b_cg_direction(int N, const int* __restrict__ cfg_of, const int* __restrict__ conv,
                                 const BScal* __restrict__ sc, const double* __restrict__ z, double* d) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * N) return;
    const int c = cfg_of[t % N];
    if (conv[c]) return;
    d[t] = fma(sc[c].beta, d[t], z[t]);
}

// Total forces: f = f_pair + cu (f_dir + q E_rec + G mu); G kept for the adjoint.
__global__ void k_b_forces(int N, const double* __restrict__ fp, const double* __restrict__ fd,
                           const double* __restrict__ Erec, const double* __restrict__ G, const double* __restrict__ q,
                           const double* __restrict__ mu, double cu, int coul, double* f) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    if (!coul) {
        for (int c = 0; c < 3; ++c) f[(size_t)c * N + i] = fp[(size_t)c * N + i];
        return;
    }
    const double m[3] = {mu[i], mu[N + i], mu[2 * N + i]};
    const double g[6] = {G[i], G[N + i], G[2 * N + i], G[3 * N + i], G[4 * N + i], G[5 * N + i]};
    const double Gm[3] = {g[0] * m[0] + g[3] * m[1] + g[4] * m[2], g[3] * m[0] + g[1] * m[1] + g[5] * m[2],
                          g[4] * m[0] + g[5] * m[1] + g[2] * m[2]};
    for (int c = 0; c < 3; ++c) {
        const size_t o = (size_t)c * N + i;
        f[o] = fp[o] + cu * (fd[o] + q[i] * Erec[o] + Gm[c]);
    }
}

// R = 2 cF (F - F*), per-atom loss cF |F - F*|^2.
__global__ void k_b_residual(int N, const int* __restrict__ cfg_of, const BCfg* __restrict__ cf,
                             const double* __restrict__ f, const double* __restrict__ ft, double* R, double* lossa) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double cF = cf[cfg_of[i]].cF;
    double l = 0.0;
    for (int c = 0; c < 3; ++c) {
        const size_t o = (size_t)c * N + i;
        const double dl = f[o] - ft[o];
        R[o] = 2.0 * cF * dl;
        l += cF * dl * dl;
    }
    lossa[i] = l;
}

// h += cu G R (the field-gradient term of the reciprocal adjoint), masked to
// polarisable atoms.
__global__ void k_b_h_finish(int N, const double* __restrict__ G, const double* __restrict__ R,
                             const double* __restrict__ inv_alpha, double cu, double* h) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    if (inv_alpha[i] == 0.0) {
        h[i] = h[N + i] = h[2 * N + i] = 0.0;
        return;
    }
    const double r[3] = {R[i], R[N + i], R[2 * N + i]};
    const double g[6] = {G[i], G[N + i], G[2 * N + i], G[3 * N + i], G[4 * N + i], G[5 * N + i]};
    h[i] += cu * (g[0] * r[0] + g[3] * r[1] + g[4] * r[2]);
    h[N + i] += cu * (g[3] * r[0] + g[1] * r[1] + g[5] * r[2]);
    h[2 * N + i] += cu * (g[4] * r[0] + g[5] * r[1] + g[2] * r[2]);
}

// out[k] = sum_b buf[b*K + k] for any K: one warp per k, lanes stride over
// the blocks, fixed shuffle tree.
__global__ void k_b_reduce_cols(const double* __restrict__ buf, int nblocks, int K, double* out) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int k = blockIdx.x * (blockDim.x >> 5) + warp;
    if (k >= K) return;
    double s = 0.0;
    for (int b = lane; b < nblocks; b += 32) s += buf[(size_t)b * K + k];
    s = warp_sum(s);
    if (lane == 0) out[k] = s;
}

// d L / d alpha_t = sum over type-t atoms of lambda.mu / alpha^2.
__global__ void k_b_alpha_grad(int N, const int* __restrict__ type, const double* __restrict__ lam,
                               const double* __restrict__ mu, const double* __restrict__ inv_alpha, double* part) {
    double v[NTYB];
#pragma unroll
    for (int t = 0; t < NTYB; ++t) v[t] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const double ia = inv_alpha[i];
        if (ia == 0.0) continue;
        const double s = (lam[i] * mu[i] + lam[N + i] * mu[N + i] + lam[2 * N + i] * mu[2 * N + i]) * ia * ia;
        const int ti = type[i];
#pragma unroll
        for (int t = 0; t < NTYB; ++t)
            if (t == ti) v[t] += s;
    }
    block_partials<NTYB>(v, part);
}

// Condition of the lockstep PCG loop (a conditional WHILE node of the batch's
// CUDA graph): iterate while some configuration has not converged and fewer
// than max_it iterations have run.  reset != 0 starts the count (before the
// loop); otherwise one iteration has just finished.  The cap makes the loop
// finite whatever the residuals do.
__global__ void k_b_cg_cond(int nconf, const int* __restrict__ conv, int* loop_it, int max_it, int reset,
                            cudaGraphConditionalHandle h) {
    __shared__ int open_;
    if (threadIdx.x == 0) open_ = 0;
    __syncthreads();
    for (int c = threadIdx.x; c < nconf; c += blockDim.x)
        if (!conv[c]) open_ = 1;
    __syncthreads();
    if (threadIdx.x == 0) {
        const int it = reset ? 0 : *loop_it + 1;
        *loop_it = it;
        cudaGraphSetConditional(h, (open_ && it < max_it) ? 1u : 0u);
    }
}

// After a solve: out[0] = largest iteration count, out[1] = configurations
// not converged.
__global__ void k_b_cg_summary(int nconf, const int* __restrict__ conv, const BScal* __restrict__ sc, int* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int it = 0, bad = 0;
    for (int c = 0; c < nconf; ++c) {
        it = max(it, sc[c].iter);
        bad += conv[c] ? 0 : 1;
    }
    out[0] = it;
    out[1] = bad;
}

// Per configuration: total stress tau = tau_nonb + tau_coul (GPa, column-major,
// the assembly of engforce: pair sums / omega / press; real-space sums
// 0.25/omega and reciprocal sums 2 tpi_V/omega, times cu / press), the loss
// cF sum|dF|^2 + cS sum dtau^2 and S = dL/dtau (symmetrised).
__global__ void k_b_loss_tail(int nconf, const BCfg* __restrict__ cf, const double* __restrict__ red_pair,
                              const double* __restrict__ red_dir, const double* __restrict__ red_rec,
                              const double* __restrict__ lossF, const double* __restrict__ tau_t, double cu,
                              double press, int coul, double* loss_c, double* tau_c, double* Sres) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nconf) return;
    const BCfg& C = cf[c];
    const double om = C.cell.omega, tpi_V = 2.0 * PI / om;
    const int map[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
    double tau[9];
    for (int k = 0; k < 6; ++k) {
        double v = red_pair[7 * c + 1 + k] / om / press;
        if (coul) v += (red_dir[7 * c + 1 + k] * 0.25 / om + red_rec[8 * c + 1 + k] * 2.0 * tpi_V / om) * cu / press;
        tau[3 * map[k][1] + map[k][0]] = v;
        tau[3 * map[k][0] + map[k][1]] = v;
    }
    double L = lossF[c], D[9];
    for (int k = 0; k < 9; ++k) {
        D[k] = tau[k] - tau_t[9 * c + k];
        L += C.cS * D[k] * D[k];
        tau_c[9 * c + k] = tau[k];
    }
    for (int a = 0; a < 3; ++a)
        for (int bb = 0; bb < 3; ++bb) Sres[9 * c + 3 * a + bb] = C.cS * (D[3 * a + bb] + D[3 * bb + a]);
    loss_c[c] = L;
}

}  // namespace

// ==========================================================================
// host
// ==========================================================================

struct mdff_batch {
    mdff_params p;
    std::string err;
    cudaStream_t st = nullptr;
    std::vector<void*> allocs;
    double cu = 1.0, press = 1.0;
    int nconf = 0, N = 0, ntype = 0;
    BFlags fl;
    std::vector<BCfg> hcfg;
    std::vector<BChunk> hchunk;
    BCfg* cfg = nullptr;
    BChunk* chunk = nullptr;
    int nchunk = 0;
    long part_len = 0;
    int nrect_tot = 0, nzl_max = 1;
    int phw_max = 1;       // widest per-atom phase table of the structure factor (X, Y, Z0 entries)
    int* rcfg = nullptr;
    int* cfg_of = nullptr;
    int* type = nullptr;
    double *x = nullptr, *y = nullptr, *z = nullptr, *sx = nullptr, *sy = nullptr, *sz = nullptr;
    double *q = nullptr, *alpha = nullptr, *inv_alpha = nullptr;
    int *nbr = nullptr, *cnt = nullptr, cap = 0;
    int* overflow = nullptr;
    BPair* pc = nullptr;
    double *Ak = nullptr, *kcoe = nullptr;
    double *rho_re = nullptr, *rho_im = nullptr, *C_re = nullptr, *C_im = nullptr;
    double *part_re = nullptr, *part_im = nullptr;
    // per-atom vectors
    double *f = nullptr, *fpair = nullptr, *fdir = nullptr, *Erec = nullptr, *G = nullptr;
    double *Estat = nullptr, *mu = nullptr, *Eind = nullptr;
    double *cg_r = nullptr, *cg_z = nullptr, *cg_d = nullptr, *cg_Ad = nullptr;
    double *h = nullptr, *lam = nullptr, *R = nullptr, *ft = nullptr;
    double *e_pair = nullptr, *s_pair = nullptr, *e_dir = nullptr, *s_dir = nullptr, *lossa = nullptr;
    // per configuration
    int* conv = nullptr;
    BScal* sc = nullptr;
    double* red = nullptr;       // [nconf][8] scratch of the per-configuration sums
    double* Sres = nullptr;      // [nconf][9] dL/dtau
    double* gpart = nullptr;     // block partials of the gradient kernels
    int gpart_cap = 0;
    double* gsum = nullptr;      // reduced gradient slots
    std::vector<double> tau_t;   // targets [nconf][9] (column-major per configuration)
    double w_force = 1.0, w_stress = 0.0;
    bool have_targets = false;
    // results of the last forward evaluation
    std::vector<double> tau;     // [nconf][9] total stress, column-major
    std::vector<double> energy;  // [nconf]
    int fwd_iters = 0, adj_iters = 0;
    std::vector<int> hconv;
    // the loss + gradient evaluation as one CUDA graph (built on first use and
    // whenever the flags of the force field change)
    cudaStream_t st2 = nullptr;          // stream used to capture the loop bodies
    cudaGraphExec_t gexec = nullptr, gexec_loss = nullptr;   // loss + gradient; loss only
    cudaGraph_t graph = nullptr, graph_loss = nullptr;
    BFlags gflags[2];                    // flags each graph was built with
    bool gpol[2] = {false, false};
    cudaGraphConditionalHandle hcond[2] = {0, 0};
    int* loop_it = nullptr;              // device loop counter of the running solve
    int* solve_out = nullptr;            // [4]: forward iterations, not converged; adjoint iterations, not converged
    double* tau_t_dev = nullptr;         // [nconf][9]
    double* loss_c = nullptr;            // [nconf]
    double* tau_c = nullptr;             // [nconf][9]
    // the dipole operator's pair table (k_b_ddtab_build), FP64 or FP32
    int *dd_nbr = nullptr, *dd_cnt = nullptr;
    double* dd64 = nullptr;
    float* dd32 = nullptr;
    int dd_ref = -1;                     // erfc_ref the table was built with
    int g_dd = 16;                       // lanes per atom of the table operator (autotuned)
    float dd_ms[4] = {0, 0, 0, 0};       // the autotuner's timings for 4, 8, 16, 32 lanes
};

namespace {

int bfail(mdff_batch* b, int code, const std::string& m) {
    if (b) b->err = m;
    return code;
}

#define BCK(call)                                                                                     \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) return bfail(b, MDFF_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)
#define BTRY(expr)                    \
    do {                              \
        int r_ = (expr);              \
        if (r_ != MDFF_OK) return r_; \
    } while (0)

template <class T>
int balloc(mdff_batch* b, T** ptr, size_t count) {
    if (count == 0) count = 1;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, sizeof(T) * count);
    if (e != cudaSuccess) return bfail(b, MDFF_E_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    b->allocs.push_back(p);
    *ptr = (T*)p;
    return MDFF_OK;
}

int blaunch(mdff_batch* b, const char* where) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return bfail(b, MDFF_E_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
    return MDFF_OK;
}

void lattice9(const double A9[9], CellP& c, double W[3]) {
    double A[3][3], Bm[3][3];
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) A[i][j] = A9[3 * j + i];
    auto expro = [&](int out, int a, int bb) {
        Bm[0][out] = A[1][a] * A[2][bb] - A[2][a] * A[1][bb];
        Bm[1][out] = A[2][a] * A[0][bb] - A[0][a] * A[2][bb];
        Bm[2][out] = A[0][a] * A[1][bb] - A[1][a] * A[0][bb];
    };
    expro(0, 1, 2);
    expro(1, 2, 0);
    expro(2, 0, 1);
    double omega = Bm[0][0] * A[0][0] + Bm[1][0] * A[1][0] + Bm[2][0] * A[2][0];
    for (int j = 0; j < 3; ++j) W[j] = omega / std::sqrt(Bm[0][j] * Bm[0][j] + Bm[1][j] * Bm[1][j] + Bm[2][j] * Bm[2][j]);
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) { c.A[3 * i + j] = A[i][j]; c.B[3 * i + j] = Bm[i][j] / omega; }
    c.omega = omega;
}

void symmetrise_tables(mdff_params& p) {   // field_check_tag (src/field.f90:316-339)
    if (!p.symmetric_pot) return;
    const int n = p.ntype;
    for (int it = 0; it < n; ++it)
        for (int jt = 0; jt < n; ++jt) {
            p.Abmhftd[jt][it] = p.Abmhftd[it][jt];
            p.Bbmhftd[jt][it] = p.Bbmhftd[it][jt];
            p.Cbmhftd[jt][it] = p.Cbmhftd[it][jt];
            p.Dbmhftd[jt][it] = p.Dbmhftd[it][jt];
            p.BDbmhftd[jt][it] = p.BDbmhftd[it][jt];
            p.epsmor[jt][it] = p.epsmor[it][jt];
            p.sigmamor[jt][it] = p.sigmamor[it][jt];
            p.rhomor[jt][it] = p.rhomor[it][jt];
            for (int k = 0; k < n; ++k) {
                p.ldip_damping[k][jt][it] = p.ldip_damping[k][it][jt];
                p.dip_pol_damp_b[k][jt][it] = p.dip_pol_damp_b[k][it][jt];
                p.dip_pol_damp_c[k][jt][it] = p.dip_pol_damp_c[k][it][jt];
                p.dip_pol_damp_k[k][jt][it] = p.dip_pol_damp_k[k][it][jt];
            }
        }
}

int check_batch_params(mdff_batch* b, const mdff_params& p) {
    if (p.ntype < 1 || p.ntype > NTYB)
        return bfail(b, MDFF_E_UNSUPPORTED, "batch path: ntype must be 1 or 2");
    if (p.lnmlj) return bfail(b, MDFF_E_UNSUPPORTED, "batch path: Lennard-Jones is not on the force-matching path");
    if (p.lsurf) return bfail(b, MDFF_E_UNSUPPORTED, "batch path: lsurf is not supported");
    for (int t = 0; t < p.ntype; ++t)
        for (int c = 0; c < 3; ++c)
            if (p.dip[t][c] != 0.0) return bfail(b, MDFF_E_UNSUPPORTED, "batch path: static dipoles are not supported");
    for (int a = 0; a < p.ntype; ++a)
        for (int bb = 0; bb < p.ntype; ++bb)
            for (int c = 0; c < p.ntype; ++c)
                if (p.dip_pol_damp_k[a][bb][c] > MDFF_TT_MAX_ORDER || p.dip_pol_damp_k[a][bb][c] < 0)
                    return bfail(b, MDFF_E_ARG, "Tang-Toennies expansion order too large (dip_pol_damp_k)");
    if (p.conv_tol_ind <= 0.0 || p.max_scf_pol_iter < 1) return bfail(b, MDFF_E_ARG, "conv_tol_ind / max_scf_pol_iter");
    return MDFF_OK;
}

// Pair constants of the (symmetrised) tables; per ordered pair (ti,tj).
int upload_params(mdff_batch* b, const mdff_params& pin) {
    BTRY(check_batch_params(b, pin));
    if (pin.ntype != b->ntype) return bfail(b, MDFF_E_ARG, "batch: ntype differs from the batch's");
    mdff_params p = pin;
    symmetrise_tables(p);
    b->p = p;
    std::vector<BPair> tab(NT * NT);
    std::memset(tab.data(), 0, sizeof(BPair) * NT * NT);
    for (int it = 0; it < p.ntype; ++it)
        for (int jt = 0; jt < p.ntype; ++jt) {
            BPair& P = tab[it * NT + jt];
            P.A = p.Abmhftd[it][jt]; P.B = p.Bbmhftd[it][jt]; P.C = p.Cbmhftd[it][jt]; P.D = p.Dbmhftd[it][jt];
            P.BD = p.BDbmhftd[it][jt];
            P.eps = p.epsmor[it][jt]; P.rho = p.rhomor[it][jt]; P.sig = p.sigmamor[it][jt];
            P.rs = std::exp(p.rhomor[it][jt] * p.sigmamor[it][jt]);
            P.db_i = p.dip_pol_damp_b[it][it][jt]; P.dc_i = p.dip_pol_damp_c[it][it][jt]; P.dk_i = p.dip_pol_damp_k[it][it][jt];
            P.db_j = p.dip_pol_damp_b[jt][it][jt]; P.dc_j = p.dip_pol_damp_c[jt][it][jt]; P.dk_j = p.dip_pol_damp_k[jt][it][jt];
            P.ldamp = (p.lcoulomb && (p.ldip_damping[it][it][jt] || p.ldip_damping[jt][it][jt])) ? 1 : 0;
        }
    BCK(cudaMemcpyAsync(b->pc, tab.data(), sizeof(BPair) * NT * NT, cudaMemcpyHostToDevice, b->st));
    // per-atom polarisabilities and charges
    std::vector<int> ht(b->N);
    BCK(cudaMemcpyAsync(ht.data(), b->type, sizeof(int) * b->N, cudaMemcpyDeviceToHost, b->st));
    BCK(cudaStreamSynchronize(b->st));
    std::vector<double> hq(b->N), ha(b->N), hia(b->N);
    for (int i = 0; i < b->N; ++i) {
        int t = ht[i];
        hq[i] = p.qch[t];
        ha[i] = p.ldip_polar[t] ? p.poldip_iso[t] : 0.0;
        hia[i] = ha[i] != 0.0 ? 1.0 / ha[i] : 0.0;
    }
    for (auto& C : b->hcfg) {
        C.npol = 0;
        for (int i = C.off; i < C.off + C.n; ++i) if (hia[i] != 0.0) C.npol++;
    }
    BCK(cudaMemcpyAsync(b->q, hq.data(), sizeof(double) * b->N, cudaMemcpyHostToDevice, b->st));
    BCK(cudaMemcpyAsync(b->alpha, ha.data(), sizeof(double) * b->N, cudaMemcpyHostToDevice, b->st));
    BCK(cudaMemcpyAsync(b->inv_alpha, hia.data(), sizeof(double) * b->N, cudaMemcpyHostToDevice, b->st));
    BCK(cudaMemcpyAsync(b->cfg, b->hcfg.data(), sizeof(BCfg) * b->nconf, cudaMemcpyHostToDevice, b->st));
    b->fl.bmh = p.lbmhft;
    b->fl.bmhftd = p.lbmhftd;
    b->fl.morse = p.lmorse;
    b->fl.coul = p.lcoulomb;
    b->fl.erfc_ref = p.erfc_ref;
    b->fl.cu = b->cu;
    b->fl.press = b->press;
    BCK(cudaStreamSynchronize(b->st));
    return MDFF_OK;
}

// Structure factor of the amplitudes MODE into the chunk partials, then the
// coefficients C_k (RMODE of k_b_sfac_reduce).
template <int MODE, int RMODE>
int structure_factor(mdff_batch* b, const int* conv, const double* mu) {
    const size_t sm = sizeof(double2) * (size_t)CHUNK * b->phw_max;
    k_b_sfac<MODE><<<b->nchunk, KT, sm, b->st>>>(b->chunk, b->cfg, conv, b->N, b->sx, b->sy, b->sz, b->q, mu, b->R,
                                                 b->part_re, b->part_im);
    k_b_sfac_reduce<RMODE><<<nblk(b->nrect_tot, 256), 256, 0, b->st>>>(b->nrect_tot, b->rcfg, b->cfg, b->chunk, conv,
                                                                       b->part_re, b->part_im, b->Ak, b->kcoe, b->Sres,
                                                                       b->fl, b->rho_re, b->rho_im, b->C_re, b->C_im);
    return blaunch(b, "structure factor");
}

template <int GRAD, int ADD, int SCALE>
int kfield(mdff_batch* b, const int* conv, double* V, double* G) {
    size_t sm = sizeof(double) * 2 * CT * b->nzl_max;
    k_b_kfield<GRAD, ADD, SCALE><<<b->nchunk, KT * KF_LPA, sm, b->st>>>(b->chunk, b->cfg, conv, b->N, b->sx, b->sy,
                                                                        b->sz, b->C_re, b->C_im, V, G);
    return blaunch(b, "kfield");
}

int dir_blocks(int N, int G) { return nblk((long)N * G, 256); }

// The real-space part of the dipole operator from the pair table, with G
// lanes per atom.
void launch_ddtab(mdff_batch* b, int g, const double* v, double* E) {
    const int blocks = dir_blocks(b->N, g);
#define DDT(GG)                                                                                                    \
    do {                                                                                                           \
        if (b->dd32)                                                                                               \
            k_b_ddtab<GG, float><<<blocks, 256, 0, b->st>>>(b->N, b->cfg_of, b->conv, b->dd_nbr, b->dd_cnt, b->cap, \
                                                            b->dd32, v, E);                                        \
        else                                                                                                       \
            k_b_ddtab<GG, double><<<blocks, 256, 0, b->st>>>(b->N, b->cfg_of, b->conv, b->dd_nbr, b->dd_cnt,      \
                                                             b->cap, b->dd64, v, E);                               \
    } while (0)
    if (g == 4) DDT(4);
    else if (g == 8) DDT(8);
    else if (g == 32) DDT(32);
    else DDT(16);
#undef DDT
}

// The pair table of the dipole operator (positions and alpha are fixed for the
// batch's life; erfc_ref follows the parameters), then the autotuner's choice
// of lanes per atom for it: each candidate timed over three launches after a
// warm-up, with CUDA events on the batch's stream.
int build_ddtab(mdff_batch* b) {
    const int N = b->N;
    const bool mixed = b->p.precision == MDFF_PREC_MIXED;
    const size_t NC = (size_t)N * b->cap;
    if (!b->dd_nbr) {
        BTRY(balloc(b, &b->dd_nbr, NC));
        BTRY(balloc(b, &b->dd_cnt, (size_t)N));
        if (mixed) BTRY(balloc(b, &b->dd32, 5 * NC));
        else BTRY(balloc(b, &b->dd64, 5 * NC));
    }
    const int er = b->fl.erfc_ref;
    if (mixed)
        k_b_ddtab_build<16, float><<<dir_blocks(N, 16), 256, 0, b->st>>>(N, b->cfg_of, b->cfg, b->sx, b->sy, b->sz,
                                                                         b->nbr, b->cnt, b->cap, er, b->dd_nbr,
                                                                         b->dd_cnt, b->dd32);
    else
        k_b_ddtab_build<16, double><<<dir_blocks(N, 16), 256, 0, b->st>>>(N, b->cfg_of, b->cfg, b->sx, b->sy, b->sz,
                                                                          b->nbr, b->cnt, b->cap, er, b->dd_nbr,
                                                                          b->dd_cnt, b->dd64);
    BTRY(blaunch(b, "dd table"));
    b->dd_ref = er;
    BCK(cudaMemsetAsync(b->cg_d, 0, sizeof(double) * 3 * N, b->st));
    cudaEvent_t e0, e1;
    BCK(cudaEventCreate(&e0));
    BCK(cudaEventCreate(&e1));
    const int gs[4] = {4, 8, 16, 32};
    float best = 1e30f;
    for (int k = 0; k < 4; ++k) {
        launch_ddtab(b, gs[k], b->cg_d, b->Eind);
        cudaEventRecord(e0, b->st);
        for (int r = 0; r < 3; ++r) launch_ddtab(b, gs[k], b->cg_d, b->Eind);
        cudaEventRecord(e1, b->st);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        b->dd_ms[k] = ms / 3.f;
        if (ms < best) { best = ms; b->g_dd = gs[k]; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return blaunch(b, "dd table autotune");
}

// E = T v (undamped dipole field, real + reciprocal; self term in apply_A).
int dd_field(mdff_batch* b, const double* v, double* E) {
    launch_ddtab(b, b->g_dd, v, E);
    BTRY(blaunch(b, "dd field"));
    BTRY((structure_factor<1, 0>(b, b->conv, v)));
    return kfield<0, 1, 1>(b, b->conv, E, nullptr);
}

template <int K>
int segsum(mdff_batch* b, const SegSpec& sp, double* out) {
    k_b_segsum<K><<<b->nconf, 256, 0, b->st>>>(sp, b->cfg, b->N, out);
    return blaunch(b, "segsum");
}

// Lockstep PCG of (1/alpha - T) x = rhs for every configuration.
int pcg(mdff_batch* b, const double* rhs, double* x, int* iters) {
    const int N = b->N, n3 = 3 * N;
    const double tol = b->p.conv_tol_ind;
    k_b_cg_x0<<<nblk(n3, 256), 256, 0, b->st>>>(N, rhs, b->alpha, x);
    BCK(cudaMemsetAsync(b->conv, 0, sizeof(int) * b->nconf, b->st));
    BTRY(dd_field(b, x, b->Eind));
    k_b_apply_A<<<nblk(n3, 256), 256, 0, b->st>>>(N, b->cfg_of, b->cfg, nullptr, x, b->Eind, b->inv_alpha, b->cg_Ad);
    k_b_cg_init<<<nblk(n3, 256), 256, 0, b->st>>>(N, rhs, b->cg_Ad, b->alpha, b->inv_alpha, b->cg_r, b->cg_z, b->cg_d);
    SegSpec s2;
    std::memset(&s2, 0, sizeof s2);
    s2.t[0] = {b->cg_r, b->cg_r, 3};
    s2.t[1] = {b->cg_r, b->cg_z, 3};
    BTRY(segsum<2>(b, s2, b->red));
    k_b_cg_first<<<nblk(b->nconf, 64), 64, 0, b->st>>>(b->nconf, b->cfg, b->red, b->sc, b->conv, tol);
    BTRY(blaunch(b, "pcg init"));
    SegSpec s1;
    std::memset(&s1, 0, sizeof s1);
    s1.t[0] = {b->cg_d, b->cg_Ad, 3};
    int it = 0;
    for (;;) {
        BCK(cudaMemcpyAsync(b->hconv.data(), b->conv, sizeof(int) * b->nconf, cudaMemcpyDeviceToHost, b->st));
        BCK(cudaStreamSynchronize(b->st));
        bool all = true;
        for (int c = 0; c < b->nconf; ++c) all = all && b->hconv[c];
        if (all) break;
        if (it >= b->p.max_scf_pol_iter)
            return bfail(b, MDFF_E_NOCONV, "batch: induced-dipole solve did not converge within max_scf_pol_iter");
        ++it;
        BTRY(dd_field(b, b->cg_d, b->Eind));
        k_b_apply_A<<<nblk(n3, 256), 256, 0, b->st>>>(N, b->cfg_of, b->cfg, b->conv, b->cg_d, b->Eind, b->inv_alpha,
                                                      b->cg_Ad);
        BTRY(segsum<1>(b, s1, b->red + 2 * b->nconf));
        k_b_cg_update<<<nblk(n3, 256), 256, 0, b->st>>>(N, b->cfg_of, b->conv, b->sc, b->red + 2 * b->nconf, b->cg_d,
                                                        b->cg_Ad, b->alpha, x, b->cg_r, b->cg_z);
        BTRY(segsum<2>(b, s2, b->red));
        k_b_cg_scalars<<<nblk(b->nconf, 64), 64, 0, b->st>>>(b->nconf, b->cfg, b->red, b->sc, b->conv, tol);
        k_b_cg_direction<<<nblk(n3, 256), 256, 0, b->st>>>(N, b->cfg_of, b->conv, b->sc, b->cg_z, b->cg_d);
        BTRY(blaunch(b, "pcg iteration"));
    }
    *iters = it;
    return MDFF_OK;
}

int pcg_captured(mdff_batch* b, const double* rhs, double* x, int slot);

bool any_polarisable(const mdff_batch* b) {
    for (auto& C : b->hcfg)
        if (C.npol > 0) return true;
    return false;
}

// The launches of one force evaluation (no host synchronisation when the
// dipole solve is captured): forces into b->f, per-configuration sums of the
// pair and real-space energy and stress into b->red (+16 nconf, +24 nconf),
// reciprocal sums (+8 nconf).
int forward_launches(mdff_batch* b, bool captured) {
    const int N = b->N;
    const mdff_params& p = b->p;
    if (p.lbmhft || p.lbmhftd || p.lmorse) {
        k_b_pair<8><<<nblk((long)N * 8, 256), 256, 0, b->st>>>(N, b->cfg_of, b->cfg, b->sx, b->sy, b->sz, b->type,
                                                             b->nbr, b->cnt, b->cap, b->pc, b->fl, b->fpair,
                                                             b->e_pair, b->s_pair);
        BTRY(blaunch(b, "pair"));
    } else {
        BCK(cudaMemsetAsync(b->fpair, 0, sizeof(double) * 3 * N, b->st));
        BCK(cudaMemsetAsync(b->e_pair, 0, sizeof(double) * N, b->st));
        BCK(cudaMemsetAsync(b->s_pair, 0, sizeof(double) * 6 * N, b->st));
    }
    if (!captured) b->fwd_iters = 0;
    if (p.lcoulomb) {
        // static field b: damped charges, real + reciprocal
        k_b_dir<16, 0><<<dir_blocks(N, 16), 256, 0, b->st>>>(N, b->cfg_of, b->cfg, nullptr, b->sx, b->sy, b->sz, b->type,
                                                             b->q, nullptr, b->nbr, b->cnt, b->cap, b->pc, b->fl,
                                                             b->Estat, nullptr, nullptr);
        BTRY(blaunch(b, "static field"));
        BTRY((structure_factor<0, 0>(b, nullptr, nullptr)));
        BTRY((kfield<0, 1, 1>(b, nullptr, b->Estat, nullptr)));
        if (any_polarisable(b)) {
            if (captured) BTRY(pcg_captured(b, b->Estat, b->mu, 0));
            else BTRY(pcg(b, b->Estat, b->mu, &b->fwd_iters));
        } else {
            BCK(cudaMemsetAsync(b->mu, 0, sizeof(double) * 3 * N, b->st));
        }
        // final multipole Ewald: forces, energy, stress
        k_b_dir<16, 2><<<dir_blocks(N, 16), 256, 0, b->st>>>(N, b->cfg_of, b->cfg, nullptr, b->sx, b->sy, b->sz, b->type,
                                                             b->q, b->mu, b->nbr, b->cnt, b->cap, b->pc, b->fl, b->fdir,
                                                             b->e_dir, b->s_dir);
        BTRY(blaunch(b, "final real space"));
        BTRY((structure_factor<2, 1>(b, nullptr, b->mu)));
        BTRY((kfield<1, 0, 1>(b, nullptr, b->Erec, b->G)));
        k_b_rec_sums<<<b->nconf, 256, 0, b->st>>>(b->cfg, b->rho_re, b->rho_im, b->Ak, b->kcoe, b->red + 8 * b->nconf);
        BTRY(blaunch(b, "rec sums"));
    }
    k_b_forces<<<nblk(N, 256), 256, 0, b->st>>>(N, b->fpair, b->fdir, b->Erec, b->G, b->q, b->mu, b->cu, p.lcoulomb,
                                                b->f);
    BTRY(blaunch(b, "forces"));
    // per-configuration sums: pair energy + stress, real-space energy + stress
    SegSpec a;
    std::memset(&a, 0, sizeof a);
    a.t[0] = {b->e_pair, nullptr, 1};
    for (int k = 0; k < 6; ++k) a.t[1 + k] = {b->s_pair + (size_t)k * N, nullptr, 1};
    BTRY(segsum<7>(b, a, b->red + 16 * b->nconf));
    if (p.lcoulomb) {
        std::memset(&a, 0, sizeof a);
        a.t[0] = {b->e_dir, nullptr, 1};
        for (int k = 0; k < 6; ++k) a.t[1 + k] = {b->s_dir + (size_t)k * N, nullptr, 1};
        BTRY(segsum<7>(b, a, b->red + 24 * b->nconf));
    }
    return MDFF_OK;
}

// Forces, per-configuration energy and stress at the current parameters.
int forward(mdff_batch* b) {
    const mdff_params& p = b->p;
    BTRY(forward_launches(b, false));
    std::vector<double> hp((size_t)b->nconf * 7), hd((size_t)b->nconf * 7, 0.0), hs((size_t)b->nconf * 3, 0.0),
        hr((size_t)b->nconf * 8, 0.0);
    BCK(cudaMemcpyAsync(hp.data(), b->red + 16 * b->nconf, sizeof(double) * 7 * b->nconf, cudaMemcpyDeviceToHost, b->st));
    if (p.lcoulomb) {
        BCK(cudaMemcpyAsync(hd.data(), b->red + 24 * b->nconf, sizeof(double) * 7 * b->nconf, cudaMemcpyDeviceToHost,
                            b->st));
        // self-term sums q^2 and mu^2
        SegSpec a;
        std::memset(&a, 0, sizeof a);
        a.t[0] = {b->q, b->q, 1};
        a.t[1] = {b->mu, b->mu, 3};
        double* red_self = b->red + 32 * b->nconf;
        BTRY(segsum<2>(b, a, red_self));
        std::vector<double> tmp((size_t)b->nconf * 2);
        BCK(cudaMemcpyAsync(tmp.data(), red_self, sizeof(double) * 2 * b->nconf, cudaMemcpyDeviceToHost, b->st));
        BCK(cudaMemcpyAsync(hr.data(), b->red + 8 * b->nconf, sizeof(double) * 8 * b->nconf, cudaMemcpyDeviceToHost, b->st));
        BCK(cudaStreamSynchronize(b->st));
        for (int c = 0; c < b->nconf; ++c) { hs[3 * c] = tmp[2 * c]; hs[3 * c + 1] = tmp[2 * c + 1]; }
    }
    BCK(cudaStreamSynchronize(b->st));
    // energies here exclude u_pol, which mdff_batch_forces adds when asked for
    b->tau.assign((size_t)b->nconf * 9, 0.0);
    b->energy.assign(b->nconf, 0.0);
    static const int map[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
    for (int c = 0; c < b->nconf; ++c) {
        const BCfg& C = b->hcfg[c];
        const double om = C.cell.omega;
        double tn[6], tc[6];
        for (int k = 0; k < 6; ++k) {
            tn[k] = hp[7 * c + 1 + k] / om / b->press;
            const double tpi_V = 2.0 * PI / om;
            tc[k] = (hd[7 * c + 1 + k] * 0.25 / om + hr[8 * c + 1 + k] * 2.0 * tpi_V / om) * b->cu / b->press;
        }
        for (int k = 0; k < 6; ++k) {
            const int a0 = map[k][0], b0 = map[k][1];
            b->tau[9 * c + 3 * b0 + a0] = tn[k] + tc[k];
            b->tau[9 * c + 3 * a0 + b0] = tn[k] + tc[k];
        }
        double u = hp[7 * c];
        if (p.lcoulomb) {
            const double tpi_V = 2.0 * PI / om;
            const double u_rec = hr[8 * c] * 2.0 * tpi_V;
            const double u_self = -C.selfa * hs[3 * c] - C.selfa2 * hs[3 * c + 1];
            u += (hd[7 * c] + u_rec + u_self) * b->cu;
        }
        b->energy[c] = u;
    }
    return MDFF_OK;
}

// Body of one lockstep PCG iteration (captured into a WHILE node's graph).
int pcg_body(mdff_batch* b, double* x, int slot) {
    const int N = b->N, n3 = 3 * N;
    BTRY(dd_field(b, b->cg_d, b->Eind));
    k_b_apply_A<<<nblk(n3, 256), 256, 0, b->st>>>(N, b->cfg_of, b->cfg, b->conv, b->cg_d, b->Eind, b->inv_alpha,
                                                  b->cg_Ad);
    SegSpec s1;
    std::memset(&s1, 0, sizeof s1);
    s1.t[0] = {b->cg_d, b->cg_Ad, 3};
    BTRY(segsum<1>(b, s1, b->red + 2 * b->nconf));
    k_b_cg_update<<<nblk(n3, 256), 256, 0, b->st>>>(N, b->cfg_of, b->conv, b->sc, b->red + 2 * b->nconf, b->cg_d,
                                                    b->cg_Ad, b->alpha, x, b->cg_r, b->cg_z);
    SegSpec s2;
    std::memset(&s2, 0, sizeof s2);
    s2.t[0] = {b->cg_r, b->cg_r, 3};
    s2.t[1] = {b->cg_r, b->cg_z, 3};
    BTRY(segsum<2>(b, s2, b->red));
    k_b_cg_scalars<<<nblk(b->nconf, 64), 64, 0, b->st>>>(b->nconf, b->cfg, b->red, b->sc, b->conv, b->p.conv_tol_ind);
    k_b_cg_direction<<<nblk(n3, 256), 256, 0, b->st>>>(N, b->cfg_of, b->conv, b->sc, b->cg_z, b->cg_d);
    k_b_cg_cond<<<1, 256, 0, b->st>>>(b->nconf, b->conv, b->loop_it, b->p.max_scf_pol_iter, 0, b->hcond[slot]);
    return blaunch(b, "pcg iteration");
}

// Lockstep PCG inside a stream capture: the initial residual, then a
// conditional WHILE node whose body is one iteration; the loop ends on the
// device when every configuration has converged or after max_scf_pol_iter
// iterations.  solve_out[2 slot .. 2 slot + 1] receive the iteration count
// and the number of configurations that did not converge.
int pcg_captured(mdff_batch* b, const double* rhs, double* x, int slot) {
    const int N = b->N, n3 = 3 * N;
    const double tol = b->p.conv_tol_ind;
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    // the loop's condition handle, owned by the graph under capture
    BCK(cudaStreamGetCaptureInfo(b->st, &cs, nullptr, &g, nullptr, nullptr));
    BCK(cudaGraphConditionalHandleCreate(&b->hcond[slot], g, 0, 0));
    k_b_cg_x0<<<nblk(n3, 256), 256, 0, b->st>>>(N, rhs, b->alpha, x);
    BCK(cudaMemsetAsync(b->conv, 0, sizeof(int) * b->nconf, b->st));
    BTRY(dd_field(b, x, b->Eind));
    k_b_apply_A<<<nblk(n3, 256), 256, 0, b->st>>>(N, b->cfg_of, b->cfg, nullptr, x, b->Eind, b->inv_alpha, b->cg_Ad);
    k_b_cg_init<<<nblk(n3, 256), 256, 0, b->st>>>(N, rhs, b->cg_Ad, b->alpha, b->inv_alpha, b->cg_r, b->cg_z, b->cg_d);
    SegSpec s2;
    std::memset(&s2, 0, sizeof s2);
    s2.t[0] = {b->cg_r, b->cg_r, 3};
    s2.t[1] = {b->cg_r, b->cg_z, 3};
    BTRY(segsum<2>(b, s2, b->red));
    k_b_cg_first<<<nblk(b->nconf, 64), 64, 0, b->st>>>(b->nconf, b->cfg, b->red, b->sc, b->conv, tol);
    k_b_cg_cond<<<1, 256, 0, b->st>>>(b->nconf, b->conv, b->loop_it, b->p.max_scf_pol_iter, 1, b->hcond[slot]);
    BTRY(blaunch(b, "pcg init"));
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    BCK(cudaStreamGetCaptureInfo(b->st, &cs, nullptr, &g, &deps, &nd));
    alignas(cudaGraphNodeParams) unsigned char cp_raw[sizeof(cudaGraphNodeParams)];   // the struct holds a union
    std::memset(cp_raw, 0, sizeof cp_raw);                                           // with no default constructor
    cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(cp_raw);
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = b->hcond[slot];
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    BCK(cudaGraphAddNode(&node, g, deps, nd, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    BCK(cudaStreamUpdateCaptureDependencies(b->st, &node, 1, cudaStreamSetCaptureDependencies));
    cudaStream_t main_st = b->st;
    b->st = b->st2;
    cudaError_t e = cudaStreamBeginCaptureToGraph(b->st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    int r = e == cudaSuccess ? pcg_body(b, x, slot)
                             : bfail(b, MDFF_E_CUDA, std::string("capture of the PCG body: ") + cudaGetErrorString(e));
    if (e == cudaSuccess) {
        cudaGraph_t out = body;
        cudaError_t e2 = cudaStreamEndCapture(b->st, &out);
        if (r == MDFF_OK && e2 != cudaSuccess)
            r = bfail(b, MDFF_E_CUDA, std::string("capture of the PCG body: ") + cudaGetErrorString(e2));
    }
    b->st = main_st;
    BTRY(r);
    k_b_cg_summary<<<1, 32, 0, b->st>>>(b->nconf, b->conv, b->sc, b->solve_out + 2 * slot);
    return blaunch(b, "pcg summary");
}

// The loss (and, with_grad, its gradient) as launches on b->st, for capture.
int loss_grad_launches(mdff_batch* b, bool with_grad) {
    const int N = b->N;
    const mdff_params& p = b->p;
    BCK(cudaMemsetAsync(b->solve_out, 0, sizeof(int) * 4, b->st));
    BCK(cudaMemsetAsync(b->gsum, 0, sizeof(double) * 64, b->st));
    BTRY(forward_launches(b, true));
    k_b_residual<<<nblk(N, 256), 256, 0, b->st>>>(N, b->cfg_of, b->cfg, b->f, b->ft, b->R, b->lossa);
    SegSpec a;
    std::memset(&a, 0, sizeof a);
    a.t[0] = {b->lossa, nullptr, 1};
    double* lossF = b->red + 35 * b->nconf;
    BTRY(segsum<1>(b, a, lossF));
    k_b_loss_tail<<<nblk(b->nconf, 64), 64, 0, b->st>>>(b->nconf, b->cfg, b->red + 16 * b->nconf,
                                                        b->red + 24 * b->nconf, b->red + 8 * b->nconf, lossF,
                                                        b->tau_t_dev, b->cu, b->press, p.lcoulomb, b->loss_c, b->tau_c,
                                                        b->Sres);
    BTRY(blaunch(b, "loss"));
    if (!with_grad) return MDFF_OK;
    constexpr int KA = NTYB * NTYB * 4, KR = NTYB * NTYB * 10;
    const int blk16 = dir_blocks(N, 16);
    if (p.lcoulomb && any_polarisable(b)) {
        // adjoint right-hand side h = dJ/dmu
        k_b_dir_adj<16><<<blk16, 256, 0, b->st>>>(N, b->cfg_of, b->cfg, b->sx, b->sy, b->sz, b->type, b->q, b->mu, b->R,
                                                  b->Sres, b->nbr, b->cnt, b->cap, b->pc, b->fl, b->h, b->gpart);
        k_b_reduce_cols<<<nblk(KA, 8), 256, 0, b->st>>>(b->gpart, blk16, KA, b->gsum);
        BTRY(blaunch(b, "adjoint real space"));
        BTRY((structure_factor<3, 2>(b, nullptr, b->mu)));
        BTRY((kfield<0, 1, 0>(b, nullptr, b->h, nullptr)));
        k_b_h_finish<<<nblk(N, 256), 256, 0, b->st>>>(N, b->G, b->R, b->inv_alpha, b->cu, b->h);
        BTRY(blaunch(b, "adjoint rhs"));
        BTRY(pcg_captured(b, b->h, b->lam, 1));
        const int ab = std::min(592, nblk(N, 256));
        k_b_alpha_grad<<<ab, 256, 0, b->st>>>(N, b->type, b->lam, b->mu, b->inv_alpha, b->gpart);
        k_b_reduce_cols<<<1, 256, 0, b->st>>>(b->gpart, ab, NTYB, b->gsum + KA + KR);
        BTRY(blaunch(b, "alpha gradient"));
    } else {
        BCK(cudaMemsetAsync(b->lam, 0, sizeof(double) * 3 * N, b->st));
    }
    k_b_grad_rows<16><<<blk16, 256, 0, b->st>>>(N, b->cfg_of, b->cfg, b->sx, b->sy, b->sz, b->type, b->q, b->R, b->Sres,
                                                b->lam, b->nbr, b->cnt, b->cap, b->pc, b->fl, b->gpart);
    k_b_reduce_cols<<<nblk(KR, 8), 256, 0, b->st>>>(b->gpart, blk16, KR, b->gsum + KA);
    return blaunch(b, "row gradient");
}

void drop_graph(mdff_batch* b, int which) {
    cudaGraphExec_t& ge = which ? b->gexec : b->gexec_loss;
    cudaGraph_t& g = which ? b->graph : b->graph_loss;
    if (ge) cudaGraphExecDestroy(ge);
    if (g) cudaGraphDestroy(g);
    ge = nullptr;
    g = nullptr;
}

// Capture the evaluation (which = 1: loss and gradient; 0: loss only) as one
// CUDA graph and instantiate it.
int build_graph(mdff_batch* b, int which) {
    drop_graph(b, which);
    BCK(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
    int r = loss_grad_launches(b, which == 1);
    cudaGraph_t out = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->st, &out);
    if (r == MDFF_OK && e != cudaSuccess) r = bfail(b, MDFF_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    if (r != MDFF_OK) {
        if (out) cudaGraphDestroy(out);
        cudaGetLastError();
        return r;
    }
    cudaGraphExec_t ge = nullptr;
    e = cudaGraphInstantiate(&ge, out, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(out);
        return bfail(b, MDFF_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    }
    (which ? b->graph : b->graph_loss) = out;
    (which ? b->gexec : b->gexec_loss) = ge;
    b->gflags[which] = b->fl;
    b->gpol[which] = any_polarisable(b);
    return MDFF_OK;
}

int loss_and_gradient(mdff_batch* b, double* loss, mdff_param_grad* grad) {
    const int which = grad ? 1 : 0;
    const bool stale = (which ? !b->gexec : !b->gexec_loss) ||
                       std::memcmp(&b->gflags[which], &b->fl, sizeof(BFlags)) != 0 ||
                       b->gpol[which] != any_polarisable(b);
    if (stale) BTRY(build_graph(b, which));
    BCK(cudaGraphLaunch(which ? b->gexec : b->gexec_loss, b->st));
    constexpr int KA = NTYB * NTYB * 4, KR = NTYB * NTYB * 10;
    std::vector<double> lc(b->nconf), gs(64);
    int so[4];
    BCK(cudaMemcpyAsync(lc.data(), b->loss_c, sizeof(double) * b->nconf, cudaMemcpyDeviceToHost, b->st));
    BCK(cudaMemcpyAsync(b->tau.data(), b->tau_c, sizeof(double) * 9 * b->nconf, cudaMemcpyDeviceToHost, b->st));
    BCK(cudaMemcpyAsync(gs.data(), b->gsum, sizeof(double) * 64, cudaMemcpyDeviceToHost, b->st));
    BCK(cudaMemcpyAsync(so, b->solve_out, sizeof(int) * 4, cudaMemcpyDeviceToHost, b->st));
    BCK(cudaStreamSynchronize(b->st));
    b->fwd_iters = so[0];
    b->adj_iters = so[2];
    if (so[1] || so[3])
        return bfail(b, MDFF_E_NOCONV, "batch: induced-dipole solve did not converge within max_scf_pol_iter");
    double L = 0.0;
    for (int c = 0; c < b->nconf; ++c) L += lc[c];
    *loss = L;
    if (!grad) return MDFF_OK;
    std::memset(grad, 0, sizeof(mdff_param_grad));
    const double* gA = gs.data();
    const double* gR = gs.data() + KA;
    const double* gP = gs.data() + KA + KR;
    // fold ordered slots (ti,tj) into the upper-triangle parameter slots
    for (int ti = 0; ti < b->ntype; ++ti)
        for (int tj = 0; tj < b->ntype; ++tj) {
            const int lo = std::min(ti, tj), hi = std::max(ti, tj);
            const double* r = &gR[(ti * NTYB + tj) * 10];
            grad->Abmhftd[lo][hi] += r[0];
            grad->Bbmhftd[lo][hi] += r[1];
            grad->Cbmhftd[lo][hi] += r[2];
            grad->Dbmhftd[lo][hi] += r[3];
            grad->BDbmhftd[lo][hi] += r[4];
            grad->epsmor[lo][hi] += r[5];
            grad->rhomor[lo][hi] += r[6];
            grad->sigmamor[lo][hi] += r[7];
            // static-field damping at i: entry (ti,ti,tj)
            grad->dip_pol_damp_b[ti][lo][hi] += r[8];
            grad->dip_pol_damp_c[ti][lo][hi] += r[9];
            const double* d = &gA[(ti * NTYB + tj) * 4];
            grad->dip_pol_damp_b[ti][lo][hi] += d[0];   // entry (ti,ti,tj)
            grad->dip_pol_damp_c[ti][lo][hi] += d[1];
            grad->dip_pol_damp_b[tj][lo][hi] += d[2];   // entry (tj,ti,tj)
            grad->dip_pol_damp_c[tj][lo][hi] += d[3];
        }
    for (int t = 0; t < b->ntype; ++t) grad->poldip_iso[t] += gP[t];
    return MDFF_OK;
}

}  // namespace

extern "C" {

int mdff_batch_create(const mdff_params* p, int nconf, const int* natm, const int* itype, const double* rx,
                      const double* ry, const double* rz, const double* cells, const double* rc, const double* alpha,
                      const int* kmax, mdff_batch** out) {
    if (!out) return MDFF_E_ARG;
    mdff_batch* b = new mdff_batch();
    *out = b;   // also on failure: the caller reads mdff_batch_last_error and destroys it
    auto bad = [&](int code) { return code; };
    if (!p || nconf < 1 || !natm || !itype || !rx || !ry || !rz || !cells || !rc || !alpha || !kmax)
        return bad(bfail(b, MDFF_E_ARG, "mdff_batch_create: null argument or nconf < 1"));
    if (int r = check_batch_params(b, *p)) return bad(r);
    if (!p->lcoulomb && !(p->lbmhft || p->lbmhftd || p->lmorse))
        return bad(bfail(b, MDFF_E_ARG, "batch: no interaction enabled"));
    cudaError_t e = cudaSetDevice(p->device);
    if (e != cudaSuccess) return bad(bfail(b, MDFF_E_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e)));
    e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->st2, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bad(bfail(b, MDFF_E_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e)));
    if (p->lreduced) { b->cu = 1.0; b->press = 1.0; }
    else { b->cu = 14.3996441494161; b->press = 0.00624150964712042; }
    b->nconf = nconf;
    b->ntype = p->ntype;
    long N = 0;
    for (int c = 0; c < nconf; ++c) {
        if (natm[c] < 1) return bad(bfail(b, MDFF_E_ARG, "batch: a configuration has no atoms"));
        N += natm[c];
    }
    if (N > (1L << 28)) return bad(bfail(b, MDFF_E_ARG, "batch: too many atoms"));
    b->N = (int)N;
    b->hcfg.resize(nconf);
    long off = 0;
    int roff = 0;
    int cap_est = 32;
    for (int c = 0; c < nconf; ++c) {
        BCfg& C = b->hcfg[c];
        std::memset(&C, 0, sizeof C);
        double W[3];
        lattice9(cells + 9 * c, C.cell, W);
        if (!(C.cell.omega > 0.0)) return bad(bfail(b, MDFF_E_ARG, "batch: singular or left-handed cell"));
        if (!(rc[c] > 0.0) || rc[c] > 0.5 * std::min(W[0], std::min(W[1], W[2])) * (1.0 + 1e-12))
            return bad(bfail(b, MDFF_E_ARG, "batch: rc must be positive and at most half the smallest cell width"));
        if (p->lcoulomb && !(alpha[c] > 0.0)) return bad(bfail(b, MDFF_E_ARG, "batch: Ewald alpha must be positive"));
        for (int d = 0; d < 3; ++d)
            if (kmax[3 * c + d] < 0 || kmax[3 * c + d] > 64) return bad(bfail(b, MDFF_E_ARG, "batch: kmax out of [0,64]"));
        C.off = (int)off;
        C.n = natm[c];
        off += natm[c];
        C.rc2 = rc[c] * rc[c];
        C.alpha = alpha[c];
        C.selfa = alpha[c] / std::sqrt(PI);
        C.selfa2 = 2.0 * C.selfa * alpha[c] * alpha[c] / 3.0;
        for (int d = 0; d < 3; ++d) C.kmax[d] = p->lcoulomb ? kmax[3 * c + d] : 0;
        C.ncol = (C.kmax[0] + 1) * (2 * C.kmax[1] + 1);
        C.nzl = 2 * C.kmax[2] + 1;
        C.nrect = C.ncol * C.nzl;
        C.roff = roff;
        roff += C.nrect;
        b->nzl_max = std::max(b->nzl_max, C.nzl);
        b->phw_max = std::max(b->phw_max, (C.kmax[0] + 1) + (2 * C.kmax[1] + 1) + (C.nzl + NZC - 1) / NZC);
        double dens = natm[c] / C.cell.omega;
        int est = (int)(dens * 4.0 / 3.0 * PI * rc[c] * rc[c] * rc[c] * 1.3) + 32;
        cap_est = std::max(cap_est, std::min(est, natm[c]));
        C.cs = (int)b->hchunk.size();
        for (int a0 = 0; a0 < C.n; a0 += CHUNK) {
            BChunk ch;
            ch.c = c;
            ch.a0 = C.off + a0;
            ch.na = std::min(CHUNK, C.n - a0);
            ch.poff = b->part_len;
            b->part_len += C.nrect;
            b->hchunk.push_back(ch);
        }
        C.ce = (int)b->hchunk.size();
    }
    b->nrect_tot = roff;
    b->nchunk = (int)b->hchunk.size();
    b->hconv.assign(nconf, 0);
    // device buffers
    int r = MDFF_OK;
    auto A = [&](auto** ptr, size_t n) { if (r == MDFF_OK) r = balloc(b, ptr, n); };
    A(&b->cfg, nconf);
    A(&b->chunk, b->nchunk);
    A(&b->rcfg, b->nrect_tot);
    A(&b->cfg_of, N);
    A(&b->type, N);
    for (double** v : {&b->x, &b->y, &b->z, &b->sx, &b->sy, &b->sz, &b->q, &b->alpha, &b->inv_alpha, &b->e_pair,
                       &b->e_dir, &b->lossa})
        A(v, N);
    for (double** v : {&b->f, &b->fpair, &b->fdir, &b->Erec, &b->Estat, &b->mu, &b->Eind, &b->cg_r, &b->cg_z, &b->cg_d,
                       &b->cg_Ad, &b->h, &b->lam, &b->R, &b->ft})
        A(v, 3 * N);
    A(&b->G, 6 * N);
    A(&b->s_pair, 6 * N);
    A(&b->s_dir, 6 * N);
    A(&b->pc, NT * NT);
    for (double** v : {&b->Ak, &b->kcoe, &b->rho_re, &b->rho_im, &b->C_re, &b->C_im}) A(v, b->nrect_tot);
    A(&b->part_re, b->part_len);
    A(&b->part_im, b->part_len);
    A(&b->conv, nconf);
    A(&b->sc, nconf);
    A(&b->red, 40 * nconf);
    A(&b->Sres, 9 * nconf);
    A(&b->overflow, 1);
    A(&b->loop_it, 1);
    A(&b->solve_out, 4);
    A(&b->tau_t_dev, 9 * nconf);
    A(&b->loss_c, nconf);
    A(&b->tau_c, 9 * nconf);
    b->gpart_cap = dir_blocks(b->N, 16) * NTYB * NTYB * 10 + 1024;
    A(&b->gpart, b->gpart_cap);
    A(&b->gsum, 64);
    if (r) return bad(r);
    // host tables
    std::vector<int> hcfg_of(N), ht(N), hr(b->nrect_tot);
    std::vector<double> hak(b->nrect_tot, 0.0), hkc(b->nrect_tot, 0.0);
    for (int c = 0; c < nconf; ++c) {
        const BCfg& C = b->hcfg[c];
        for (int i = C.off; i < C.off + C.n; ++i) {
            hcfg_of[i] = c;
            if (itype[i] < 1 || itype[i] > p->ntype) return bad(bfail(b, MDFF_E_ARG, "batch: atom type out of range"));
            ht[i] = itype[i] - 1;
        }
        const double a2 = C.alpha * C.alpha;
        for (int l = 0; l < C.nrect; ++l) {
            hr[C.roff + l] = c;
            int col = l / C.nzl, nx = col / (2 * C.kmax[1] + 1), ny = col % (2 * C.kmax[1] + 1) - C.kmax[1];
            int nz = l % C.nzl - C.kmax[2];
            bool keep = nx > 0 || (nx == 0 && ny > 0) || (nx == 0 && ny == 0 && nz > 0);
            if (!keep) continue;
            const double* B = C.cell.B;
            double kx = 2.0 * PI * (nx * B[0] + ny * B[1] + nz * B[2]);
            double ky = 2.0 * PI * (nx * B[3] + ny * B[4] + nz * B[5]);
            double kz = 2.0 * PI * (nx * B[6] + ny * B[7] + nz * B[8]);
            double kk = kx * kx + ky * ky + kz * kz;
            if (kk == 0.0) continue;
            hak[C.roff + l] = std::exp(-kk * 0.25 / a2) / kk;
            hkc[C.roff + l] = 2.0 * (1.0 / kk + 1.0 / a2 / 4.0);
        }
    }
    if ((e = cudaMemcpyAsync(b->chunk, b->hchunk.data(), sizeof(BChunk) * b->nchunk, cudaMemcpyHostToDevice, b->st)) ||
        (e = cudaMemcpyAsync(b->rcfg, hr.data(), sizeof(int) * b->nrect_tot, cudaMemcpyHostToDevice, b->st)) ||
        (e = cudaMemcpyAsync(b->cfg_of, hcfg_of.data(), sizeof(int) * N, cudaMemcpyHostToDevice, b->st)) ||
        (e = cudaMemcpyAsync(b->type, ht.data(), sizeof(int) * N, cudaMemcpyHostToDevice, b->st)) ||
        (e = cudaMemcpyAsync(b->Ak, hak.data(), sizeof(double) * b->nrect_tot, cudaMemcpyHostToDevice, b->st)) ||
        (e = cudaMemcpyAsync(b->kcoe, hkc.data(), sizeof(double) * b->nrect_tot, cudaMemcpyHostToDevice, b->st)) ||
        (e = cudaMemcpyAsync(b->x, rx, sizeof(double) * N, cudaMemcpyHostToDevice, b->st)) ||
        (e = cudaMemcpyAsync(b->y, ry, sizeof(double) * N, cudaMemcpyHostToDevice, b->st)) ||
        (e = cudaMemcpyAsync(b->z, rz, sizeof(double) * N, cudaMemcpyHostToDevice, b->st)) ||
        (e = cudaMemsetAsync(b->mu, 0, sizeof(double) * 3 * N, b->st)) ||
        (e = cudaMemsetAsync(b->Erec, 0, sizeof(double) * 3 * N, b->st)) ||
        (e = cudaMemsetAsync(b->G, 0, sizeof(double) * 6 * N, b->st)) ||
        (e = cudaMemsetAsync(b->fdir, 0, sizeof(double) * 3 * N, b->st)) ||
        (e = cudaMemsetAsync(b->ft, 0, sizeof(double) * 3 * N, b->st)) ||
        (e = cudaMemsetAsync(b->Sres, 0, sizeof(double) * 9 * nconf, b->st)))
        return bad(bfail(b, MDFF_E_CUDA, std::string("batch upload: ") + cudaGetErrorString(e)));
    b->tau_t.assign((size_t)9 * nconf, 0.0);
    b->tau.assign((size_t)9 * nconf, 0.0);
    if (int r2 = upload_params(b, *p)) return bad(r2);
    k_b_wrap_frac<<<nblk(N, 256), 256, 0, b->st>>>(b->N, b->cfg_of, b->cfg, b->x, b->y, b->z, b->sx, b->sy, b->sz);
    if (int r2 = blaunch(b, "wrap")) return bad(r2);
    // neighbour rows (no skin: the positions of a batch do not move)
    int cap = p->nlist_capacity > 0 ? p->nlist_capacity : cap_est;
    for (int attempt = 0; attempt < 4; ++attempt) {
        if (b->nbr) {
            cudaFree(b->nbr);
            b->allocs.erase(std::find(b->allocs.begin(), b->allocs.end(), (void*)b->nbr));
            b->nbr = nullptr;
        }
        if (int r2 = balloc(b, &b->nbr, (size_t)N * cap)) return bad(r2);
        if (!b->cnt)
            if (int r2 = balloc(b, &b->cnt, N)) return bad(r2);
        b->cap = cap;
        if ((e = cudaMemsetAsync(b->overflow, 0, sizeof(int), b->st)))
            return bad(bfail(b, MDFF_E_CUDA, cudaGetErrorString(e)));
        k_b_nlist<<<nblk((long)N * 32, 256), 256, 0, b->st>>>(b->N, b->cfg_of, b->cfg, b->sx, b->sy, b->sz, b->nbr,
                                                              b->cnt, cap, b->overflow);
        if (int r2 = blaunch(b, "batch nlist")) return bad(r2);
        int ovf = 0;
        if ((e = cudaMemcpyAsync(&ovf, b->overflow, sizeof(int), cudaMemcpyDeviceToHost, b->st)) ||
            (e = cudaStreamSynchronize(b->st)))
            return bad(bfail(b, MDFF_E_CUDA, cudaGetErrorString(e)));
        if (ovf == 0) break;
        if (attempt == 3) return bad(bfail(b, MDFF_E_LISTOVF, "batch: neighbour list capacity exceeded"));
        cap = (int)(ovf * 1.25) + 32;
    }
    {   // the structure factor's per-atom phase tables live in dynamic shared memory
        const size_t sm = sizeof(double2) * (size_t)CHUNK * b->phw_max;
        if (sm > 200 * 1024)
            return bad(bfail(b, MDFF_E_UNSUPPORTED, "batch: k rectangle too large for the structure factor's tables"));
        cudaError_t e2 = cudaFuncSetAttribute(k_b_sfac<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e2 == cudaSuccess) e2 = cudaFuncSetAttribute(k_b_sfac<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e2 == cudaSuccess) e2 = cudaFuncSetAttribute(k_b_sfac<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e2 == cudaSuccess) e2 = cudaFuncSetAttribute(k_b_sfac<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e2 != cudaSuccess) return bad(bfail(b, MDFF_E_CUDA, cudaGetErrorString(e2)));
    }
    if (int r2 = build_ddtab(b)) return bad(r2);
    return MDFF_OK;
}

void mdff_batch_destroy(mdff_batch* b) {
    if (!b) return;
    if (b->st) cudaStreamSynchronize(b->st);
    drop_graph(b, 0);
    drop_graph(b, 1);
    for (void* p : b->allocs) cudaFree(p);
    if (b->st) cudaStreamDestroy(b->st);
    if (b->st2) cudaStreamDestroy(b->st2);
    delete b;
}

const char* mdff_batch_last_error(const mdff_batch* b) { return b ? b->err.c_str() : "null batch"; }

int mdff_batch_set_params(mdff_batch* b, const mdff_params* p) {
    if (!b || !p) return MDFF_E_ARG;
    if (p->lcoulomb != b->p.lcoulomb) return bfail(b, MDFF_E_ARG, "batch: lcoulomb cannot change after creation");
    if (p->precision != b->p.precision) return bfail(b, MDFF_E_ARG, "batch: precision cannot change after creation");
    BTRY(upload_params(b, *p));
    if (b->fl.erfc_ref != b->dd_ref) BTRY(build_ddtab(b));   // the table's erfc follows the parameters
    return MDFF_OK;
}

int mdff_batch_forces(mdff_batch* b, double* fx, double* fy, double* fz, double* tau, double* energy, int* iters) {
    if (!b) return MDFF_E_ARG;
    BTRY(forward(b));
    const int N = b->N;
    double* outs[3] = {fx, fy, fz};
    for (int c = 0; c < 3; ++c)
        if (outs[c]) BCK(cudaMemcpyAsync(outs[c], b->f + (size_t)c * N, sizeof(double) * N, cudaMemcpyDeviceToHost, b->st));
    BCK(cudaStreamSynchronize(b->st));
    if (tau) std::memcpy(tau, b->tau.data(), sizeof(double) * 9 * b->nconf);
    if (energy) {
        // add u_pol = 1/2 sum mu.alpha^-1.mu per configuration (coul_unit)
        std::vector<double> hmu((size_t)3 * N), hia(N);
        BCK(cudaMemcpyAsync(hmu.data(), b->mu, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, b->st));
        BCK(cudaMemcpyAsync(hia.data(), b->inv_alpha, sizeof(double) * N, cudaMemcpyDeviceToHost, b->st));
        BCK(cudaStreamSynchronize(b->st));
        for (int c = 0; c < b->nconf; ++c) {
            const BCfg& C = b->hcfg[c];
            double up = 0.0;
            for (int i = C.off; i < C.off + C.n; ++i)
                for (int k = 0; k < 3; ++k) up += hmu[(size_t)k * N + i] * hia[i] * hmu[(size_t)k * N + i];
            energy[c] = b->energy[c] + 0.5 * up * b->cu;
        }
    }
    if (iters) *iters = b->fwd_iters;
    return MDFF_OK;
}

int mdff_batch_set_targets(mdff_batch* b, const double* fx, const double* fy, const double* fz, const double* tau,
                           double w_force, double w_stress) {
    if (!b || !fx || !fy || !fz || !tau) return MDFF_E_ARG;
    const int N = b->N;
    BCK(cudaMemcpyAsync(b->ft, fx, sizeof(double) * N, cudaMemcpyHostToDevice, b->st));
    BCK(cudaMemcpyAsync(b->ft + N, fy, sizeof(double) * N, cudaMemcpyHostToDevice, b->st));
    BCK(cudaMemcpyAsync(b->ft + 2 * (size_t)N, fz, sizeof(double) * N, cudaMemcpyHostToDevice, b->st));
    std::memcpy(b->tau_t.data(), tau, sizeof(double) * 9 * b->nconf);
    BCK(cudaMemcpyAsync(b->tau_t_dev, tau, sizeof(double) * 9 * b->nconf, cudaMemcpyHostToDevice, b->st));
    b->w_force = w_force;
    b->w_stress = w_stress;
    for (auto& C : b->hcfg) {
        C.cF = w_force / (3.0 * C.n * b->nconf);
        C.cS = w_stress / (9.0 * b->nconf);
    }
    BCK(cudaMemcpyAsync(b->cfg, b->hcfg.data(), sizeof(BCfg) * b->nconf, cudaMemcpyHostToDevice, b->st));
    BCK(cudaStreamSynchronize(b->st));
    b->have_targets = true;
    return MDFF_OK;
}

int mdff_batch_loss_grad(mdff_batch* b, double* loss, mdff_param_grad* grad, int iters[2]) {
    if (!b || !loss) return MDFF_E_ARG;
    if (!b->have_targets) return bfail(b, MDFF_E_STATE, "batch: set the targets first (mdff_batch_set_targets)");
    BTRY(loss_and_gradient(b, loss, grad));
    if (iters) { iters[0] = b->fwd_iters; iters[1] = b->adj_iters; }
    return MDFF_OK;
}

int mdff_batch_stream(mdff_batch* b, void** stream) {
    if (!b || !stream) return MDFF_E_ARG;
    *stream = (void*)b->st;
    return MDFF_OK;
}

}  // extern "C"
