// ewald_real.cu -- real-space part of the multipole Ewald sum for point
// charges and dipoles: energy, electric field, field gradient, forces, stress.
//
// Replaces multipole_ES_dir (src/field.f90:2057-2643) for the charge-charge,
// charge-dipole and dipole-dipole tasks with the Tang-Toennies damping of the
// charge-dipole interaction.  The reference builds the full rank-0..5
// interaction tensors for every pair; here each contraction is written in
// closed form from the screened radial functions F0..F3
// (F1 = F0 + 2 a r e, F2 = F1 + 4/3 a^3 r^3 e, F3 = F2 + 8/15 a^5 r^5 e with
// e = exp(-a^2 r^2)/sqrt(pi), src/field.f90:2220-2225):
//   T1 v   = -(r.v) F1/r^3
//   T2 v   =  r (r.v) 3F2/r^5 - v F1/r^3
//   T3 uv  = -r (r.u)(r.v) 15F3/r^7 + [u (r.v) + v (r.u) + r (u.v)] 3F2/r^5
// G lanes share one atom's full neighbour row and accumulate onto that atom
// only; energies and stresses are halved per ordered pair.
#include "common.cuh"

namespace mdff {

// MODE 0: full evaluation (tasks from flags; field / efg / forces from flags)
// MODE 1: induced-dipole field operator E_i = sum_j T2(r_ij) mu_j (no damping),
//         the dipole-dipole field of src/field.f90:3354.
// MODE 2: the damped field of the charges alone (the static field before the
//         dipole solve: qq, field, damping, optional pair table), with only
//         what that needs -- one damping factor per pair, no dipoles, no
//         energy, stress or block partials; the field is MODE 0's, bit for bit.
// MODE 3: MODE 0 without the field gradient (every step but the EFG steps),
//         so its registers are not sized for it.
template <int G, int MODE>
__global__ void __launch_bounds__(256, MODE == 2 ? 3 : 2) k_ewald_dir(int n, const double* __restrict__ sx, const double* __restrict__ sy,
                                                   const double* __restrict__ sz, const int* __restrict__ type,
                                                   const double* __restrict__ q, const double* __restrict__ mu,
                                                   CellP c, const int* __restrict__ nbr, const int* __restrict__ cnt,
                                                   int cap, const PairConst* __restrict__ pc, DirFlags fl,
                                                   double* __restrict__ ef, double* __restrict__ efg,
                                                   double* __restrict__ fo, double* part) {
    const int gid = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    const int sub = threadIdx.x & (G - 1);
    const bool active = gid < n;
    const int i = active ? gid : 0;
    const double a = fl.alpha, a2 = a * a, a3 = a2 * a, a5 = a3 * a2;
    const double c43a3 = 4.0 * a3 / 3.0, c815a5 = 8.0 * a5 / 15.0;
    const double rsqpi = 0.56418958354775628695;   // 1/sqrt(pi)
    double E[3] = {0, 0, 0}, Gd[6] = {0, 0, 0, 0, 0, 0}, F[3] = {0, 0, 0};
    double u = 0.0, S[6] = {0, 0, 0, 0, 0, 0};
    if (active) {
        const double si1 = sx[i], si2 = sy[i], si3 = sz[i];
        const int ti = type[i];
        const double qi = (MODE == 0 || MODE == 3) ? q[i] : 0.0;
        const double mi0 = MODE == 2 ? 0.0 : mu[i], mi1 = MODE == 2 ? 0.0 : mu[n + i],
                     mi2 = MODE == 2 ? 0.0 : mu[2 * n + i];
        const int m = cnt[i];
        const int* row = nbr + (size_t)i * cap;
        // pair table: the lanes of the group compact the entries inside the
        // cutoff in list order (a ballot per sweep of G entries)
        const int g0 = (threadIdx.x & 31) & ~(G - 1);
        const unsigned gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << g0);
        int cbase = 0, pos = 0;
        for (int k0 = 0; k0 < m; k0 += G) {
            const int k = k0 + sub;
            const bool valid = k < m;
            const int j = valid ? row[k] : i;
            double rx = 0.0, ry = 0.0, rz = 0.0, d2 = 0.0;
            if (valid) d2 = pairvec_exact(c, si1, si2, si3, sx[j], sy[j], sz[j], rx, ry, rz);
            const bool in = valid && d2 <= fl.cutsq;
            if (MODE != 1 && fl.ddtab) {
                const unsigned bal = (__ballot_sync(gmask, in) & gmask) >> g0;
                pos = cbase + __popc(bal & ((1u << sub) - 1u));
                if (in) fl.ddnbr[(size_t)i * cap + pos] = j;
                cbase += __popc(bal);
            }
            if (!in) continue;
            const double d = sqrt(d2);
            const double dm1 = 1.0 / d, dm2 = dm1 * dm1, dm3 = dm1 * dm2, dm5 = dm3 * dm2, dm7 = dm5 * dm2;
            const double ex2 = exp(-a2 * d2), expon = ex2 * rsqpi;
            const double F0 = fl.erfc_ref ? erfc_fit(a * d) : erfc_ex2(a * d, ex2);
            const double F1 = F0 + 2.0 * a * d * expon;
            const double F2 = F1 + c43a3 * d2 * d * expon;
            const double A1 = F1 * dm3;
            const double B2 = 3.0 * F2 * dm5;
            if (MODE != 1 && fl.ddtab) fl.ddtab[(size_t)i * cap + pos] = make_float2((float)A1, (float)B2);
            if (MODE == 2) {
                double gi = 0.0;
                if (fl.damp) {
                    const PairConst& P = pc[ti * NT + type[j]];
                    if (P.ldamp && P.dc_i != 0.0) {   // c = 0 gives f = 1 exactly
                        double f1, gd;
                        tt_damp_d(P.db_i, P.dc_i, d, P.dk_i, f1, gd);
                        gi = 1.0 - f1;
                    }
                }
                const double s = q[j] * (F1 - gi) * dm3;
                E[0] += s * rx; E[1] += s * ry; E[2] += s * rz;
                continue;
            }
            const double mj0 = mu[j], mj1 = mu[n + j], mj2 = mu[2 * n + j];
            const double rmj = rx * mj0 + ry * mj1 + rz * mj2;
            if (MODE == 1) {
                E[0] += rx * rmj * B2 - mj0 * A1;
                E[1] += ry * rmj * B2 - mj1 * A1;
                E[2] += rz * rmj * B2 - mj2 * A1;
                continue;
            }
            const int tj = type[j];
            const double qj = q[j];
            const double rmi = rx * mi0 + ry * mi1 + rz * mi2;
            const double F3 = F2 + c815a5 * d2 * d2 * d * expon;
            const double C3 = 15.0 * F3 * dm7;
            // Tang-Toennies damping of the charge-dipole terms (src/field.f90:2205-2217).
            double gi = 0.0, gdi = 0.0, gj = 0.0, gdj = 0.0;
            bool ldamp = false;
            if (fl.damp) {
                const PairConst& P = pc[ti * NT + tj];
                if (P.ldamp) {
                    ldamp = true;
                    // c = 0 gives f = 1 and f' = 0 exactly; identical constants at
                    // i and j (like-type pairs) give identical values
                    double f1 = 1.0, f2 = 1.0;
                    if (P.dc_i != 0.0) tt_damp_d(P.db_i, P.dc_i, d, P.dk_i, f1, gdi);
                    if (P.dc_j != 0.0) {
                        if (P.db_j == P.db_i && P.dc_j == P.dc_i && P.dk_j == P.dk_i) {
                            f2 = f1;
                            gdj = gdi;
                        } else {
                            tt_damp_d(P.db_j, P.dc_j, d, P.dk_j, f2, gdj);
                        }
                    }
                    gi = 1.0 - f1;
                    gj = 1.0 - f2;
                }
            }
            double fi0 = 0.0, fi1 = 0.0, fi2 = 0.0;
            if (fl.qq) {
                u += 0.5 * qi * qj * F0 * dm1;
                if (fl.field) {
                    const double s = qj * (F1 - gi) * dm3;
                    E[0] += s * rx; E[1] += s * ry; E[2] += s * rz;
                }
                if (MODE == 0 && fl.efg) {
                    const double b = -qj * B2, dg = qj * A1;
                    Gd[0] += b * rx * rx + dg; Gd[1] += b * ry * ry + dg; Gd[2] += b * rz * rz + dg;
                    Gd[3] += b * rx * ry; Gd[4] += b * rx * rz; Gd[5] += b * ry * rz;
                }
                const double s = qi * qj * A1;
                fi0 += s * rx; fi1 += s * ry; fi2 += s * rz;
            }
            if (fl.dd) {
                const double mimj = mi0 * mj0 + mi1 * mj1 + mi2 * mj2;
                u -= 0.5 * (rmi * rmj * B2 - mimj * A1);
                if (fl.field) {
                    E[0] += rx * rmj * B2 - mj0 * A1;
                    E[1] += ry * rmj * B2 - mj1 * A1;
                    E[2] += rz * rmj * B2 - mj2 * A1;
                }
                if (MODE == 0 && fl.efg) {
                    const double t = -rmj * C3;
                    Gd[0] += t * rx * rx + rmj * B2 + 2.0 * rx * mj0 * B2;
                    Gd[1] += t * ry * ry + rmj * B2 + 2.0 * ry * mj1 * B2;
                    Gd[2] += t * rz * rz + rmj * B2 + 2.0 * rz * mj2 * B2;
                    Gd[3] += t * rx * ry + (ry * mj0 + rx * mj1) * B2;
                    Gd[4] += t * rx * rz + (rz * mj0 + rx * mj2) * B2;
                    Gd[5] += t * ry * rz + (rz * mj1 + ry * mj2) * B2;
                }
                const double t3 = -rmi * rmj * C3 + mimj * B2;
                fi0 += t3 * rx + (mi0 * rmj + mj0 * rmi) * B2;
                fi1 += t3 * ry + (mi1 * rmj + mj1 * rmi) * B2;
                fi2 += t3 * rz + (mi2 * rmj + mj2 * rmi) * B2;
            }
            if (fl.qd) {
                u += 0.5 * (qi * A1 * rmj - qj * A1 * rmi);
                // qi T2 mu_j - qj T2 mu_i
                const double s = (qi * rmj - qj * rmi) * B2;
                fi0 += rx * s - (qi * mj0 - qj * mi0) * A1;
                fi1 += ry * s - (qi * mj1 - qj * mi1) * A1;
                fi2 += rz * s - (qi * mj2 - qj * mi2) * A1;
                if (ldamp) {
                    u += 0.5 * (-qi * gj * dm3 * rmj + qj * gi * dm3 * rmi);
                    const double F2d = gi + (d / 3.0) * gdi, F2d2 = gj + (d / 3.0) * gdj;
                    const double Bi = 3.0 * F2d * dm5, Ai = gi * dm3;     // T2d  (damping at i)
                    const double Bj = 3.0 * F2d2 * dm5, Aj = gj * dm3;    // T2d2 (damping at j)
                    // qj T2d mu_i - qi T2d2 mu_j
                    fi0 += qj * (rx * rmi * Bi - mi0 * Ai) - qi * (rx * rmj * Bj - mj0 * Aj);
                    fi1 += qj * (ry * rmi * Bi - mi1 * Ai) - qi * (ry * rmj * Bj - mj1 * Aj);
                    fi2 += qj * (rz * rmi * Bi - mi2 * Ai) - qi * (rz * rmj * Bj - mj2 * Aj);
                }
            }
            if (fl.forces) {
                F[0] += fi0; F[1] += fi1; F[2] += fi2;
                S[0] += 2.0 * rx * fi0; S[1] += 2.0 * ry * fi1; S[2] += 2.0 * rz * fi2;
                S[3] += rx * fi1 + ry * fi0; S[4] += rx * fi2 + rz * fi0; S[5] += ry * fi2 + rz * fi1;
            }
        }
        if (MODE != 1 && fl.ddtab && sub == 0) fl.ddcnt[i] = cbase;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) E[k] = group_sum<G>(E[k]);
    if (MODE == 0 || MODE == 3) {
        if (MODE == 0 && fl.efg) {
#pragma unroll
            for (int k = 0; k < 6; ++k) Gd[k] = group_sum<G>(Gd[k]);
        }
        if (fl.forces) {
#pragma unroll
            for (int k = 0; k < 3; ++k) F[k] = group_sum<G>(F[k]);
        }
    }
    if (active && sub == 0) {
        if (MODE == 1 || MODE == 2 || fl.field) { ef[i] = E[0]; ef[n + i] = E[1]; ef[2 * n + i] = E[2]; }
        if (MODE == 0 && fl.efg)
            for (int k = 0; k < 6; ++k) efg[(size_t)k * n + i] = Gd[k];
        if ((MODE == 0 || MODE == 3) && fl.forces) { fo[i] = F[0]; fo[n + i] = F[1]; fo[2 * n + i] = F[2]; }
    }
    if (MODE == 0 || MODE == 3) {
        double v[8] = {u, S[0], S[1], S[2], S[3], S[4], S[5], 0.0};
        block_partials<8>(v, part);
    }
}

// Mixed path: the dipole field operator E_i = sum_j T2(r_ij) mu_j in FP32
// arithmetic with FP64 accumulation.  The minimum image comes exactly from the
// 32-bit fixed-point fractional coordinates (the wrapped integer difference is
// d - NINT(d)), r = A d in FP32; erfc, exp and the contraction in FP32.  r_ji
// is exactly -r_ij, so the operator stays symmetric, which the conjugate
// gradient needs.
template <int G>
__global__ void __launch_bounds__(256) k_ewald_dd32(int n, const uint32_t* __restrict__ fx,
                                                    const double* __restrict__ mu, CellP c,
                                                    const int* __restrict__ nbr, const int* __restrict__ cnt, int cap,
                                                    float cutsq, float alpha, double* __restrict__ ef) {
    const int gid = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    const int sub = threadIdx.x & (G - 1);
    const bool active = gid < n;
    const int i = active ? gid : 0;
    const float sc = 2.3283064365386963e-10f;   // 2^-32
    const float A0 = (float)c.A[0], A1 = (float)c.A[1], A2 = (float)c.A[2];
    const float A3 = (float)c.A[3], A4 = (float)c.A[4], A5 = (float)c.A[5];
    const float A6 = (float)c.A[6], A7 = (float)c.A[7], A8 = (float)c.A[8];
    const float a2 = alpha * alpha;
    const float two_a_rpi = 2.0f * alpha * 0.5641895835477563f;          // 2 a / sqrt(pi)
    const float four3_a3_rpi = 4.0f / 3.0f * a2 * alpha * 0.5641895835477563f;
    double E0 = 0.0, E1 = 0.0, E2 = 0.0;
    if (active) {
        const uint32_t u1 = fx[i], u2 = fx[n + i], u3 = fx[2 * n + i];
        const int m = cnt[i];
        const int* row = nbr + (size_t)i * cap;
        for (int k = sub; k < m; k += G) {
            const int j = row[k];
            const float d0 = (float)(int)(u1 - fx[j]) * sc;
            const float d1 = (float)(int)(u2 - fx[n + j]) * sc;
            const float d2 = (float)(int)(u3 - fx[2 * n + j]) * sc;
            const float rx = fmaf(d0, A0, fmaf(d1, A1, d2 * A2));
            const float ry = fmaf(d0, A3, fmaf(d1, A4, d2 * A5));
            const float rz = fmaf(d0, A6, fmaf(d1, A7, d2 * A8));
            const float r2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
            if (r2 > cutsq) continue;
            const float dm1 = rsqrtf(r2);
            const float d = r2 * dm1;
            const float dm2 = dm1 * dm1, dm3 = dm1 * dm2, dm5 = dm3 * dm2;
            const float ex = __expf(-a2 * r2);
            const float F1 = erfcf(alpha * d) + two_a_rpi * d * ex;
            const float F2 = F1 + four3_a3_rpi * r2 * d * ex;
            const float a1c = F1 * dm3, b2c = 3.0f * F2 * dm5;
            const float mj0 = (float)mu[j], mj1 = (float)mu[n + j], mj2 = (float)mu[2 * n + j];
            const float rb = fmaf(rx, mj0, fmaf(ry, mj1, rz * mj2)) * b2c;
            E0 += (double)fmaf(rx, rb, -mj0 * a1c);
            E1 += (double)fmaf(ry, rb, -mj1 * a1c);
            E2 += (double)fmaf(rz, rb, -mj2 * a1c);
        }
    }
    E0 = group_sum<G>(E0);
    E1 = group_sum<G>(E1);
    E2 = group_sum<G>(E2);
    if (active && sub == 0) { ef[i] = E0; ef[n + i] = E1; ef[2 * n + i] = E2; }
}

// The same operator from the per-step pair table written by the charge pass:
// the Coulomb list compacted to the entries inside the cutoff, with
// A1 = F1/r^3 and B2 = 3 F2/r^5 per entry (FP64 rounded to FP32), so no
// special functions per iteration.  Each neighbour is one 32-byte gather of
// its record (fixed-point coordinates, FP32 dipole); r comes from the exact
// fixed-point difference, so the operator stays symmetric.  Two entries per
// lane are in flight per sweep.
__global__ void k_dd_records(int n, const uint32_t* __restrict__ fx, const double* __restrict__ mu,
                             uint4* __restrict__ rec) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    rec[2 * i] = make_uint4(fx[i], fx[n + i], fx[2 * n + i], 0u);
    rec[2 * i + 1] = make_uint4(__float_as_uint((float)mu[i]), __float_as_uint((float)mu[n + i]),
                                __float_as_uint((float)mu[2 * n + i]), 0u);
}

// One atom's 32-byte record (fixed-point coordinates, then the FP32 dipole)
// in one 256-bit load: a scattered gather costs one L1 request per record
// instead of two, and the operator below is bound by those requests.
__device__ __forceinline__ void ld_rec32(const uint4* __restrict__ p, uint4& a, uint4& b) {
    asm("ld.global.nc.v8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(a.x), "=r"(a.y), "=r"(a.z), "=r"(a.w), "=r"(b.x), "=r"(b.y), "=r"(b.z), "=r"(b.w)
        : "l"(p));
}

template <int G>
__global__ void __launch_bounds__(256) k_ewald_ddtab(int n, const uint4* __restrict__ rec, CellP c,
                                                     const int* __restrict__ nbr, const int* __restrict__ cnt, int cap,
                                                     const float2* __restrict__ tab, double* __restrict__ ef) {
    const int gid = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    const int sub = threadIdx.x & (G - 1);
    const bool active = gid < n;
    const int i = active ? gid : 0;
    const float sc = 2.3283064365386963e-10f;   // 2^-32
    const float A0 = (float)c.A[0], A1 = (float)c.A[1], A2 = (float)c.A[2];
    const float A3 = (float)c.A[3], A4 = (float)c.A[4], A5 = (float)c.A[5];
    const float A6 = (float)c.A[6], A7 = (float)c.A[7], A8 = (float)c.A[8];
    double E0 = 0.0, E1 = 0.0, E2 = 0.0;
    if (active) {
        const uint4 ri = rec[2 * i];
        const int m = cnt[i];
        const int* row = nbr + (size_t)i * cap;
        const float2* trow = tab + (size_t)i * cap;
        auto term = [&](float2 t, const uint4& p, const uint4& q) {
            const float d0 = (float)(int)(ri.x - p.x) * sc;
            const float d1 = (float)(int)(ri.y - p.y) * sc;
            const float d2 = (float)(int)(ri.z - p.z) * sc;
            const float rx = fmaf(d0, A0, fmaf(d1, A1, d2 * A2));
            const float ry = fmaf(d0, A3, fmaf(d1, A4, d2 * A5));
            const float rz = fmaf(d0, A6, fmaf(d1, A7, d2 * A8));
            const float mj0 = __uint_as_float(q.x), mj1 = __uint_as_float(q.y), mj2 = __uint_as_float(q.z);
            const float rb = fmaf(rx, mj0, fmaf(ry, mj1, rz * mj2)) * t.y;
            E0 += (double)fmaf(rx, rb, -mj0 * t.x);
            E1 += (double)fmaf(ry, rb, -mj1 * t.x);
            E2 += (double)fmaf(rz, rb, -mj2 * t.x);
        };
        int k = sub;
        for (; k + G < m; k += 2 * G) {
            const int ja = row[k], jb = row[k + G];
            const float2 ta = trow[k], tb = trow[k + G];
            uint4 pa, qa, pb, qb;
            ld_rec32(rec + 2 * ja, pa, qa);
            ld_rec32(rec + 2 * jb, pb, qb);
            term(ta, pa, qa);
            term(tb, pb, qb);
        }
        if (k < m) {
            const int ja = row[k];
            uint4 pa, qa;
            ld_rec32(rec + 2 * ja, pa, qa);
            term(trow[k], pa, qa);
        }
    }
    E0 = group_sum<G>(E0);
    E1 = group_sum<G>(E1);
    E2 = group_sum<G>(E2);
    if (active && sub == 0) { ef[i] = E0; ef[n + i] = E1; ef[2 * n + i] = E2; }
}

void launch_ewald_ddtab(cudaStream_t st, int n, const uint32_t* fx, const double* mu, CellP c, const int* nbr,
                        const int* cnt, int cap, const float2* tab, uint4* rec, double* ef, int g) {
    k_dd_records<<<(n + 255) / 256, 256, 0, st>>>(n, fx, mu, rec);
    const int blocks = (int)(((size_t)n * g + 255) / 256);
#define DDT(G) k_ewald_ddtab<G><<<blocks, 256, 0, st>>>(n, rec, c, nbr, cnt, cap, tab, ef)
    if (g == 8) DDT(8);
    else if (g == 32) DDT(32);
    else DDT(16);
#undef DDT
}

// g: lanes per atom (8, 16 or 32; the autotuner's choice).
void launch_ewald_dd32(cudaStream_t st, int n, const uint32_t* fx, const double* mu, CellP c, const NList& l,
                       double cutsq, double alpha, double* ef, int g) {
    const int blocks = (int)(((size_t)n * g + 255) / 256);
#define DD32(G) k_ewald_dd32<G><<<blocks, 256, 0, st>>>(n, fx, mu, c, l.nbr, l.cnt, l.cap, (float)cutsq, (float)alpha, ef)
    if (g == 8) DD32(8);
    else if (g == 32) DD32(32);
    else DD32(16);
#undef DD32
}

// g: lanes per atom (8, 16 or 32; the autotuner's choice).
void launch_ewald_dir(cudaStream_t st, int n, const double* sx, const double* sy, const double* sz,
                      const int* type, const double* q, const double* mu, CellP c, const NList& l,
                      const PairConst* pc, DirFlags fl, double* ef, double* efg, double* f, Partials& part,
                      DevScalars* d, int g) {
    const int threads = 256;
    const int blocks = (int)(((size_t)n * g + threads - 1) / threads);
#define DIR(G, M, P) k_ewald_dir<G, M><<<blocks, threads, 0, st>>>(n, sx, sy, sz, type, q, mu, c, l.nbr, l.cnt, l.cap, \
                                                                   pc, fl, ef, efg, f, P)
    if (!q) {
        if (g == 8) DIR(8, 1, nullptr);
        else if (g == 32) DIR(32, 1, nullptr);
        else DIR(16, 1, nullptr);
        return;
    }
    if (fl.qq && fl.field && !fl.qd && !fl.dd && !fl.efg && !fl.forces) {   // the charges' field alone
        if (g == 8) DIR(8, 2, nullptr);
        else if (g == 32) DIR(32, 2, nullptr);
        else DIR(16, 2, nullptr);
        return;
    }
    if (!fl.efg) {   // no field gradient this step
        if (g == 8) DIR(8, 3, part.buf);
        else if (g == 32) DIR(32, 3, part.buf);
        else DIR(16, 3, part.buf);
    } else if (g == 8) DIR(8, 0, part.buf);
    else if (g == 32) DIR(32, 0, part.buf);
    else DIR(16, 0, part.buf);
#undef DIR
    launch_reduce_partials(st, part.buf, blocks, 8, d->dir, 0);
}

}  // namespace mdff
