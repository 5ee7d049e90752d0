// pair.cu -- short-range pair loop: n-m Lennard-Jones, BMH / BMHFTD with
// Tang-Toennies dispersion damping, and Morse.
//
// Replaces engforce_nmlj_pbc (src/field.f90:1181-1345), engforce_bmhftd_pbc
// (src/field.f90:2876-3026) and engforce_morse_pbc (src/field.f90:3039-3185).
// Layout: G lanes cooperate on one atom's full neighbour row (ELL); every
// lane accumulates the force on atom i only, so there are no atomics and the
// result is deterministic.  Energies, virial and stress are halved per
// ordered pair (each unordered pair is visited from both ends).
#include "common.cuh"

namespace mdff {

__device__ __forceinline__ void tt_damp(double b, double c, double r, int k, double& f, double& fd) {
    tt_damp_d(b, c, r, k, f, fd);
}

__device__ __forceinline__ double ipow_half(double x, double p) {
    // x^(p/2): repeated multiplication when p/2 is a small integer, pow otherwise.
    double h = 0.5 * p;
    int k = (int)h;
    if ((double)k == h && k >= 0 && k <= 16) {
        double r = 1.0, b = x;
        while (k) {
            if (k & 1) r *= b;
            b *= b;
            k >>= 1;
        }
        return r;
    }
    return pow(x, h);
}

template <int G>
__global__ void __launch_bounds__(256) k_pair(int n, const double* __restrict__ sx, const double* __restrict__ sy,
                                              const double* __restrict__ sz, const int* __restrict__ type, CellP c,
                                              const int* __restrict__ nbr, const int* __restrict__ cnt, int cap,
                                              const PairConst* __restrict__ pc, PairFlags fl, double* fx,
                                              double* fy, double* fz, double* part) {
    const int gid = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    const int sub = threadIdx.x & (G - 1);
    const bool active = gid < n;
    const int i = active ? gid : 0;
    double f0 = 0.0, f1 = 0.0, f2 = 0.0;
    double acc[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};   // u_lj vir_lj u_bmh vir_bmh u_mor vir_mor tau(6 -> 4 more below)
    double tau[6] = {0, 0, 0, 0, 0, 0};
    if (active) {
        const double si1 = sx[i], si2 = sy[i], si3 = sz[i];
        const int ti = type[i];
        const int m = cnt[i];
        const int* row = nbr + (size_t)i * cap;
        for (int k = sub; k < m; k += G) {
            const int j = row[k];
            double rx, ry, rz;
            const double rsq = pairvec_exact(c, si1, si2, si3, sx[j], sy[j], sz[j], rx, ry, rz);
            const PairConst& P = pc[ti * NT + type[j]];
            if (!(rsq < P.rcutsq)) continue;
            double w = 0.0;
            if (fl.lj) {
                const double sr2 = P.sigsq / rsq;
                const double srp = ipow_half(sr2, P.plj);
                const double srq = ipow_half(sr2, P.qlj);
                double u = P.epsp * (P.plj * srq - P.qlj * srp);
                if (fl.trunc == 1) u -= P.uc;
                if (fl.trunc == 2) u += P.uc1 * rsq - P.uc2;
                const double wl = P.fc * (srq - srp) * sr2;
                acc[0] += 0.5 * u;
                acc[1] += 0.5 * wl * rsq;
                w += wl;
            }
            if ((fl.bmh || fl.bmhftd) && P.A != 0.0) {
                const double ir2 = 1.0 / rsq;
                const double d = sqrt(rsq);
                const double erh = P.A * exp(-P.B * d);
                double ir6 = ir2 * ir2 * ir2;
                double ir8 = ir6 * ir2;
                ir6 *= P.C;
                ir8 *= P.D;
                double ir6d = ir6, ir8d = ir8, fd6 = 0.0, fd8 = 0.0;
                if (fl.bmhftd) {
                    double f6, f8;
                    tt_damp(P.BD, 1.0, d, 6, f6, fd6);
                    tt_damp(P.BD, 1.0, d, 8, f8, fd8);
                    ir6d = ir6 * f6;
                    ir8d = ir8 * f8;
                }
                const double wb = (P.B * erh - 6.0 * ir6d / d - 8.0 * ir8d / d + ir6 * fd6 + ir8 * fd8) / d;
                acc[2] += 0.5 * (erh - ir6d - ir8d);
                acc[3] += 0.5 * wb * rsq;
                w += wb;
            }
            if (fl.morse) {
                const double d = sqrt(rsq);
                const double e = exp(-d * P.rhomor) * P.rs;
                const double em1 = e - 1.0;
                acc[4] += 0.5 * P.epsmor * (em1 * em1 - 1.0);
                const double wm = 2.0 * P.epsmor * P.rhomor * e * em1 / d;
                acc[5] += 0.5 * wm * rsq;
                w += wm;
            }
            f0 += w * rx;
            f1 += w * ry;
            f2 += w * rz;
            const double hw = 0.5 * w;
            tau[0] += hw * rx * rx;
            tau[1] += hw * ry * ry;
            tau[2] += hw * rz * rz;
            tau[3] += hw * rx * ry;
            tau[4] += hw * rx * rz;
            tau[5] += hw * ry * rz;
        }
    }
    f0 = group_sum<G>(f0);
    f1 = group_sum<G>(f1);
    f2 = group_sum<G>(f2);
    if (active && sub == 0) {
        fx[i] = f0;
        fy[i] = f1;
        fz[i] = f2;
    }
    double v[12] = {acc[0], acc[1], acc[2], acc[3], acc[4], acc[5], tau[0], tau[1], tau[2], tau[3], tau[4], tau[5]};
    block_partials<12>(v, part);
}

void launch_pair(cudaStream_t st, int n, const double* sx, const double* sy, const double* sz, const int* type,
                 CellP c, const NList& l, const PairConst* pc, PairFlags fl, double* fx, double* fy, double* fz,
                 Partials& part, DevScalars* d) {
    constexpr int G = 8;
    const int threads = 256;
    const int blocks = (int)(((size_t)n * G + threads - 1) / threads);
    k_pair<G><<<blocks, threads, 0, st>>>(n, sx, sy, sz, type, c, l.nbr, l.cnt, l.cap, pc, fl, fx, fy, fz, part.buf);
    // u_lj vir_lj u_bmh vir_bmh u_mor vir_mor, then the stress sums
    launch_reduce_partials(st, part.buf, blocks, 12, d->nonb, 0);
}

}  // namespace mdff
