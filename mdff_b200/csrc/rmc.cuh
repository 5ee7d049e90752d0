// Reverse Monte Carlo on the pair distribution (rmc_main, src/rmc.f90:196-640,
// with g(r) from gr_main, src/radial_distrib.f90) on the device.
//
// g(r): every ordered pair (ia, ja != ia) within cutgr adds to bin
// INT(r / resg) of the all-pairs row and of the ordered type row (ita, jta),
// r from the minimum-image fractional difference in the reference's order of
// operations; rmc_gr (src/rmc.f90:1431-1497) normalises row (it1 <= it2) by
// 4 pi (res r^2 + res^3 / 12) / V x natmi(it1) natmi(it2) (natm^2 for row 0).
//
// The Markov chain runs in one persistent CTA: a trial move changes only the
// N - 1 pairs of the moved atom, so the counts are updated from those pairs
// (old bin out, new bin in) -- exactly the integers a full recount gives --
// then chi^2, the reference's per-component Metropolis tests and the accept /
// reject all stay on the device.  Random numbers come from a stream in device
// memory (the caller's, or a counter-based generator's), consumed in the
// reference's order: particle, three displacement components, then one for
// each chi^2 component whose change is not negative.
#pragma once
#include "common.cuh"

namespace mdff {

constexpr int RMC_THREADS = 1024;
constexpr int RMC_MAX_BINS = 4096;
constexpr int RMC_NT_MAX = 4;
constexpr int RMC_SMEM_INTS = RMC_MAX_BINS * 4;   // delta counts, (1 + nt^2) rows of nbins

// the binning of one pair distance
struct RmcBin {
    double cut2, resg;
    int nbins, ntype;
};

struct RmcConst {
    int n, ntype, nbins, nrow;   // nrow = 1 + ntype^2 count rows (row 0 all pairs, 1 + ita*ntype + jta)
    int npairs;                  // ntype (ntype + 1) / 2
    RmcBin bin;
    double dmax[3];              // max_displacement / ANORM(d): the fractional displacement bound
    double temp[6];              // temp_rmc(1..5) and the total's
    double natm, natmi[RMC_NT_MAX];
    double volnorm[RMC_MAX_BINS];   // 4 pi (res rr^2 + res^3/12) / V per bin, in the reference's order
};

// bin of the pair (s_i, s_j) as gr_main forms it, or -1 beyond cutgr
__device__ __forceinline__ int rmc_bin(const CellP& c, const RmcBin& k, double s1, double s2, double s3, double t1,
                                       double t2, double t3) {
    double rx, ry, rz;
    const double rsq = pairvec_exact(c, s1, s2, s3, t1, t2, t3, rx, ry, rz);
    if (!(rsq < k.cut2)) return -1;
    const int b = (int)__ddiv_rn(__dsqrt_rn(rsq), k.resg);
    return b < k.nbins ? b : -1;
}

// gr_main over all ordered pairs: one thread per atom ia, counts by global
// integer atomics (order-free)
__global__ void k_gr_full(int n, const double* __restrict__ s, const int* __restrict__ type, CellP c, RmcBin k,
                          int* hist) {
    const int ia = blockIdx.x * blockDim.x + threadIdx.x;
    if (ia >= n) return;
    const double s1 = s[ia], s2 = s[(size_t)n + ia], s3 = s[2 * (size_t)n + ia];
    const int ti = type[ia];
    for (int ja = 0; ja < n; ++ja) {
        if (ja == ia) continue;
        const int b = rmc_bin(c, k, s1, s2, s3, s[ja], s[(size_t)n + ja], s[2 * (size_t)n + ja]);
        if (b < 0) continue;
        atomicAdd(&hist[b], 1);
        atomicAdd(&hist[(size_t)(1 + ti * k.ntype + type[ja]) * k.nbins + b], 1);
    }
}

// rmc_gr's normalised g(r) of counts h, row mp (0 = all, then it1 <= it2)
__device__ __forceinline__ double rmc_g(const RmcConst& k, const int* h, const int* d, int mp, int b) {
    int row, it1 = 0, it2 = 0;
    if (mp == 0) row = 0;
    else {
        int m = mp - 1;
        for (it1 = 0; it1 < k.ntype; ++it1) {
            const int len = k.ntype - it1;
            if (m < len) { it2 = it1 + m; break; }
            m -= len;
        }
        row = 1 + it1 * k.ntype + it2;
    }
    const int cnt = h[row * k.nbins + b] + (d ? d[row * k.nbins + b] : 0);
    // vol * natm * natm and vol * natmi(it1) * natmi(it2), left to right
    const double den = mp == 0 ? __dmul_rn(__dmul_rn(k.volnorm[b], k.natm), k.natm)
                               : __dmul_rn(__dmul_rn(k.volnorm[b], k.natmi[it1]), k.natmi[it2]);
    return __ddiv_rn((double)cnt, den);
}

// Chain state carried across launches (a launch ends when the neighbour
// list must be rebuilt).
struct RmcOut {
    long long kall, kacc, used;   // trial moves, accepted count (starting at 1 as the reference), uniforms consumed
    double chisq[6];              // of the last accepted configuration
    double maxd;                  // largest displacement of an atom since the list was built (A)
    int status;                   // 0 done, 1 the random stream ran out, 2 the list needs rebuilding
    int started;                  // chi^2 of the start evaluated
};

// Neighbour lists of the chain: for each atom every other atom within
// cut + skin (full lists), capacity cap per atom; *ovf = largest count seen
// beyond cap.
__global__ void k_rmc_list(int n, const double* __restrict__ s, CellP c, double rl2, int cap, int* nbr, int* cnt,
                           int* ovf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double s1 = s[i], s2 = s[(size_t)n + i], s3 = s[2 * (size_t)n + i];
    int k = 0;
    for (int j = 0; j < n; ++j) {
        if (j == i) continue;
        double rx, ry, rz;
        const double rsq = pairvec_exact(c, s1, s2, s3, s[j], s[(size_t)n + j], s[2 * (size_t)n + j], rx, ry, rz);
        if (rsq < rl2) {
            if (k < cap) nbr[(size_t)i * cap + k] = j;
            ++k;
        }
    }
    cnt[i] = min(k, cap);
    if (k > cap) atomicMax(ovf, k);
}

// The chain: until kacc reaches acc_max or kall reaches max_trials.  s: the
// fractional coordinates [3][n] (updated); hist: counts [nrow][nbins]
// (updated); gexp [npairs+1][nbins]; uni: nuni uniforms in [0, 1).
__global__ void __launch_bounds__(RMC_THREADS) k_rmc_chain(double* s, const int* __restrict__ type, CellP c,
                                                          const RmcConst* __restrict__ kp, int* hist,
                                                          const double* __restrict__ gexp,
                                                          const double* __restrict__ uni, long long nuni,
                                                          long long acc_max, long long max_trials,
                                                          const int* __restrict__ nbr, const int* __restrict__ ncnt,
                                                          int cap, const double* __restrict__ sb, double dlim,
                                                          RmcOut* out) {
    extern __shared__ int dcnt[];
    __shared__ double wsum[RMC_THREADS / 32];
    __shared__ double chi_old[6], chi_new[6], snew[3], disp[3];
    __shared__ int sh_i, sh_acc, sh_stop;
    __shared__ long long u_at;
    const RmcConst& k = *kp;
    const int n = k.n, tid = threadIdx.x;
    const int ncount = k.nrow * k.nbins;
    const int nterm = (k.npairs + 1) * k.nbins;
    for (int q = tid; q < ncount; q += RMC_THREADS) dcnt[q] = 0;
    // chi^2 (eval_chisq_rmc, src/rmc.f90:667-690) of the terms q = bin x
    // (npairs + 1) + mp by a fixed tree: thread t sums terms t, t + 1024, ...
    // in order, then a shuffle-down tree within each warp and the same tree
    // over the 32 warp sums (the oracle restates this order)
    const int lane = tid & 31, warp = tid >> 5;
    auto chisq_of = [&](const int* d) -> double {
        double v = 0.0;
        for (int q = tid; q < nterm; q += RMC_THREADS) {
            const int b = q / (k.npairs + 1), mp = q - b * (k.npairs + 1);
            const double dv = __dsub_rn(rmc_g(k, hist, d, mp, b), gexp[(size_t)mp * k.nbins + b]);
            v = __dadd_rn(v, __dmul_rn(dv, dv));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = __dadd_rn(v, __shfl_down_sync(0xffffffffu, v, o));
        if (lane == 0) wsum[warp] = v;
        __syncthreads();
        double t = 0.0;
        if (warp == 0) {
            t = wsum[lane];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t = __dadd_rn(t, __shfl_down_sync(0xffffffffu, t, o));
        }
        __syncthreads();
        return t;   // valid in thread 0
    };
    __shared__ double sh_maxd;
    const int started = out->started;
    const double c0 = started ? 0.0 : chisq_of(nullptr);
    if (tid == 0) {
        if (started) {
            for (int q = 0; q < 6; ++q) chi_old[q] = out->chisq[q];
        } else {
            for (int q = 0; q < 6; ++q) chi_old[q] = 0.0;
            chi_old[0] = c0;
            chi_old[5] = c0;
        }
        u_at = started ? out->used : 0;
        sh_maxd = started ? out->maxd : 0.0;
        sh_stop = 0;
    }
    long long kall = started ? out->kall : 1, kacc = started ? out->kacc : 1;
    __syncthreads();
    while (kacc < acc_max && kall < max_trials) {
        if (sh_maxd > dlim) {   // an atom moved too far for the list: rebuild first
            if (tid == 0) sh_stop = 2;
            break;
        }
        ++kall;
        // rmc_move (src/rmc.f90:1366-1428): particle and displacement
        if (tid == 0) {
            if (u_at + 4 > nuni) sh_stop = 1;
            else {
                const int i = (int)(uni[u_at] * n);
                sh_i = i < n ? i : n - 1;
                for (int d = 0; d < 3; ++d) {
                    const double x = uni[u_at + 1 + d];
                    disp[d] = __dmul_rn(k.dmax[d], __dsub_rn(__dmul_rn(2.0, x), 1.0));
                    double v = __dadd_rn(s[(size_t)d * n + sh_i], disp[d]);
                    if (v > 1.0 || v < 0.0) v = __dsub_rn(v, round(v));
                    snew[d] = v;
                }
                u_at += 4;
            }
        }
        __syncthreads();
        if (sh_stop) break;
        const int i = sh_i;
        const double o1 = s[i], o2 = s[(size_t)n + i], o3 = s[2 * (size_t)n + i];
        const int ti = type[i];
        const int nn = ncnt[i];
        const int* nl = nbr + (size_t)i * cap;
        for (int q = tid; q < nn; q += RMC_THREADS) {
            const int j = nl[q];
            const double t1 = s[j], t2 = s[(size_t)n + j], t3 = s[2 * (size_t)n + j];
            const int tj = type[j];
            const int bo = rmc_bin(c, k.bin, o1, o2, o3, t1, t2, t3);
            const int bn = rmc_bin(c, k.bin, snew[0], snew[1], snew[2], t1, t2, t3);
            if (bo == bn) continue;
            // the pair appears as (i, j) and (j, i): twice in row 0, once in each ordered type row
            if (bo >= 0) {
                atomicSub(&dcnt[bo], 2);
                atomicSub(&dcnt[(1 + ti * k.ntype + tj) * k.nbins + bo], 1);
                atomicSub(&dcnt[(1 + tj * k.ntype + ti) * k.nbins + bo], 1);
            }
            if (bn >= 0) {
                atomicAdd(&dcnt[bn], 2);
                atomicAdd(&dcnt[(1 + ti * k.ntype + tj) * k.nbins + bn], 1);
                atomicAdd(&dcnt[(1 + tj * k.ntype + ti) * k.nbins + bn], 1);
            }
        }
        __syncthreads();
        const double c1 = chisq_of(dcnt);
        // Metropolis per component (src/rmc.f90:521-540); the total decides
        if (tid == 0) {
            chi_new[0] = c1;
            for (int q = 1; q < 5; ++q) chi_new[q] = 0.0;
            chi_new[5] = c1;
            bool acc6 = false;
            for (int q = 0; q < 6 && !sh_stop; ++q) {
                const double dq = __dsub_rn(chi_new[q], chi_old[q]);
                bool a;
                if (dq < 0.0) a = true;
                else {
                    if (u_at + 1 > nuni) { sh_stop = 1; break; }
                    const double metro = exp(-__dmul_rn(dq, 0.5) / k.temp[q]);
                    a = metro >= uni[u_at];
                    ++u_at;
                }
                if (q == 5) acc6 = a;
            }
            sh_acc = acc6 && !sh_stop;
            if (sh_acc) {
                for (int q = 0; q < 6; ++q) chi_old[q] = chi_new[q];
                for (int d = 0; d < 3; ++d) s[(size_t)d * n + i] = snew[d];
                // displacement from the list's build position
                double rx, ry, rz;
                const double d2 = pairvec_exact(c, snew[0], snew[1], snew[2], sb[i], sb[(size_t)n + i],
                                                sb[2 * (size_t)n + i], rx, ry, rz);
                sh_maxd = fmax(sh_maxd, sqrt(d2));
            } else if (!sh_stop) {
                // the rejected atom goes back by the displacement (src/rmc.f90:628-636)
                for (int d = 0; d < 3; ++d) s[(size_t)d * n + i] = __dsub_rn(snew[d], disp[d]);
            }
        }
        __syncthreads();
        if (sh_stop) { --kall; break; }
        if (sh_acc) {
            ++kacc;
            for (int q = tid; q < ncount; q += RMC_THREADS) hist[q] += dcnt[q];
        }
        for (int q = tid; q < ncount; q += RMC_THREADS) dcnt[q] = 0;
        __syncthreads();
    }
    if (tid == 0) {
        out->kall = kall;
        out->kacc = kacc;
        out->used = u_at;
        for (int q = 0; q < 6; ++q) out->chisq[q] = chi_old[q];
        out->maxd = sh_maxd;
        out->status = sh_stop;
        out->started = 1;
    }
}

// counter-based uniforms in [0, 1): splitmix64 of (seed, index), 53 bits
__global__ void k_rmc_uniforms(long long count, unsigned long long seed, double* u) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(t + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    u[t] = (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

}  // namespace mdff
