// ewald_recip.cu -- reciprocal-space part of the multipole Ewald sum.
//
// Replaces multipole_ES_rec (src/field.f90:2646-2873) and the k-vector set of
// kpoint_sum_init (src/kspace.f90:142-207).  The reference loops over k in the
// outer loop and over all atoms twice inside, with one sin/cos per (k, atom).
// Here:
//   pass 1 (k_sfac):  S(k) = sum_i (q_i + i k.mu_i) e^{i k.r_i}
//       one thread per (k-column (nx,ny), chunk of CH consecutive nz); the
//       phase is exact from direct coordinates, e^{ik.r} = e^{2 pi i n.s},
//       with one sincospi per (atom, chunk) and a complex rotation by
//       e^{2 pi i s_z} per further nz.  The atoms are split over blockIdx.y;
//       the per-chunk partial sums are added in a fixed order (k_sfac_reduce),
//       which also forms A_k S(k), the energy and the stress per k.
//   pass 2 (k_kfield): per atom, E_i = -sum_k k A_k Im(S* e^{ik.r_i}) and the
//       field gradient sum_k k k^T A_k Re(S* e^{ik.r_i}); one thread per atom,
//       k-columns staged in shared memory, split over blockIdx.y and reduced
//       in a fixed order (k_kfield_reduce), which also forms the forces
//       F_i = q_i E_i + G_i mu_i (src/field.f90:2776-2789).
// The k set is the full rectangle nx in [0,kx], ny in [-ky,ky], nz in
// [-kz,kz] with A_k = 0 on the half that the reference skips.
#include "common.cuh"
#include "ewald_tc.cuh"
#include "ewald_tc4.cuh"

namespace mdff {

constexpr int SF_THREADS = 128;
constexpr int SF_TILE = 64;

template <int CH>
__global__ void __launch_bounds__(SF_THREADS) k_sfac(int n, int natom_chunk, const double* __restrict__ sx,
                                                     const double* __restrict__ sy, const double* __restrict__ sz,
                                                     const double* __restrict__ q, const double* __restrict__ mu,
                                                     CellP c, int kx, int ky, int kz, int ncol, int ncolblk,
                                                     int nchunk, int with_q, int with_mu, double* __restrict__ part_re,
                                                     double* __restrict__ part_im, const int* __restrict__ items,
                                                     int nitems) {
    __shared__ double t_s1[SF_TILE], t_s2[SF_TILE], t_s3[SF_TILE], t_q[SF_TILE];
    __shared__ double t_m1[SF_TILE], t_m2[SF_TILE], t_m3[SF_TILE], t_cs[SF_TILE], t_sn[SF_TILE];
    // one (column, nz chunk) per thread: the whole rectangle, or the work list
    // of the vectors inside a k sphere (items, one entry per thread)
    int h, col;
    bool valid;
    if (items) {
        const int t = blockIdx.x * SF_THREADS + threadIdx.x;
        valid = t < nitems;
        const int tt = valid ? t : nitems - 1;
        col = items[2 * tt];
        h = items[2 * tt + 1];
    } else {
        h = blockIdx.x / ncolblk;
        col = (blockIdx.x % ncolblk) * SF_THREADS + threadIdx.x;
        valid = col < ncol;
    }
    const int p = blockIdx.y;
    const int ny_n = 2 * ky + 1;
    const int colc = col < ncol ? col : ncol - 1;
    const double nx = (double)(colc / ny_n);
    const double ny = (double)(colc % ny_n - ky);
    const double nz0 = (double)(-kz + h * CH);
    double are[CH], aim[CH];
#pragma unroll
    for (int m = 0; m < CH; ++m) { are[m] = 0.0; aim[m] = 0.0; }
    const int a0 = p * natom_chunk;
    const int a1 = min(n, a0 + natom_chunk);
    for (int base = a0; base < a1; base += SF_TILE) {
        __syncthreads();
        if (threadIdx.x < SF_TILE) {
            int ia = base + threadIdx.x;
            if (ia < a1) {
                double s1 = sx[ia], s2 = sy[ia], s3 = sz[ia];
                t_s1[threadIdx.x] = s1; t_s2[threadIdx.x] = s2; t_s3[threadIdx.x] = s3;
                t_q[threadIdx.x] = with_q ? q[ia] : 0.0;
                double m0 = 0, m1 = 0, m2 = 0;
                if (with_mu) { m0 = mu[ia]; m1 = mu[n + ia]; m2 = mu[2 * n + ia]; }
                // 2 pi (b_j . mu), b_j = column j of B: k.mu = nx*t_m1 + ny*t_m2 + nz*t_m3
                t_m1[threadIdx.x] = 2.0 * PI * (c.B[0] * m0 + c.B[3] * m1 + c.B[6] * m2);
                t_m2[threadIdx.x] = 2.0 * PI * (c.B[1] * m0 + c.B[4] * m1 + c.B[7] * m2);
                t_m3[threadIdx.x] = 2.0 * PI * (c.B[2] * m0 + c.B[5] * m1 + c.B[8] * m2);
                double fz = s3 - rint(s3);
                double sn, cs;
                sincospi(2.0 * fz, &sn, &cs);
                t_cs[threadIdx.x] = cs; t_sn[threadIdx.x] = sn;
            }
        }
        __syncthreads();
        const int tn = min(SF_TILE, a1 - base);
        for (int t = 0; t < tn; ++t) {
            double ph = fma(nx, t_s1[t], fma(ny, t_s2[t], nz0 * t_s3[t]));
            ph -= rint(ph);
            double sn, cs;
            sincospi(2.0 * ph, &sn, &cs);
            const double qa = t_q[t];
            double km = fma(nx, t_m1[t], fma(ny, t_m2[t], nz0 * t_m3[t]));
            const double dm = t_m3[t], rc = t_cs[t], rs = t_sn[t];
#pragma unroll
            for (int m = 0; m < CH; ++m) {
                are[m] = fma(qa, cs, fma(-km, sn, are[m]));
                aim[m] = fma(qa, sn, fma(km, cs, aim[m]));
                const double cn = cs * rc - sn * rs;
                sn = fma(sn, rc, cs * rs);
                cs = cn;
                km += dm;
            }
        }
    }
    if (valid) {
        const size_t plane = (size_t)ncol * CH * nchunk;
#pragma unroll
        for (int m = 0; m < CH; ++m) {
            size_t idx = (size_t)p * plane + ((size_t)h * CH + m) * ncol + col;
            part_re[idx] = are[m];
            part_im[idx] = aim[m];
        }
    }
}

// Sum the atom-chunk partials in order; A_k S(k); energy and stress per k
// (src/field.f90:2742-2745, 2803-2815).
__global__ void k_sfac_reduce(int P, int ch, int nchunk, int ncol, int nzl, int kx, int ky, int kz,
                              const double* __restrict__ part_re, const double* __restrict__ part_im,
                              const double* __restrict__ Ak, const double* __restrict__ kcoe, CellP c,
                              double* __restrict__ aks, int nrect, int energy, double* partials) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int total = ncol * nzl;
    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    if (t < total) {
        const int col = t % ncol;
        const int mz = t / ncol;          // 0 .. nzl-1
        const size_t plane = (size_t)ncol * ch * nchunk;
        const size_t off = (size_t)mz * ncol + col;   // (h*ch + m) == mz
        const int r = col * nzl + mz;
        const double ak = Ak[r];
        double sr = 0.0, si = 0.0;
        if (ak != 0.0)   // entries outside the work list have no partials
            for (int p = 0; p < P; ++p) {
                sr += part_re[(size_t)p * plane + off];
                si += part_im[(size_t)p * plane + off];
            }
        aks[r] = ak * sr;
        aks[nrect + r] = ak * si;
        if (energy && ak != 0.0) {
            const int ny_n = 2 * ky + 1;
            const double nx = (double)(col / ny_n), ny = (double)(col % ny_n - ky), nz = (double)(mz - kz);
            const double k0 = 2.0 * PI * (nx * c.B[0] + ny * c.B[1] + nz * c.B[2]);
            const double k1 = 2.0 * PI * (nx * c.B[3] + ny * c.B[4] + nz * c.B[5]);
            const double k2 = 2.0 * PI * (nx * c.B[6] + ny * c.B[7] + nz * c.B[8]);
            const double str = (sr * sr + si * si) * ak;
            const double kc = kcoe[r];
            v[0] = str;
            v[1] = (1.0 - kc * k0 * k0) * str;
            v[2] = (1.0 - kc * k1 * k1) * str;
            v[3] = (1.0 - kc * k2 * k2) * str;
            v[4] = -kc * k0 * k1 * str;
            v[5] = -kc * k0 * k2 * str;
            v[6] = -kc * k1 * k2 * str;
        }
    }
    if (energy) block_partials<7>(v, partials);
}

constexpr int KF_THREADS = 128;
constexpr int KF_COLS = 4;   // columns staged per shared-memory round
constexpr int KF_COLS32 = 16;   // the same for the packed FP32 field kernel

template <int GRAD>
__global__ void __launch_bounds__(KF_THREADS) k_kfield(int n, const double* __restrict__ sx, const double* __restrict__ sy,
                                                       const double* __restrict__ sz, CellP c, int kx, int ky, int kz,
                                                       int ncol, int nzl, int cols_per_split,
                                                       const double* __restrict__ aks, int nrect,
                                                       double* __restrict__ fpart, const int* __restrict__ clist,
                                                       const int* __restrict__ czr) {
    extern __shared__ double sm[];
    double* s_re = sm;
    double* s_im = sm + KF_COLS * nzl;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int split = blockIdx.y;
    const int c0 = split * cols_per_split;
    const int c1 = min(ncol, c0 + cols_per_split);
    const bool active = i < n;
    const int ii = active ? i : 0;
    const double s1 = sx[ii], s2 = sy[ii], s3 = sz[ii];
    double rs, rc;
    sincospi(2.0 * (s3 - rint(s3)), &rs, &rc);
    const double dk0 = 2.0 * PI * c.B[2], dk1 = 2.0 * PI * c.B[5], dk2 = 2.0 * PI * c.B[8];
    const int ny_n = 2 * ky + 1;
    double E0 = 0, E1 = 0, E2 = 0;
    double G0 = 0, G1 = 0, G2 = 0, G3 = 0, G4 = 0, G5 = 0;
    // columns c0..c1 of the rectangle, or of the list clist (columns inside a
    // k sphere) with the nz index range [czr[0], czr[0] + czr[1]) of each
    for (int cb = c0; cb < c1; cb += KF_COLS) {
        const int nc = min(KF_COLS, c1 - cb);
        __syncthreads();
        if (clist) {
            for (int t = threadIdx.x; t < nc * nzl; t += blockDim.x) {
                const int cc = t / nzl;
                const size_t r = (size_t)clist[cb + cc] * nzl + (t - cc * nzl);
                s_re[t] = aks[r];
                s_im[t] = aks[(size_t)nrect + r];
            }
        } else {
            for (int t = threadIdx.x; t < nc * nzl; t += blockDim.x) {
                s_re[t] = aks[(size_t)cb * nzl + t];
                s_im[t] = aks[(size_t)nrect + (size_t)cb * nzl + t];
            }
        }
        __syncthreads();
        for (int cc = 0; cc < nc; ++cc) {
            const int col = clist ? clist[cb + cc] : cb + cc;
            const int mlo = czr ? czr[2 * (cb + cc)] : 0;
            const int mn = czr ? czr[2 * (cb + cc) + 1] : nzl;
            const double nx = (double)(col / ny_n), ny = (double)(col % ny_n - ky), nz0 = (double)(mlo - kz);
            double ph = fma(nx, s1, fma(ny, s2, nz0 * s3));
            ph -= rint(ph);
            double sn, cs;
            sincospi(2.0 * ph, &sn, &cs);
            double k0 = 2.0 * PI * (nx * c.B[0] + ny * c.B[1] + nz0 * c.B[2]);
            double k1 = 2.0 * PI * (nx * c.B[3] + ny * c.B[4] + nz0 * c.B[5]);
            double k2 = 2.0 * PI * (nx * c.B[6] + ny * c.B[7] + nz0 * c.B[8]);
            const double* pr = s_re + cc * nzl + mlo;
            const double* pi = s_im + cc * nzl + mlo;
            for (int m = 0; m < mn; ++m) {
                const double ar = pr[m], ai = pi[m];
                const double recarg = ai * cs - ar * sn;
                E0 = fma(-k0, recarg, E0);
                E1 = fma(-k1, recarg, E1);
                E2 = fma(-k2, recarg, E2);
                if (GRAD) {
                    const double r2 = ar * cs + ai * sn;
                    const double a0 = k0 * r2, a1 = k1 * r2;
                    G0 = fma(k0, a0, G0);
                    G1 = fma(k1, a1, G1);
                    G2 = fma(k2, k2 * r2, G2);
                    G3 = fma(k1, a0, G3);
                    G4 = fma(k2, a0, G4);
                    G5 = fma(k2, a1, G5);
                }
                const double cn = cs * rc - sn * rs;
                sn = fma(sn, rc, cs * rs);
                cs = cn;
                k0 += dk0; k1 += dk1; k2 += dk2;
            }
        }
    }
    if (active) {
        const int nv = GRAD ? 9 : 3;
        double* o = fpart + (size_t)split * nv * n;
        o[i] = E0; o[n + i] = E1; o[2 * n + i] = E2;
        if (GRAD) {
            o[3 * n + i] = G0; o[4 * n + i] = G1; o[5 * n + i] = G2;
            o[6 * n + i] = G3; o[7 * n + i] = G4; o[8 * n + i] = G5;
        }
    }
}

// Sum the column splits in order and scale by 2 (half mesh) * 4 pi / V.
// ef (3n) += E_rec; efg (6n: xx yy zz xy xz yz) += G_rec; fo (3n) +=
// q E_rec + G_rec mu.
__global__ void k_kfield_reduce(int n, int nsplit, int grad, const double* __restrict__ fpart, double scale,
                                const double* __restrict__ q, const double* __restrict__ mu, double* ef,
                                double* efg, double* fo, const double* __restrict__ flow, int nlow) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int nv = grad ? 9 : 3;
    double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int s = 0; s < nsplit; ++s)
        for (int k = 0; k < nv; ++k) v[k] += fpart[((size_t)s * nv + k) * n + i];
    for (int s = 0; s < nlow; ++s)
        for (int k = 0; k < nv; ++k) v[k] += flow[((size_t)s * 9 + k) * n + i];
    for (int k = 0; k < nv; ++k) v[k] *= scale;
    if (ef) { ef[i] += v[0]; ef[n + i] += v[1]; ef[2 * n + i] += v[2]; }
    if (grad && efg)
        for (int k = 0; k < 6; ++k) efg[(size_t)k * n + i] += v[3 + k];
    if (fo) {
        const double qi = q ? q[i] : 0.0;
        double f0 = qi * v[0], f1 = qi * v[1], f2 = qi * v[2];
        if (grad && mu) {
            const double m0 = mu[i], m1 = mu[n + i], m2 = mu[2 * n + i];
            f0 += v[3] * m0 + v[6] * m1 + v[7] * m2;
            f1 += v[6] * m0 + v[4] * m1 + v[8] * m2;
            f2 += v[7] * m0 + v[8] * m1 + v[5] * m2;
        }
        fo[i] += f0; fo[n + i] += f1; fo[2 * n + i] += f2;
    }
}

// ------------------------------------------------------------------------
// Mixed-precision (FP32) kernels.  The phase is exact: fractional coordinates
// as 32-bit fixed point, so n.s mod 1 is an integer multiply-add that wraps
// mod 2^32.  e^{2 pi i t} comes from FP32 sincospif of the top 24 bits (exact
// in a float) with a first-order correction for the low 8 bits
// (|delta| < 3.7e-7 rad); further nz use a per-atom table T_m = e^{2 pi i m s_z}
// built in FP64, so errors do not grow along a column.  The inner loops run on
// packed pairs (fma.rn.f32x2, sm_100): the complex multiply-accumulates are two
// packed FMAs each.  FP32 partial sums are flushed to FP64 every tile of atoms
// (pass 1) or every chunk of 16 k-vectors (pass 2).

__device__ __forceinline__ void phase32(uint32_t ph, float& cs, float& sn) {
    const int p = (int)ph;
    const float hi = (float)(p & ~0xff) * 4.656612873077393e-10f;   // 2^-31: sin(pi*hi) = sin(2 pi t)
    sincospif(hi, &sn, &cs);
    const float d = (float)(p & 0xff) * 1.4629180792671596e-09f;    // 2 pi 2^-32
    const float c2 = fmaf(-sn, d, cs);
    sn = fmaf(cs, d, sn);
    cs = c2;
}

// ---- second-generation FP32 kernels --------------------------------------
// e^{ik.r} = e0 * T_m with T_m = e^{2 pi i m s_z} (m = 0..15) tabulated per atom
// once per position update from FP64, so the error does not grow along nz.
constexpr int TM = 16;     // table length = nz chunk of both passes

// Per-atom phase table T_m, fixed-point coordinates.
__global__ void k_phase_table(int n, const double* __restrict__ sx, const double* __restrict__ sy,
                              const double* __restrict__ sz, uint32_t* __restrict__ fx, float2* __restrict__ tab,
                              double2* __restrict__ tab64) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double s[3] = {sx[i], sy[i], sz[i]};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double w = s[d] - floor(s[d]);
        unsigned long long u = (unsigned long long)llrint(w * 4294967296.0);
        fx[(size_t)d * n + i] = (uint32_t)(u & 0xffffffffull);
    }
    const double z = s[2] - rint(s[2]);
#pragma unroll 4
    for (int m = 0; m < TM; ++m) {
        double t = m * z;
        t -= rint(t);
        double sn, cs;
        sincospi(2.0 * t, &sn, &cs);
        tab[(size_t)i * TM + m] = make_float2((float)cs, (float)sn);
        if (tab64) tab64[(size_t)i * TM + m] = make_double2(cs, sn);
    }
}

// conj-ready FP32 copy of A_k S(k) for the packed field kernel: per k the
// pairs (re, re) and (im, im), each column padded to nzp (a multiple of TM)
// with zeros.
__global__ void k_aks32_pad(int ncol, int nzl, int nzp, int nrect, const double* __restrict__ aks,
                            float4* __restrict__ out) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ncol * nzp) return;
    int col = t / nzp, m = t % nzp;
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (m < nzl) {
        size_t r = (size_t)col * nzl + m;
        const float re = (float)aks[r], im = (float)aks[nrect + r];
        v = make_float4(re, re, im, im);
    }
    out[t] = v;
}

// Pass 1: each thread sweeps two (column, chunk) work items over the same
// atoms, so one shared-memory load of the atom's table entry T_m serves both.
// The amplitude of item k at nz index m is w_m = w0 + m dw (w0 = (q + i k0.mu)
// e0, dw = i (2 pi b3.mu) e0, e0 the item's base phase): six scalar FMAs per
// (atom, k), the minimum for a complex multiply-accumulate with a linearly
// advancing amplitude.  When the second item is the next chunk of the same
// column its base phase is the first one's times e^{2 pi i 16 s_z} (tabulated
// per atom) instead of a second sin/cos.  FP32 sums over a tile of atoms go to
// FP32 block sums in shared memory (a two-level tree) and are written as FP64
// partials.
constexpr int SF32_TILE = 32;
template <int WITH_MU>
__global__ void __launch_bounds__(SF_THREADS) k_sfac32(int n, int natom_chunk, const uint32_t* __restrict__ fx,
                                                         const float2* __restrict__ tab, const double* __restrict__ q,
                                                         const double* __restrict__ mu, CellP c, int ky, int kz,
                                                         int ncol, int nchunk, int with_q, const int* __restrict__ items,
                                                         int nitems, double* __restrict__ part_re,
                                                         double* __restrict__ part_im) {
    __shared__ uint4 t_a[SF32_TILE];                 // u1, u2, u3, q (float bits)
    __shared__ float4 t_m[SF32_TILE];                // 2 pi b_d . mu (d = 1..3), unused
    __shared__ float2 t_16[SF32_TILE];               // e^{2 pi i 16 s_z}
    __shared__ float4 t_T[SF32_TILE][TM / 2];        // (T_m, T_m+1)
    __shared__ float s_acc[4 * TM][SF_THREADS];     // second-level sums: [item][re/im][m] x thread
    const int t0 = 2 * (blockIdx.x * SF_THREADS + threadIdx.x);
    const int p = blockIdx.y;
    const int ny_n = 2 * ky + 1;
    int inx[2], iny[2], inz0[2];
#pragma unroll
    for (int it = 0; it < 2; ++it) {
        const int kc = min(t0 + it, nitems - 1);
        const int cl = items[2 * kc];
        inx[it] = cl / ny_n;
        iny[it] = cl % ny_n - ky;
        inz0[it] = -kz + items[2 * kc + 1] * TM;
    }
    // the second item continues the first one's column: rotate instead of sin/cos
    const bool chain = inx[1] == inx[0] && iny[1] == iny[0] && inz0[1] == inz0[0] + TM;
#pragma unroll
    for (int k = 0; k < 4 * TM; ++k) s_acc[k][threadIdx.x] = 0.f;
    const int a0 = p * natom_chunk;
    const int a1 = min(n, a0 + natom_chunk);
    for (int base = a0; base < a1; base += SF32_TILE) {
        __syncthreads();
        const int tn = min(SF32_TILE, a1 - base);
        for (int t = threadIdx.x; t < tn * (TM / 2); t += blockDim.x) {
            const int a = t / (TM / 2), m2 = t % (TM / 2);
            const float2* src = tab + (size_t)(base + a) * TM + 2 * m2;
            const float2 A = src[0], B = src[1];
            t_T[a][m2] = make_float4(A.x, A.y, B.x, B.y);
        }
        if (threadIdx.x < tn) {
            const int ia = base + threadIdx.x;
            const float qa = with_q ? (float)q[ia] : 0.f;
            const uint32_t u3 = fx[2 * n + ia];
            t_a[threadIdx.x] = make_uint4(fx[ia], fx[n + ia], u3, __float_as_uint(qa));
            double m0 = 0, m1 = 0, m2 = 0;
            if (WITH_MU) { m0 = mu[ia]; m1 = mu[n + ia]; m2 = mu[2 * n + ia]; }
            t_m[threadIdx.x] = make_float4((float)(2.0 * PI * (c.B[0] * m0 + c.B[3] * m1 + c.B[6] * m2)),
                                           (float)(2.0 * PI * (c.B[1] * m0 + c.B[4] * m1 + c.B[7] * m2)),
                                           (float)(2.0 * PI * (c.B[2] * m0 + c.B[5] * m1 + c.B[8] * m2)), 0.f);
            float c16, s16;
            phase32(u3 * 16u, c16, s16);
            t_16[threadIdx.x] = make_float2(c16, s16);
        }
        __syncthreads();
        float ar0[TM], ai0[TM], ar1[TM], ai1[TM];
#pragma unroll
        for (int m = 0; m < TM; ++m) { ar0[m] = 0.f; ai0[m] = 0.f; ar1[m] = 0.f; ai1[m] = 0.f; }
        for (int a = 0; a < tn; ++a) {
            const uint4 A = t_a[a];
            const float qa = __uint_as_float(A.w);
            float c0[2], s0[2];
            phase32((uint32_t)inx[0] * A.x + (uint32_t)iny[0] * A.y + (uint32_t)inz0[0] * A.z, c0[0], s0[0]);
            if (chain) {
                const float2 e16 = t_16[a];
                c0[1] = fmaf(c0[0], e16.x, -s0[0] * e16.y);
                s0[1] = fmaf(s0[0], e16.x, c0[0] * e16.y);
            } else {
                phase32((uint32_t)inx[1] * A.x + (uint32_t)iny[1] * A.y + (uint32_t)inz0[1] * A.z, c0[1], s0[1]);
            }
            float w0r[2], w0i[2], dwr[2] = {0.f, 0.f}, dwi[2] = {0.f, 0.f};
            const float4 M = t_m[a];
#pragma unroll
            for (int it = 0; it < 2; ++it) {
                if (WITH_MU) {
                    const float km = fmaf((float)inx[it], M.x, fmaf((float)iny[it], M.y, (float)inz0[it] * M.z));
                    w0r[it] = fmaf(qa, c0[it], -km * s0[it]);
                    w0i[it] = fmaf(qa, s0[it], km * c0[it]);
                    dwr[it] = -M.z * s0[it];
                    dwi[it] = M.z * c0[it];
                } else {
                    w0r[it] = qa * c0[it];
                    w0i[it] = qa * s0[it];
                }
            }
#pragma unroll
            for (int m2 = 0; m2 < TM / 2; ++m2) {
                const float4 TT = t_T[a][m2];
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const int m = 2 * m2 + j;
                    const float tx = j ? TT.z : TT.x, ty = j ? TT.w : TT.y;
                    const float wr0 = WITH_MU ? fmaf((float)m, dwr[0], w0r[0]) : w0r[0];
                    const float wi0 = WITH_MU ? fmaf((float)m, dwi[0], w0i[0]) : w0i[0];
                    const float wr1 = WITH_MU ? fmaf((float)m, dwr[1], w0r[1]) : w0r[1];
                    const float wi1 = WITH_MU ? fmaf((float)m, dwi[1], w0i[1]) : w0i[1];
                    ar0[m] = fmaf(wr0, tx, fmaf(-wi0, ty, ar0[m]));
                    ai0[m] = fmaf(wr0, ty, fmaf(wi0, tx, ai0[m]));
                    ar1[m] = fmaf(wr1, tx, fmaf(-wi1, ty, ar1[m]));
                    ai1[m] = fmaf(wr1, ty, fmaf(wi1, tx, ai1[m]));
                }
            }
        }
#pragma unroll
        for (int m = 0; m < TM; ++m) {
            s_acc[2 * m][threadIdx.x] += ar0[m];
            s_acc[2 * m + 1][threadIdx.x] += ai0[m];
            s_acc[2 * TM + 2 * m][threadIdx.x] += ar1[m];
            s_acc[2 * TM + 2 * m + 1][threadIdx.x] += ai1[m];
        }
    }
    const size_t plane = (size_t)ncol * TM * nchunk;
#pragma unroll
    for (int it = 0; it < 2; ++it) {
        const int k = t0 + it;
        if (k >= nitems) continue;
        const int cl = items[2 * k], hh = items[2 * k + 1];
#pragma unroll
        for (int m = 0; m < TM; ++m) {
            const size_t idx = (size_t)p * plane + ((size_t)hh * TM + m) * ncol + cl;
            part_re[idx] = (double)s_acc[2 * TM * it + 2 * m][threadIdx.x];
            part_im[idx] = (double)s_acc[2 * TM * it + 2 * m + 1][threadIdx.x];
        }
    }
}

// Pass 2: thread = atom.  Per chunk of TM k-vectors along nz, with
// P_m = conj(a_m) T_m (a_m = A_k S(k), T_m = e^{2 pi i m s_z}):
//   Z0 = sum_m P_m,  Z1 = sum_m m P_m  (and Z2 = sum_m m^2 P_m for the gradient),
// then with the chunk's base phase e0 and k_m = kb + m dk:
//   sum_m k_m recarg_m = -(kb Im(e0 Z0) + dk Im(e0 Z1)),
//   sum_m k_m k_m^T recarg2_m = kb kb^T Re(e0 Z0) + (kb dk^T + dk kb^T) Re(e0 Z1) + dk dk^T Re(e0 Z2).
// The inner loop is packed FP32 (f32x2): P_m = a_re (T) + a_im (T_im, -T_re)
// from a 16-byte shared-memory load of (a_re, a_re, a_im, a_im), and the
// m-weighted sums come from running suffix sums over m descending
// (R = sum_{m>=j} P_m, Q = sum R, W = sum Q: Z1 = Q, Z2 = 2W - Q), so no
// per-m constants are needed.  Each column's FP32 sum is flushed to FP64.
template <int GRAD>
__global__ void __launch_bounds__(KF_THREADS) k_kfield32v5(int n, const uint32_t* __restrict__ fx,
                                                           const float2* __restrict__ tab, CellP c, int kx, int ky,
                                                           int kz, int ncol, int nzp, int cols_per_split,
                                                           const float4* __restrict__ aks, const int* __restrict__ colrange,
                                                           double* __restrict__ fpart) {
    extern __shared__ float4 ska4[];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int split = blockIdx.y;
    const int c0 = split * cols_per_split;
    const int c1 = min(ncol, c0 + cols_per_split);
    const bool active = i < n;
    const int ii = active ? i : 0;
    const uint32_t u1 = fx[ii], u2 = fx[n + ii], u3 = fx[2 * n + ii];
    f2p T[TM], Tn[TM];
#pragma unroll
    for (int m = 0; m < TM; ++m) {
        const float2 t = tab[(size_t)ii * TM + m];
        T[m] = pk2(t.x, t.y);
        Tn[m] = pk2(t.y, -t.x);
    }
    float e16c, e16s;
    phase32(u3 * 16u, e16c, e16s);
    const float b1x = (float)(2.0 * PI * c.B[0]), b1y = (float)(2.0 * PI * c.B[3]), b1z = (float)(2.0 * PI * c.B[6]);
    const float b2x = (float)(2.0 * PI * c.B[1]), b2y = (float)(2.0 * PI * c.B[4]), b2z = (float)(2.0 * PI * c.B[7]);
    const float dk0 = (float)(2.0 * PI * c.B[2]), dk1 = (float)(2.0 * PI * c.B[5]), dk2 = (float)(2.0 * PI * c.B[8]);
    const int ny_n = 2 * ky + 1;
    double E0 = 0, E1 = 0, E2 = 0;
    double G0 = 0, G1 = 0, G2 = 0, G3 = 0, G4 = 0, G5 = 0;
    for (int cb = c0; cb < c1; cb += KF_COLS32) {
        const int nc = min(KF_COLS32, c1 - cb);
        __syncthreads();
        for (int t = threadIdx.x; t < nc * nzp; t += blockDim.x) ska4[t] = aks[(size_t)cb * nzp + t];
        __syncthreads();
        for (int cc = 0; cc < nc; ++cc) {
            const int col = cb + cc;
            int clo = 0, cn = nzp / TM;
            if (colrange) { clo = colrange[2 * col]; cn = colrange[2 * col + 1]; }
            if (cn == 0) continue;
            const int inx = col / ny_n, iny = col % ny_n - ky;
            const int nzb = -kz + TM * clo;
            const uint32_t ph = (uint32_t)inx * u1 + (uint32_t)iny * u2 + (uint32_t)nzb * u3;
            float ec, es;
            phase32(ph, ec, es);
            const float fnx = (float)inx, fny = (float)iny, fnz = (float)nzb;
            float kb0 = fmaf(fnx, b1x, fmaf(fny, b2x, fnz * dk0));
            float kb1 = fmaf(fnx, b1y, fmaf(fny, b2y, fnz * dk1));
            float kb2 = fmaf(fnx, b1z, fmaf(fny, b2z, fnz * dk2));
            const ulonglong2* pk = reinterpret_cast<const ulonglong2*>(ska4 + cc * nzp);
            float e0 = 0.f, e1 = 0.f, e2 = 0.f;
            float g0 = 0.f, g1 = 0.f, g2 = 0.f, g3 = 0.f, g4 = 0.f, g5 = 0.f;
            for (int m0 = TM * clo; m0 < TM * (clo + cn); m0 += TM) {
                f2p R = 0ull, Q = 0ull, W = 0ull;
#pragma unroll
                for (int m = TM - 1; m >= 1; --m) {
                    const ulonglong2 a = pk[m0 + m];
                    const f2p P = ffma2(a.x, T[m], fmul2(a.y, Tn[m]));
                    R = fadd2(R, P);
                    Q = fadd2(Q, R);
                    if (GRAD) W = fadd2(W, Q);
                }
                {
                    const ulonglong2 a = pk[m0];
                    R = fadd2(R, ffma2(a.x, T[0], fmul2(a.y, Tn[0])));
                }
                float z0r, z0i, z1r, z1i;
                upk2(R, z0r, z0i);
                upk2(Q, z1r, z1i);
                const float p0r = fmaf(ec, z0r, -es * z0i), p0i = fmaf(ec, z0i, es * z0r);
                const float p1r = fmaf(ec, z1r, -es * z1i), p1i = fmaf(ec, z1i, es * z1r);
                e0 = fmaf(kb0, p0i, fmaf(dk0, p1i, e0));
                e1 = fmaf(kb1, p0i, fmaf(dk1, p1i, e1));
                e2 = fmaf(kb2, p0i, fmaf(dk2, p1i, e2));
                if (GRAD) {
                    float wr, wi;
                    upk2(W, wr, wi);
                    const float z2r = 2.f * wr - z1r, z2i = 2.f * wi - z1i;
                    const float p2r = fmaf(ec, z2r, -es * z2i);
                    g0 += kb0 * kb0 * p0r + 2.f * kb0 * dk0 * p1r + dk0 * dk0 * p2r;
                    g1 += kb1 * kb1 * p0r + 2.f * kb1 * dk1 * p1r + dk1 * dk1 * p2r;
                    g2 += kb2 * kb2 * p0r + 2.f * kb2 * dk2 * p1r + dk2 * dk2 * p2r;
                    g3 += kb0 * kb1 * p0r + (kb0 * dk1 + dk0 * kb1) * p1r + dk0 * dk1 * p2r;
                    g4 += kb0 * kb2 * p0r + (kb0 * dk2 + dk0 * kb2) * p1r + dk0 * dk2 * p2r;
                    g5 += kb1 * kb2 * p0r + (kb1 * dk2 + dk1 * kb2) * p1r + dk1 * dk2 * p2r;
                }
                const float nc_ = fmaf(ec, e16c, -es * e16s);
                es = fmaf(es, e16c, ec * e16s);
                ec = nc_;
                kb0 = fmaf(16.f, dk0, kb0);
                kb1 = fmaf(16.f, dk1, kb1);
                kb2 = fmaf(16.f, dk2, kb2);
            }
            E0 += (double)e0; E1 += (double)e1; E2 += (double)e2;
            if (GRAD) {
                G0 += (double)g0; G1 += (double)g1; G2 += (double)g2;
                G3 += (double)g3; G4 += (double)g4; G5 += (double)g5;
            }
        }
    }
    if (active) {
        const int nv = GRAD ? 9 : 3;
        double* o = fpart + (size_t)split * nv * n;
        o[i] = E0; o[n + i] = E1; o[2 * n + i] = E2;
        if (GRAD) {
            o[3 * n + i] = G0; o[4 * n + i] = G1; o[5 * n + i] = G2;
            o[6 * n + i] = G3; o[7 * n + i] = G4; o[8 * n + i] = G5;
        }
    }
}

// ---- FP64 low-|k| set of the mixed path ------------------------------------
// The error of an FP32 reciprocal sum is weighted by A_k |k|, which peaks at
// |k| ~ alpha; the short list of k-vectors with |k| < ksplit (about 5 % of the
// half space at ksplit = 3.4 alpha) is therefore summed in FP64 and removed
// from the FP32 set.  The list is stored as columns (nx, ny) with a
// contiguous nz range [nzlo, nzlo + nzn).

constexpr int LK_SPLIT = 4;   // column splits of the low-|k| field pass

// Pass 1 over the low set: thread = (list column, chunk of TM nz).  Same
// scheme as the FP32 pass (exact fixed-point base phase, per-atom table T_m),
// in FP64.
constexpr int LK_TILE = 32;
__global__ void __launch_bounds__(SF_THREADS) k_sfac64_low(int n, int natom_chunk, const uint32_t* __restrict__ fx,
                                                           const double2* __restrict__ tab, const double* __restrict__ q,
                                                           const double* __restrict__ mu, CellP c,
                                                           const int* __restrict__ cols, int ncol, int nzmax, int nchunk,
                                                           int with_q, int with_mu, double* __restrict__ part_re,
                                                           double* __restrict__ part_im) {
    __shared__ uint32_t t_u1[LK_TILE], t_u2[LK_TILE], t_u3[LK_TILE];
    __shared__ double t_q[LK_TILE], t_m1[LK_TILE], t_m2[LK_TILE], t_m3[LK_TILE];
    __shared__ double2 t_T[LK_TILE][TM];
    const int h = blockIdx.x % nchunk;
    const int cidx = (blockIdx.x / nchunk) * SF_THREADS + threadIdx.x;
    const int p = blockIdx.y;
    const int cc = cidx < ncol ? cidx : ncol - 1;
    const int inx = cols[4 * cc], iny = cols[4 * cc + 1], inz0 = cols[4 * cc + 2] + h * TM;
    const double fnx = inx, fny = iny, fnz0 = inz0;
    double are[TM], aim[TM];
#pragma unroll
    for (int m = 0; m < TM; ++m) { are[m] = 0.0; aim[m] = 0.0; }
    const int a0 = p * natom_chunk;
    const int a1 = min(n, a0 + natom_chunk);
    for (int base = a0; base < a1; base += LK_TILE) {
        __syncthreads();
        for (int t = threadIdx.x; t < LK_TILE * TM; t += blockDim.x) {
            int ia = base + t / TM;
            if (ia < a1) t_T[t / TM][t % TM] = tab[(size_t)ia * TM + (t % TM)];
        }
        if (threadIdx.x < LK_TILE) {
            int ia = base + threadIdx.x;
            if (ia < a1) {
                t_u1[threadIdx.x] = fx[ia];
                t_u2[threadIdx.x] = fx[n + ia];
                t_u3[threadIdx.x] = fx[2 * n + ia];
                t_q[threadIdx.x] = with_q ? q[ia] : 0.0;
                double m0 = 0, m1 = 0, m2 = 0;
                if (with_mu) { m0 = mu[ia]; m1 = mu[n + ia]; m2 = mu[2 * n + ia]; }
                t_m1[threadIdx.x] = 2.0 * PI * (c.B[0] * m0 + c.B[3] * m1 + c.B[6] * m2);
                t_m2[threadIdx.x] = 2.0 * PI * (c.B[1] * m0 + c.B[4] * m1 + c.B[7] * m2);
                t_m3[threadIdx.x] = 2.0 * PI * (c.B[2] * m0 + c.B[5] * m1 + c.B[8] * m2);
            }
        }
        __syncthreads();
        const int tn = min(LK_TILE, a1 - base);
        for (int t = 0; t < tn; ++t) {
            const uint32_t ph = (uint32_t)inx * t_u1[t] + (uint32_t)iny * t_u2[t] + (uint32_t)inz0 * t_u3[t];
            double s0, c0;
            sincospi((double)(int)ph * 4.656612873077393e-10, &s0, &c0);   // 2 pi t, t = ph / 2^32
            const double qa = t_q[t];
            const double km = fma(fnx, t_m1[t], fma(fny, t_m2[t], fnz0 * t_m3[t]));
            const double m3 = t_m3[t];
            const double w0r = fma(qa, c0, -km * s0), w0i = fma(qa, s0, km * c0);
            const double dwr = -m3 * s0, dwi = m3 * c0;
#pragma unroll
            for (int m = 0; m < TM; ++m) {
                const double wr = fma((double)m, dwr, w0r), wi = fma((double)m, dwi, w0i);
                const double2 T = t_T[t][m];
                are[m] = fma(wr, T.x, fma(-wi, T.y, are[m]));
                aim[m] = fma(wr, T.y, fma(wi, T.x, aim[m]));
            }
        }
    }
    if (cidx < ncol) {
        const size_t plane = (size_t)nzmax * ncol;
#pragma unroll
        for (int m = 0; m < TM; ++m) {
            int mz = h * TM + m;
            if (mz < nzmax) {
                size_t idx = (size_t)p * plane + (size_t)mz * ncol + cidx;
                part_re[idx] = are[m];
                part_im[idx] = aim[m];
            }
        }
    }
}

// One warp per low-set k-vector: sum of the atom-chunk partials, A_k S(k),
// energy and stress terms.
__global__ void k_sfac64_low_reduce(int P, int ncol, int nzmax, const int* __restrict__ cols,
                                    const double* __restrict__ part_re, const double* __restrict__ part_im,
                                    const double* __restrict__ Ak, const double* __restrict__ kcoe, CellP c,
                                    double* __restrict__ aks, int energy, double* partials) {
    const int lane = threadIdx.x & 31;
    const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    const bool valid = t < ncol * nzmax;
    const int cidx = valid ? t % ncol : 0, mz = valid ? t / ncol : 0;
    const size_t plane = (size_t)nzmax * ncol;
    double sr = 0.0, si = 0.0;
    if (valid)
        for (int p = lane; p < P; p += 32) {
            sr += part_re[(size_t)p * plane + (size_t)mz * ncol + cidx];
            si += part_im[(size_t)p * plane + (size_t)mz * ncol + cidx];
        }
    sr = warp_sum(sr);
    si = warp_sum(si);
    if (valid && lane == 0) {
        const size_t r = (size_t)cidx * nzmax + mz;
        const double ak = (mz < cols[4 * cidx + 3]) ? Ak[r] : 0.0;
        aks[r] = ak * sr;
        aks[(size_t)ncol * nzmax + r] = ak * si;
        if (energy && ak != 0.0) {
            const double nx = cols[4 * cidx], ny = cols[4 * cidx + 1], nz = cols[4 * cidx + 2] + mz;
            const double k0 = 2.0 * PI * (nx * c.B[0] + ny * c.B[1] + nz * c.B[2]);
            const double k1 = 2.0 * PI * (nx * c.B[3] + ny * c.B[4] + nz * c.B[5]);
            const double k2 = 2.0 * PI * (nx * c.B[6] + ny * c.B[7] + nz * c.B[8]);
            const double str = (sr * sr + si * si) * ak;
            const double kc = kcoe[r];
            v[0] = str;
            v[1] = (1.0 - kc * k0 * k0) * str;
            v[2] = (1.0 - kc * k1 * k1) * str;
            v[3] = (1.0 - kc * k2 * k2) * str;
            v[4] = -kc * k0 * k1 * str;
            v[5] = -kc * k0 * k2 * str;
            v[6] = -kc * k1 * k2 * str;
        }
    }
    if (energy) block_partials<7>(v, partials);
}

// Pass 2 over the low set: thread = atom, blockIdx.y = range of list columns.
// Along a column the phase advances by the per-atom FP64 step e^{2 pi i s_z};
// the k-vector is applied once per column through the moments
// R0 = sum r_m, R1 = sum m r_m (Q0..Q2 for the field gradient).
template <int GRAD>
__global__ void __launch_bounds__(KF_THREADS) k_kfield64_low(int n, const uint32_t* __restrict__ fx,
                                                             const double2* __restrict__ tab, CellP c,
                                                             const int* __restrict__ cols, int ncol, int nzmax,
                                                             const double* __restrict__ aks, double* __restrict__ fpart) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int per = (ncol + gridDim.y - 1) / gridDim.y;
    const int cbeg = blockIdx.y * per, cend = min(ncol, cbeg + per);
    fpart += (size_t)blockIdx.y * 9 * n;
    const bool active = i < n;
    const int ii = active ? i : 0;
    const uint32_t u1 = fx[ii], u2 = fx[n + ii], u3 = fx[2 * n + ii];
    const double2 st = tab[(size_t)ii * TM + 1];   // e^{2 pi i s_z}
    const double rc = st.x, rs = st.y;
    const double dk0 = 2.0 * PI * c.B[2], dk1 = 2.0 * PI * c.B[5], dk2 = 2.0 * PI * c.B[8];
    double E0 = 0, E1 = 0, E2 = 0, G0 = 0, G1 = 0, G2 = 0, G3 = 0, G4 = 0, G5 = 0;
    const double* aim_base = aks + (size_t)ncol * nzmax;
    for (int cc = cbeg; cc < cend; ++cc) {
        const int inx = cols[4 * cc], iny = cols[4 * cc + 1], inz0 = cols[4 * cc + 2];
        const int nzn = cols[4 * cc + 3];
        const uint32_t ph = (uint32_t)inx * u1 + (uint32_t)iny * u2 + (uint32_t)inz0 * u3;
        double sn, cs;
        sincospi((double)(int)ph * 4.656612873077393e-10, &sn, &cs);
        const double kb0 = 2.0 * PI * (inx * c.B[0] + iny * c.B[1] + inz0 * c.B[2]);
        const double kb1 = 2.0 * PI * (inx * c.B[3] + iny * c.B[4] + inz0 * c.B[5]);
        const double kb2 = 2.0 * PI * (inx * c.B[6] + iny * c.B[7] + inz0 * c.B[8]);
        const double* pr = aks + (size_t)cc * nzmax;
        const double* pi = aim_base + (size_t)cc * nzmax;
        double R0 = 0, R1 = 0, Q0 = 0, Q1 = 0, Q2 = 0;
        for (int m = 0; m < nzn; ++m) {
            const double ar = __ldg(pr + m), ai = __ldg(pi + m);
            const double r = ai * cs - ar * sn;
            R0 += r;
            R1 = fma((double)m, r, R1);
            if (GRAD) {
                const double r2 = ar * cs + ai * sn;
                Q0 += r2;
                Q1 = fma((double)m, r2, Q1);
                Q2 = fma((double)(m * m), r2, Q2);
            }
            const double cn = cs * rc - sn * rs;
            sn = fma(sn, rc, cs * rs);
            cs = cn;
        }
        E0 -= fma(kb0, R0, dk0 * R1);
        E1 -= fma(kb1, R0, dk1 * R1);
        E2 -= fma(kb2, R0, dk2 * R1);
        if (GRAD) {
            G0 += kb0 * kb0 * Q0 + 2.0 * kb0 * dk0 * Q1 + dk0 * dk0 * Q2;
            G1 += kb1 * kb1 * Q0 + 2.0 * kb1 * dk1 * Q1 + dk1 * dk1 * Q2;
            G2 += kb2 * kb2 * Q0 + 2.0 * kb2 * dk2 * Q1 + dk2 * dk2 * Q2;
            G3 += kb0 * kb1 * Q0 + (kb0 * dk1 + dk0 * kb1) * Q1 + dk0 * dk1 * Q2;
            G4 += kb0 * kb2 * Q0 + (kb0 * dk2 + dk0 * kb2) * Q1 + dk0 * dk2 * Q2;
            G5 += kb1 * kb2 * Q0 + (kb1 * dk2 + dk1 * kb2) * Q1 + dk1 * dk2 * Q2;
        }
    }
    if (active) {
        fpart[i] = E0; fpart[n + i] = E1; fpart[2 * n + i] = E2;
        if (GRAD) {
            fpart[3 * n + i] = G0; fpart[4 * n + i] = G1; fpart[5 * n + i] = G2;
            fpart[6 * n + i] = G3; fpart[7 * n + i] = G4; fpart[8 * n + i] = G5;
        }
    }
}

struct RecLaunch {
    int CH, nchunk, ncolblk, P, natom_chunk, nsplit, cols_per_split;
};

// ---- reuse of the solver's structure factors ------------------------------
// The structure factor is linear in the sources: with the PCG iterate
// x = x0 + sum_k a_k d_k, S(q + x) = S(q + x0) + sum_k a_k S(d_k).  The
// solver accumulates A_k S over its own evaluations (k_aks_axpy), so the
// final force evaluation needs no structure-factor pass.

// acc = src (copy), or acc += a src with a = rz / dAd, the step of the
// current PCG iteration (read before the iteration's last kernel advances rz).
__global__ void k_aks_axpy(int m, const DevScalars* __restrict__ sc, int copy, const double* __restrict__ src,
                           double* __restrict__ acc) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    if (copy) acc[t] = src[t];
    else acc[t] = fma(sc->rz / sc->dAd, src[t], acc[t]);
}

// Energy and stress sums (as k_sfac_reduce) of a given A_k S(k) set of the
// rectangle: A |S|^2 = |A S|^2 / A.
__global__ void k_aks_energy(int ncol, int nzl, int ky, int kz, const double* __restrict__ aks, int nrect,
                             const double* __restrict__ Ak, const double* __restrict__ kcoe, CellP c,
                             double* partials) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    if (r < ncol * nzl) {
        const double ak = Ak[r];
        if (ak != 0.0) {
            const int col = r / nzl, mz = r % nzl;
            const int ny_n = 2 * ky + 1;
            const double nx = (double)(col / ny_n), ny = (double)(col % ny_n - ky), nz = (double)(mz - kz);
            const double k0 = 2.0 * PI * (nx * c.B[0] + ny * c.B[1] + nz * c.B[2]);
            const double k1 = 2.0 * PI * (nx * c.B[3] + ny * c.B[4] + nz * c.B[5]);
            const double k2 = 2.0 * PI * (nx * c.B[6] + ny * c.B[7] + nz * c.B[8]);
            const double ar = aks[r], ai = aks[nrect + r];
            const double str = (ar * ar + ai * ai) / ak;
            const double kc = kcoe[r];
            v[0] = str;
            v[1] = (1.0 - kc * k0 * k0) * str;
            v[2] = (1.0 - kc * k1 * k1) * str;
            v[3] = (1.0 - kc * k2 * k2) * str;
            v[4] = -kc * k0 * k1 * str;
            v[5] = -kc * k0 * k2 * str;
            v[6] = -kc * k1 * k2 * str;
        }
    }
    block_partials<7>(v, partials);
}

// The same over the FP64 low-|k| list.
__global__ void k_aks_energy_low(int ncol, int nzmax, const int* __restrict__ cols, const double* __restrict__ aks,
                                 const double* __restrict__ Ak, const double* __restrict__ kcoe, CellP c,
                                 double* partials) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    if (r < ncol * nzmax) {
        const int cidx = r / nzmax, mz = r % nzmax;
        const double ak = (mz < cols[4 * cidx + 3]) ? Ak[r] : 0.0;
        if (ak != 0.0) {
            const double nx = cols[4 * cidx], ny = cols[4 * cidx + 1], nz = cols[4 * cidx + 2] + mz;
            const double k0 = 2.0 * PI * (nx * c.B[0] + ny * c.B[1] + nz * c.B[2]);
            const double k1 = 2.0 * PI * (nx * c.B[3] + ny * c.B[4] + nz * c.B[5]);
            const double k2 = 2.0 * PI * (nx * c.B[6] + ny * c.B[7] + nz * c.B[8]);
            const double ar = aks[r], ai = aks[(size_t)ncol * nzmax + r];
            const double str = (ar * ar + ai * ai) / ak;
            const double kc = kcoe[r];
            v[0] = str;
            v[1] = (1.0 - kc * k0 * k0) * str;
            v[2] = (1.0 - kc * k1 * k1) * str;
            v[3] = (1.0 - kc * k2 * k2) * str;
            v[4] = -kc * k0 * k1 * str;
            v[5] = -kc * k0 * k2 * str;
            v[6] = -kc * k1 * k2 * str;
        }
    }
    block_partials<7>(v, partials);
}

// Snapshot (copy != 0) or PCG-step accumulation of the current A_k S sets
// (rectangle and, on the mixed path, the low-|k| list) into the solver's
// accumulators.
void launch_aks_accumulate(cudaStream_t st, const KGrid& kg, RecScratch& rs, const DevScalars* d, int copy) {
    const int m = 2 * kg.nrect;
    k_aks_axpy<<<(m + 255) / 256, 256, 0, st>>>(m, d, copy, rs.aks, rs.aks_acc);
    if (rs.low.ncol > 0 && rs.low.aks_acc) {
        const int ml = 2 * rs.low.ncol * rs.low.nzmax;
        k_aks_axpy<<<(ml + 255) / 256, 256, 0, st>>>(ml, d, copy, rs.low.aks, rs.low.aks_acc);
    }
}

static RecLaunch plan(int n, const KGrid& kg) {
    RecLaunch L;
    L.CH = 16;
    if (kg.nzl <= 8) L.CH = 8;
    else if (kg.nzl <= 12) L.CH = 12;
    L.nchunk = (kg.nzl + L.CH - 1) / L.CH;
    L.ncolblk = (kg.ncol + SF_THREADS - 1) / SF_THREADS;
    // the FP64 sphere: one thread per work-list item, columns of the list
    long threads1 = kg.nfitems > 0 ? (long)((kg.nfitems + SF_THREADS - 1) / SF_THREADS) * SF_THREADS
                                   : (long)L.nchunk * L.ncolblk * SF_THREADS;
    const int ncl = kg.nfcol > 0 ? kg.nfcol : kg.ncol;
    long want = 148L * 1536;
    int P = (int)((want + threads1 - 1) / threads1);
    P = std::max(1, std::min(P, (n + 63) / 64));
    L.natom_chunk = (n + P - 1) / P;
    L.P = (n + L.natom_chunk - 1) / L.natom_chunk;
    long threads2 = (long)((n + KF_THREADS - 1) / KF_THREADS) * KF_THREADS;
    int S = (int)((want + threads2 - 1) / threads2);
    S = std::max(1, std::min(S, ncl));
    L.cols_per_split = (ncl + S - 1) / S;
    L.nsplit = (ncl + L.cols_per_split - 1) / L.cols_per_split;
    return L;
}

// Launch shape of the mixed path's FP32 passes: the atom split of the
// structure factor sized for its (column, chunk) work list and the column
// split of the field, each scaled by mul/2 (mul = 1, 2 or 4; chosen by the
// autotuner, 2 by default).
static RecLaunch plan_mixed(int n, const KGrid& kg, int p_mul, int s_mul) {
    RecLaunch L = plan(n, kg);
    const long want = 148L * 1536;
    const int nitems = kg.nitems > 0 ? kg.nitems : kg.ncol * ((kg.nzl + TM - 1) / TM);
    const int nthr = (nitems + 1) / 2;   // two work items per thread
    const long threads1 = (long)((nthr + SF_THREADS - 1) / SF_THREADS) * SF_THREADS;
    int P = (int)((want + threads1 - 1) / threads1);
    P = std::max(1, std::min(P * p_mul / 2, (n + 31) / 32));
    L.natom_chunk = (n + P - 1) / P;
    L.P = (n + L.natom_chunk - 1) / L.natom_chunk;
    const long threads2 = (long)((n + KF_THREADS - 1) / KF_THREADS) * KF_THREADS;
    int S = (int)((want + threads2 - 1) / threads2);
    S = std::max(1, std::min(S * s_mul / 2, kg.ncol));
    L.cols_per_split = (kg.ncol + S - 1) / S;
    L.nsplit = (kg.ncol + L.cols_per_split - 1) / L.cols_per_split;
    return L;
}

// Scratch for every launch shape the path may use (on the mixed path up to
// the autotuner's largest splits).
size_t rec_scratch_doubles(int n, const KGrid& kg, size_t* fpart, int mixed) {
    RecLaunch L = plan(n, kg);
    size_t rows = std::max((size_t)L.nchunk * L.CH, (size_t)((kg.nzl + TM - 1) / TM) * TM);
    size_t part = (size_t)L.P * rows * kg.ncol * 2;
    *fpart = (size_t)L.nsplit * 9 * n;
    if (mixed) {
        RecLaunch M = plan_mixed(n, kg, 4, 4);
        part = std::max(part, (size_t)M.P * rows * kg.ncol * 2);
        *fpart = std::max(*fpart, (size_t)M.nsplit * 9 * n);
    }
    return part;
}

// The mixed path's fixed-point coordinates and phase tables for the current
// positions (built once per position update).
// (plus, with the tensor-core structure factor, its X/Y tables and B digit
// images); returns the number of kernels launched.
int ensure_phase_tables(cudaStream_t st, int n, const double* sx, const double* sy, const double* sz, RecScratch& rs) {
    if (rs.tab_epoch == rs.want_epoch) return 0;
    const LowK& lk = rs.low;
    k_phase_table<<<(n + 127) / 128, 128, 0, st>>>(n, sx, sy, sz, rs.fixed, rs.tab,
                                                   lk.ncol > 0 && !lk.tc ? lk.tab : nullptr);
    rs.tab_epoch = rs.want_epoch;
    int nk = 1;
    if (rs.tc.on) {
        const TcK& t = rs.tc;
        const long nxy = (long)t.npad * t.XYW, nb = (long)t.npad * (t.N / 2);
        tcs::k_tc_xy<<<(unsigned)((nxy + 255) / 256), 256, 0, st>>>(n, t.npad, rs.fixed, t.kx, t.ky, t.XYW, t.xy);
        tcs::k_tc_bimage<<<(unsigned)((nb + 255) / 256), 256, 0, st>>>(n, t.npad, rs.fixed, t.kz, t.nzl, t.N, t.bimg);
        const long na = (long)t.ntile_f * 128 * (t.KZ / 16), nt = (long)t.ntile_f * 128 * t.XYW;
        tcf::k_tcf_aimage<<<(unsigned)((na + 255) / 256), 256, 0, st>>>(n, t.ntile_f, rs.fixed, t.kz, t.nzl, t.KZ,
                                                                       t.aimg);
        tcf::k_tcf_xyt<<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(t.npad, t.ntile_f, t.xy, t.XYW, t.xyt);
        nk += 4;
    }
    if (lk.tc) {
        const long nxy = (long)lk.npad * lk.XYW, nb = (long)lk.npad * (lk.N / 2);
        tc4::k_tc4_xy<<<(unsigned)((nxy + 255) / 256), 256, 0, st>>>(n, lk.npad, rs.fixed, lk.kx, lk.ky, lk.XYW, lk.xy);
        tc4::k_tc4_bimage<<<(unsigned)((nb + 255) / 256), 256, 0, st>>>(n, lk.npad, rs.fixed, lk.kz, lk.nzl, lk.N,
                                                                       lk.bimg);
        const long na = (long)lk.ntile_f * 128 * (lk.KZ / 16), nt = (long)lk.ntile_f * 128 * lk.XYW;
        tc4::k_tc4f_aimage<<<(unsigned)((na + 255) / 256), 256, 0, st>>>(n, lk.ntile_f, rs.fixed, lk.kz, lk.nzl,
                                                                        lk.KZ, lk.aimg);
        tc4::k_tc4f_xyt<<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(lk.npad, lk.ntile_f, lk.xy, lk.XYW, lk.xyt);
        nk += 4;
    }
    return nk;
}

// Field pass over the low-|k| list: the 32-bit tensor-core kernels or the
// FP64 CUDA-core kernel; returns the number of kernels launched.
int launch_low_field(cudaStream_t st, int n, CellP c, bool grad, RecScratch& rs, DevScalars* d, Prof* prof) {
    LowK& lk = rs.low;
    if (lk.tc) {
        const int nch = lk.KZ / 16;
        if (grad) {
            using C3 = tc4::Cfg<3>;
            const int ncb = (lk.ncol + C3::CB - 1) / C3::CB;
            tc4::k_tc4f_bimage<3><<<ncb, C3::NB * nch, 0, st>>>(lk.ncol, lk.col, lk.nzmax, lk.kx, lk.ky, lk.kz,
                                                                lk.nzl, lk.KZ, lk.aks, c, lk.fimg);
            prof->detail_begin(PD_TC4_FIELD);
            tc4::k_kfield_tc4<3><<<lk.ntile_f, tc4::FTHREADS, lk.smem_f3, st>>>(n, ncb, lk.aimg, lk.xyt, lk.fimg,
                                                                               lk.KZ, lk.XYW, c, lk.fpart, &d->tc_err);
            prof->detail_end(PD_TC4_FIELD, 10.0 * 2.0 * n * (6.0 * lk.ncol) * (2.0 * lk.nzl));
        } else {
            using C2 = tc4::Cfg<2>;
            const int ncb = (lk.ncol + C2::CB - 1) / C2::CB;
            tc4::k_tc4f_bimage<2><<<ncb, C2::NB * nch, 0, st>>>(lk.ncol, lk.col, lk.nzmax, lk.kx, lk.ky, lk.kz,
                                                                lk.nzl, lk.KZ, lk.aks, c, lk.fimg);
            prof->detail_begin(PD_TC4_FIELD);
            tc4::k_kfield_tc4<2><<<lk.ntile_f, tc4::FTHREADS, lk.smem_f2, st>>>(n, ncb, lk.aimg, lk.xyt, lk.fimg,
                                                                               lk.KZ, lk.XYW, c, lk.fpart, &d->tc_err);
            prof->detail_end(PD_TC4_FIELD, 10.0 * 2.0 * n * (4.0 * lk.ncol) * (2.0 * lk.nzl));
        }
        return 2;
    }
    if (grad)
        k_kfield64_low<1><<<dim3((n + KF_THREADS - 1) / KF_THREADS, LK_SPLIT), KF_THREADS, 0, st>>>(
            n, rs.fixed, lk.tab, c, lk.col, lk.ncol, lk.nzmax, lk.aks, lk.fpart);
    else
        k_kfield64_low<0><<<dim3((n + KF_THREADS - 1) / KF_THREADS, LK_SPLIT), KF_THREADS, 0, st>>>(
            n, rs.fixed, lk.tab, c, lk.col, lk.ncol, lk.nzmax, lk.aks, lk.fpart);
    return 1;
}

#define CUDA_COPY_ACC(st, dst, src, bytes) cudaMemcpyAsync((dst), (src), (bytes), cudaMemcpyDeviceToDevice, (st))

void launch_ewald_rec(cudaStream_t st, int n, const double* sx, const double* sy, const double* sz,
                      const double* q, const double* mu, CellP c, const KGrid& kg, RecFlags fl, RecScratch& rs,
                      double* ef, double* efg, double* fo, Partials& part, DevScalars* d, Prof* prof) {
    const bool mixed = fl.prec == MDFF_PREC_MIXED;
    RecLaunch L = mixed ? plan_mixed(n, kg, rs.p_mul, rs.s_mul) : plan(n, kg);
    const size_t plane = (size_t)L.P * std::max(L.nchunk * L.CH, ((kg.nzl + TM - 1) / TM) * TM) * kg.ncol;
    double* pre = rs.part;
    double* pim = rs.part + plane;
    const int kx = kg.kmax[0], ky = kg.kmax[1], kz = kg.kmax[2];
    const bool low = mixed && rs.low.ncol > 0;
    const int nchunk32 = (kg.nzl + TM - 1) / TM;
    const int total = kg.ncol * kg.nzl;
    const int rb = (total + 255) / 256;
    prof->begin(PK_SFAC);
    int nk = 2 + (fl.energy ? 1 : 0);
    if (fl.reuse) {
        // A_k S from the solver's accumulators: no structure-factor pass
        CUDA_COPY_ACC(st, rs.aks, rs.aks_acc, sizeof(double) * 2 * kg.nrect);
        nk = 0;
        if (fl.energy) {
            const double* akr = mixed ? kg.Ak_hi : kg.Ak;
            k_aks_energy<<<rb, 256, 0, st>>>(kg.ncol, kg.nzl, ky, kz, rs.aks, kg.nrect, akr, kg.kcoe, c, part.buf);
            launch_reduce_partials(st, part.buf, rb, 7, d->rec, 0);
            nk += 2;
        }
        if (low) {
            LowK& lk = rs.low;
            const int ml = lk.ncol * lk.nzmax;
            CUDA_COPY_ACC(st, lk.aks, lk.aks_acc, sizeof(double) * 2 * ml);
            if (fl.energy) {
                const int lb = (ml + 255) / 256;
                k_aks_energy_low<<<lb, 256, 0, st>>>(lk.ncol, lk.nzmax, lk.col, lk.aks, lk.Ak, lk.kcoe, c, part.buf);
                launch_reduce_partials(st, part.buf, lb, 7, d->rec, 1);
                nk += 2;
            }
        }
    } else if (mixed) {
        nk += ensure_phase_tables(st, n, sx, sy, sz, rs);
        // the FP32 set's (column, chunk) work list: the low-|k| vectors and
        // those outside the sphere are not in it (A_k = 0 there)
        dim3 g1(((kg.nitems + 1) / 2 + SF_THREADS - 1) / SF_THREADS, L.P);
        int Pr = L.P;
        if (rs.tc.on) {
            // tensor-core structure factor: one partial per atom split
            const TcK& t = rs.tc;
            const size_t tplane = (size_t)kg.ncol * nchunk32 * TM;
            pre = rs.part;
            pim = rs.part + (size_t)t.nsplit * tplane;
            tcs::k_tc_params<<<(t.npad + 255) / 256, 256, 0, st>>>(n, t.npad, q, mu, c, fl.with_q, fl.with_mu, kx, ky,
                                                                   kz, t.prm, t.amax);
            // int8 digit-product operations of the unpadded GEMM: 6 products of
            // 2 M N K, M = sphere columns, N = 2 nz rows, K = 4 per atom
            prof->detail_begin(PD_TC_SFAC);
            if (fl.with_q)
                tcs::k_sfac_tc<true><<<dim3(t.ntile, t.nsplit), tcs::THREADS, t.smem, st>>>(
                    t.nblk, t.bps, t.bimg, t.xy, t.prm, t.amax, t.cols, t.nsph, kx, ky, kz, kg.nzl, t.N, t.XYW,
                    kg.ncol, tplane, pre, pim, &d->tc_err);
            else
                tcs::k_sfac_tc<false><<<dim3(t.ntile, t.nsplit), tcs::THREADS, t.smem, st>>>(
                    t.nblk, t.bps, t.bimg, t.xy, t.prm, t.amax, t.cols, t.nsph, kx, ky, kz, kg.nzl, t.N, t.XYW,
                    kg.ncol, tplane, pre, pim, &d->tc_err);
            prof->detail_end(PD_TC_SFAC, 6.0 * 2.0 * t.nsph * (2.0 * kg.nzl) * (4.0 * n));
            Pr = t.nsplit;
            nk += 2;
        } else if (kg.nitems > 0) {
            if (fl.with_mu)
                k_sfac32<1><<<g1, SF_THREADS, 0, st>>>(n, L.natom_chunk, rs.fixed, rs.tab, q, mu, c, ky, kz, kg.ncol,
                                                         nchunk32, fl.with_q, kg.items, kg.nitems, pre, pim);
            else
                k_sfac32<0><<<g1, SF_THREADS, 0, st>>>(n, L.natom_chunk, rs.fixed, rs.tab, q, mu, c, ky, kz, kg.ncol,
                                                         nchunk32, fl.with_q, kg.items, kg.nitems, pre, pim);
        }
        k_sfac_reduce<<<rb, 256, 0, st>>>(Pr, TM, nchunk32, kg.ncol, kg.nzl, kx, ky, kz, pre, pim, kg.Ak_hi, kg.kcoe, c,
                                          rs.aks, kg.nrect, fl.energy, part.buf);
    } else {
        const bool sph = kg.nfitems > 0;
        dim3 g1(sph ? (kg.nfitems + SF_THREADS - 1) / SF_THREADS : L.nchunk * L.ncolblk, L.P);
#define SFAC(CHV) k_sfac<CHV><<<g1, SF_THREADS, 0, st>>>(n, L.natom_chunk, sx, sy, sz, q, mu, c, kx, ky, kz, kg.ncol, \
                                                     L.ncolblk, L.nchunk, fl.with_q, fl.with_mu, pre, pim, \
                                                     sph ? kg.fitems : nullptr, kg.nfitems)
        if (L.CH == 16) SFAC(16);
        else if (L.CH == 12) SFAC(12);
        else SFAC(8);
#undef SFAC
        k_sfac_reduce<<<rb, 256, 0, st>>>(L.P, L.CH, L.nchunk, kg.ncol, kg.nzl, kx, ky, kz, pre, pim, kg.Ak, kg.kcoe,
                                          c, rs.aks, kg.nrect, fl.energy, part.buf);
    }
    if (fl.energy && !fl.reuse) launch_reduce_partials(st, part.buf, rb, 7, d->rec, 0);
    if (low && !fl.reuse) {
        LowK& lk = rs.low;
        int Pl = lk.P;
        if (lk.tc) {
            // 32-bit fixed point on the tensor cores: one partial per atom split
            Pl = lk.nsplit;
            const size_t lplane = (size_t)Pl * lk.nzmax * lk.ncol;
            tc4::k_tc4_params<<<(lk.npad + 255) / 256, 256, 0, st>>>(n, lk.npad, q, mu, c, fl.with_q, fl.with_mu, lk.kx,
                                                                     lk.ky, lk.kz, lk.prm, lk.amax);
            // int8 digit-product operations of the unpadded GEMM: ten products
            // of 2 M N K, M = list columns, N = 2 nz rows, K = 4 per atom
            prof->detail_begin(PD_TC4_SFAC);
            tc4::k_sfac_tc4<<<dim3(lk.ntile, lk.nsplit), tc4::THREADS, lk.smem, st>>>(
                lk.nblk, lk.bps, lk.nin, lk.bimg, lk.xy, lk.prm, lk.amax, lk.col, lk.ncol, lk.nzmax, lk.kx, lk.ky, lk.kz, lk.N,
                lk.XYW, lk.part, lk.part + lplane, &d->tc_err);
            prof->detail_end(PD_TC4_SFAC, 10.0 * 2.0 * lk.ncol * (2.0 * lk.nzl) * (4.0 * n));
            nk += 1;
        } else {
            const int nch = (lk.nzmax + TM - 1) / TM;
            const int cb = (lk.ncol + SF_THREADS - 1) / SF_THREADS;
            dim3 gl(nch * cb, lk.P);
            const size_t lplane = (size_t)lk.P * lk.nzmax * lk.ncol;
            k_sfac64_low<<<gl, SF_THREADS, 0, st>>>(n, lk.natom_chunk, rs.fixed, lk.tab, q, mu, c, lk.col, lk.ncol,
                                                    lk.nzmax, nch, fl.with_q, fl.with_mu, lk.part, lk.part + lplane);
        }
        const size_t lplane = (size_t)Pl * lk.nzmax * lk.ncol;
        const int lb = (lk.ncol * lk.nzmax * 32 + 255) / 256;
        k_sfac64_low_reduce<<<lb, 256, 0, st>>>(Pl, lk.ncol, lk.nzmax, lk.col, lk.part, lk.part + lplane, lk.Ak,
                                                lk.kcoe, c, lk.aks, fl.energy, part.buf);
        if (fl.energy) launch_reduce_partials(st, part.buf, lb, 7, d->rec, 1);
        nk += 2 + (fl.energy ? 1 : 0);
    }
    prof->end(nk);
    if (!fl.field && !fl.grad && !fl.forces) return;
    prof->begin(PK_KFIELD);
    nk = 1;
    dim3 g2((n + KF_THREADS - 1) / KF_THREADS, L.nsplit);
    const bool grad = fl.grad || (fl.forces && fl.with_mu);
    int nsplit_f = L.nsplit;
    if (mixed && rs.tc.on) {
        // field pass on the tensor cores: NQ column parts per atom
        const TcK& t = rs.tc;
        const int nch = t.KZ / 16;
        if (grad) {
            using C3 = tcf::Cfg<3>;
            const int ncb = (t.nsph + C3::CB - 1) / C3::CB;
            tcf::k_tcf_bimage<3><<<ncb, C3::NB * nch, 0, st>>>(t.nsph, t.cols, kx, ky, kz, kg.nzl, t.KZ, rs.aks,
                                                                kg.nrect, c, t.fimg);
            prof->detail_begin(PD_TC_FIELD);
            tcf::k_kfield_tc<3><<<t.grid_f, tcf::THREADS, t.smem_f3, st>>>(n, t.ntile_f, ncb, t.aimg, t.xyt, t.fimg,
                                                                            t.KZ, t.XYW, c, rs.fpart, &d->tc_err);
            prof->detail_end(PD_TC_FIELD, 6.0 * 2.0 * n * (6.0 * t.nsph) * (2.0 * kg.nzl));
        } else {
            using C2 = tcf::Cfg<2>;
            const int ncb = (t.nsph + C2::CB - 1) / C2::CB;
            tcf::k_tcf_bimage<2><<<ncb, C2::NB * nch, 0, st>>>(t.nsph, t.cols, kx, ky, kz, kg.nzl, t.KZ, rs.aks,
                                                                kg.nrect, c, t.fimg);
            prof->detail_begin(PD_TC_FIELD);
            tcf::k_kfield_tc<2><<<t.grid_f, tcf::THREADS, t.smem_f2, st>>>(n, t.ntile_f, ncb, t.aimg, t.xyt, t.fimg,
                                                                            t.KZ, t.XYW, c, rs.fpart, &d->tc_err);
            prof->detail_end(PD_TC_FIELD, 6.0 * 2.0 * n * (4.0 * t.nsph) * (2.0 * kg.nzl));
        }
        nsplit_f = 2 * tcf::NQ;   // NQ column parts in each of the 2 column slots
        nk += 1;
        if (low) nk += launch_low_field(st, n, c, grad, rs, d, prof);
    } else if (mixed) {
        const int nzp = nchunk32 * TM;
        k_aks32_pad<<<(kg.ncol * nzp + 255) / 256, 256, 0, st>>>(kg.ncol, kg.nzl, nzp, kg.nrect, rs.aks, rs.aks2);
        const size_t sm32 = sizeof(float4) * KF_COLS32 * nzp;
        if (grad)
            k_kfield32v5<1><<<g2, KF_THREADS, sm32, st>>>(n, rs.fixed, rs.tab, c, kx, ky, kz, kg.ncol, nzp,
                                                         L.cols_per_split, rs.aks2, kg.colrange, rs.fpart);
        else
            k_kfield32v5<0><<<g2, KF_THREADS, sm32, st>>>(n, rs.fixed, rs.tab, c, kx, ky, kz, kg.ncol, nzp,
                                                         L.cols_per_split, rs.aks2, kg.colrange, rs.fpart);
        nk += 2;
        if (low) nk += launch_low_field(st, n, c, grad, rs, d, prof);
    } else {
        size_t smem = sizeof(double) * 2 * KF_COLS * kg.nzl;
        const bool sph = kg.nfcol > 0;
        const int ncl = sph ? kg.nfcol : kg.ncol;
        if (grad)
            k_kfield<1><<<g2, KF_THREADS, smem, st>>>(n, sx, sy, sz, c, kx, ky, kz, ncl, kg.nzl, L.cols_per_split,
                                                      rs.aks, kg.nrect, rs.fpart, sph ? kg.fcols : nullptr,
                                                      sph ? kg.fzr : nullptr);
        else
            k_kfield<0><<<g2, KF_THREADS, smem, st>>>(n, sx, sy, sz, c, kx, ky, kz, ncl, kg.nzl, L.cols_per_split,
                                                      rs.aks, kg.nrect, rs.fpart, sph ? kg.fcols : nullptr,
                                                      sph ? kg.fzr : nullptr);
        nk++;
    }
    const double scale = 2.0 * 4.0 * PI / c.omega;
    k_kfield_reduce<<<(n + 255) / 256, 256, 0, st>>>(n, nsplit_f, grad ? 1 : 0, rs.fpart, scale, fl.with_q ? q : nullptr,
                                                    fl.with_mu ? mu : nullptr, fl.field ? ef : nullptr, efg,
                                                    fl.forces ? fo : nullptr, low ? rs.low.fpart : nullptr,
                                                    low ? (rs.low.tc ? tc4::NQ : LK_SPLIT) : 0);
    prof->end(nk);
}

}  // namespace mdff
